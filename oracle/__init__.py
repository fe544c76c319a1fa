"""CPU parity oracle for paragram_b200 (test infrastructure, not the product)."""
