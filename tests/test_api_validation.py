"""Python API argument validation mirrors paragram/_api.py:16-62 (no GPU needed)."""

import pytest
import torch

import paragram_b200 as pg
from paragram_b200 import _api


def test_points_type_and_device():
    with pytest.raises(TypeError, match="points must be a torch.Tensor"):
        pg.voronoi_diagram([[0.0, 0.0, 0.0]])
    with pytest.raises(ValueError, match="points must be on a CUDA device"):
        pg.voronoi_diagram(torch.zeros(4, 3))
    with pytest.raises(ValueError, match="points must be on a CUDA device"):
        pg.power_diagram(torch.zeros(4, 3), torch.zeros(4))


def test_weights_validation_order():
    with pytest.raises(TypeError, match="weights must be a torch.Tensor"):
        _api._validate_weights([0.0], 1, torch.device("cuda:0"))
    with pytest.raises(ValueError, match="weights must be on a CUDA device"):
        _api._validate_weights(torch.zeros(4), 4, torch.device("cuda:0"))


def test_initial_guess_pairing():
    with pytest.raises(ValueError, match="must be provided together"):
        _api._validate_initial_guesses(torch.zeros(3, dtype=torch.int32), None, 2, torch.device("cuda:0"))
    with pytest.raises(ValueError, match="must be on a CUDA device"):
        _api._validate_initial_guesses(torch.zeros(3, dtype=torch.int32), torch.zeros(3, dtype=torch.int32), 2,
                                       torch.device("cuda:0"))
    assert _api._validate_initial_guesses(None, None, 5, torch.device("cuda:0")) == (None, None)


def test_diagram_is_frozen():
    d = pg.Diagram(torch.zeros(0), torch.zeros(1), torch.zeros(0))
    with pytest.raises(Exception):
        d.adjacency = torch.zeros(1)
