"""Helpers shared by the GPU test modules (not a test module itself)."""

import numpy as np


def diff_cells(got, exp):
    """Indices of the cells whose status or sorted row differ between two (adjacency, offsets, status)."""
    adj, off, st = got
    eadj, eoff, est = exp
    deg, edeg = np.diff(off.astype(np.int64)), np.diff(eoff.astype(np.int64))
    bad = (st != est) | (deg != edeg)
    same = ~bad
    # rows of cells with equal degree: compare entry by entry
    rows = np.repeat(np.arange(len(st)), deg)
    erows = np.repeat(np.arange(len(st)), edeg)
    a, b = adj[same[rows]], eadj[same[erows]]
    r = rows[same[rows]]
    if a.size:
        bad[np.unique(r[a != b])] = True
    return np.flatnonzero(bad)
