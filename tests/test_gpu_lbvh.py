"""Invariants of the LBVH that pg_build leaves in its workspace (read through
pg_workspace_tree): the sorted points are a permutation of the input, every
sorted slot lies in exactly one leaf of its own cloud's tree, every child box in
a record is the exact bounding box of the child's points and its weight field
their maximum weight, and leaves hold at most the leaf size."""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _build(points, weights, cloud_offsets, leaf_size, dev):
    from paragram_b200 import _lib

    lib = _lib.load()
    n, clouds = len(points), len(cloud_offsets) - 1
    p = torch.from_numpy(points).to(dev)
    w = None if weights is None else torch.from_numpy(weights).to(dev)
    size = ctypes.c_size_t(0)
    assert lib.pg_batch_workspace_size(n, clouds, ctypes.byref(size)) == 0
    ws = torch.empty(size.value, dtype=torch.uint8, device=dev)
    offsets = torch.empty(n + 1, dtype=torch.int32, device=dev)
    status = torch.empty(n, dtype=torch.int32, device=dev)
    coff = torch.tensor(cloud_offsets, dtype=torch.int32, device=dev)
    opt = _lib.PgOptions(8, leaf_size, 0, 0, 0)
    e = ctypes.c_int64(0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = lib.pg_build_batch(n, clouds, coff.data_ptr(), p.data_ptr(), None if w is None else w.data_ptr(),
                            ctypes.byref(opt), ws.data_ptr(), size.value, offsets.data_ptr(), status.data_ptr(),
                            ctypes.byref(e), stream)
    assert rc == 0, _lib.last_error(lib)
    torch.cuda.synchronize()
    out = (ctypes.c_int64 * 5)()
    assert lib.pg_workspace_tree(n, clouds, out, 5) == 0
    raw = ws.cpu().numpy()
    o = list(out)
    spts = raw[o[0]:o[0] + 16 * n].view(np.float32).reshape(n, 4)
    order = raw[o[1]:o[1] + 4 * n].view(np.int32)
    rec = raw[o[2]:o[2] + 64 * max(n - 1, 1)].view(np.float32).reshape(-1, 16)
    roots = raw[o[3]:o[3] + 4 * clouds].view(np.int32)
    return spts, order, rec, roots


def _check_tree(points, weights, cloud_offsets, leaf_size, spts, order, rec, roots):
    n = len(points)
    wts = np.zeros(n, np.float32) if weights is None else weights
    # the sorted points are the input points, permuted
    assert np.array_equal(np.sort(order), np.arange(n))
    assert np.array_equal(spts[:, :3], points[order])
    assert np.array_equal(spts[:, 3], wts[order])
    recref = rec.view(np.int32)
    seen = np.zeros(n, np.int32)
    max_leaf = leaf_size if leaf_size > 0 else 16  # the default leaf size

    def leaf_range(r):
        return r & 0x3FFFFFF, ((r >> 26) & 31) + 1

    for c in range(len(cloud_offsets) - 1):
        lo_slot, hi_slot = cloud_offsets[c], cloud_offsets[c + 1]
        if hi_slot == lo_slot:
            continue
        # clouds are contiguous in the sorted order too
        assert set(order[lo_slot:hi_slot].tolist()) == set(range(lo_slot, hi_slot))
        root = int(roots[c])
        stack = [root]
        while stack:
            r = stack.pop()
            if r < 0:
                f, k = leaf_range(r)
                assert lo_slot <= f and f + k <= hi_slot and k <= max_leaf
                seen[f:f + k] += 1
                continue
            for side in (0, 1):
                box = rec[r, 0:6] if side == 0 else rec[r, 6:12]
                ref = int(recref[r, 12 + side])
                maxw = rec[r, 14 + side]
                # the child's points
                sub, todo = [], [ref]
                while todo:
                    x = todo.pop()
                    if x < 0:
                        f, k = leaf_range(x)
                        sub.append(np.arange(f, f + k))
                    else:
                        todo += [int(recref[x, 12]), int(recref[x, 13])]
                idx = np.concatenate(sub)
                pts = spts[idx]
                assert np.array_equal(box[:3], pts[:, :3].min(axis=0)), (r, side)
                assert np.array_equal(box[3:6], pts[:, :3].max(axis=0)), (r, side)
                assert maxw == pts[:, 3].max(), (r, side)
                stack.append(ref)
    assert (seen == 1).all()


@pytest.mark.parametrize("leaf_size", [-1, 1, 8, 32])
def test_lbvh_single_cloud(dev, leaf_size):
    from paragram_b200 import workloads as W

    pts, w = W.power_uniform(3000, seed=11)
    spts, order, rec, roots = _build(pts, w, [0, len(pts)], leaf_size, dev)
    _check_tree(pts, w, [0, len(pts)], leaf_size, spts, order, rec, roots)


def test_lbvh_batch_of_clouds(dev):
    from paragram_b200 import workloads as W

    rng = np.random.default_rng(12)
    sizes = [1, 2, 5, 16, 17, 33, 700, 1500]  # around the default leaf size of 16 and above it
    clouds = [W.uniform(s, seed=int(rng.integers(1 << 30))) for s in sizes]
    pts = np.concatenate(clouds).astype(np.float32)
    coff = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64).tolist()
    spts, order, rec, roots = _build(pts, None, coff, -1, dev)
    _check_tree(pts, None, coff, -1, spts, order, rec, roots)


def test_lbvh_duplicates(dev):
    # coincident points (equal Morton codes): the tree still covers every point once
    rng = np.random.default_rng(13)
    base = rng.random((200, 3)).astype(np.float32)
    pts = np.repeat(base, 5, axis=0)
    spts, order, rec, roots = _build(pts, None, [0, len(pts)], -1, dev)
    _check_tree(pts, None, [0, len(pts)], -1, spts, order, rec, roots)
