"""Multi-process plumbing of the weak-scaling run on CPU (gloo, world size 2)."""

import os

import pytest
import torch.multiprocessing as mp


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from paragram_b200 import dist

    r, w, _ = dist.init("gloo", timeout_s=60)
    b, e = dist.shard_range(256, r, w)
    mx = dist.reduce_max(float(r + 1))
    tot = dist.reduce_sum(float(e - b))
    dist.barrier()
    dist.finalize()
    q.put((r, b, e, mx, tot))


def test_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29000 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1:3] == (0, 128) and res[1][1:3] == (128, 256)
    assert all(r[3] == 2.0 and r[4] == 256.0 for r in res)


@pytest.mark.parametrize("n,world", [(10, 3), (256, 8), (5, 8)])
def test_shard_range_partitions(n, world):
    from paragram_b200 import dist

    spans = [dist.shard_range(n, r, world) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == n
    assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
    assert max(e - b for b, e in spans) - min(e - b for b, e in spans) <= 1


def _exchange_worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import torch

    from paragram_b200 import dist, sharded

    r, w, _ = dist.init("gloo", timeout_s=60)
    # ranks contribute packs of different lengths (rank 1: empty), as the sharded build's row exchange does
    local = torch.arange(10 * r, 10 * r + [5, 0, 7][r], dtype=torch.int32)
    got = sharded.exchange(local)
    pts = sharded.exchange(torch.full((3 * (r + 1),), float(r)))
    dist.barrier()
    dist.finalize()
    q.put((r, [g.tolist() for g in got], [p.tolist() for p in pts]))


def test_sharded_exchange_gloo_world3():
    """The all-gather of variable-length packs behind the sharded build: every rank receives every
    rank's tensor, in rank order, with its own length (an empty one included)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_exchange_worker, args=(r, 3, port, q)) for r in range(3)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = [list(range(0, 5)), [], list(range(20, 27))]
    for _, got, pts in res:
        assert got == expect
        assert pts == [[0.0] * 3, [1.0] * 6, [2.0] * 9]


@pytest.mark.parametrize("n,parts", [(10, 3), (5_000_000, 8), (2, 4), (0, 2)])
def test_cell_ranges_partition(n, parts):
    from paragram_b200 import sharded

    spans = sharded.cell_ranges(n, parts)
    assert len(spans) == parts and spans[0][0] == 0 and spans[-1][1] == n
    assert all(spans[i][1] == spans[i + 1][0] for i in range(parts - 1))
    assert max(e - b for b, e in spans) - min(e - b for b, e in spans) <= 1
