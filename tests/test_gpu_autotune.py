"""The autotuner times the performance knobs on the device and returns the fastest; the knobs never
change the diagram."""

import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def test_tune_single_cloud(dev):
    import paragram_b200 as pg
    import paragram_b200.cuda as pc
    from paragram_b200 import autotune
    from paragram_b200 import workloads as W

    t = torch.from_numpy(W.clustered(20000, seed=31)).to(dev)
    best = autotune.tune(t, reps=1, leaf_sizes=(8, 16), blocks_per_sm=(2, 3), key="test-single")
    assert len(best["trials"]) == 4 and best["ms"] == min(x["ms"] for x in best["trials"])
    assert best["leaf_size"] in (8, 16) and best["blocks_per_sm"] in (2, 3)
    again = autotune.tune(t, reps=1, leaf_sizes=(8, 16), blocks_per_sm=(2, 3), key="test-single")
    assert again == best  # cached per device and sample signature
    ref = pg.voronoi_diagram(t)
    a, o, s = pc._run(t, None, 8, False, None, None, best["leaf_size"], blocks_per_sm=best["blocks_per_sm"])
    assert torch.equal(a, ref.adjacency) and torch.equal(o, ref.offsets) and torch.equal(s, ref.status)


def test_tune_batch(dev):
    import paragram_b200 as pg
    from paragram_b200 import autotune
    from paragram_b200 import workloads as W

    clouds = [torch.from_numpy(c).to(dev) for c in W.surface_clouds(num_clouds=3, seed=32, size_scale=0.01)]
    best = autotune.tune(clouds, reps=1, leaf_sizes=(12, 24), blocks_per_sm=(2,), key="test-batch")
    assert len(best["trials"]) == 2
    out = pg.build_batch(clouds, leaf_size=best["leaf_size"], blocks_per_sm=best["blocks_per_sm"])
    for c, d in zip(clouds, out):
        ref = pg.voronoi_diagram(c)
        assert torch.equal(d.adjacency, ref.adjacency) and torch.equal(d.status, ref.status)


def test_tune_chunks_and_routing(dev):
    """Chunk counts and, with a learned model, routing thresholds are knobs too: every trial gives
    the same diagram, and the model is left with the fastest threshold."""
    import paragram_b200 as pg
    import paragram_b200.cuda as pc
    from paragram_b200 import autotune, learned
    from paragram_b200 import workloads as W

    model = learned.train([learned.collect(torch.from_numpy(W.clustered(20000, seed=33)).to(dev))], epochs=1)
    model.calibrate(learned.collect(torch.from_numpy(W.clustered(20000, seed=34)).to(dev)))
    t = torch.from_numpy(W.clustered(20000, seed=35)).to(dev)
    best = autotune.tune(t, reps=1, leaf_sizes=(16,), blocks_per_sm=(2,), num_chunks=(1, 3), model=model,
                         route_degrees=(0.0, 30.0), key="test-knobs")
    assert len(best["trials"]) == 4
    assert best["num_chunks"] in (1, 3) and best["route_degree"] in (0.0, 30.0)
    assert model.route_degree == best["route_degree"]
    ref = pg.voronoi_diagram(t)
    for tr in best["trials"]:
        model.set_route(tr["route_degree"])
        a, o, s = pc._run(t, None, 8, False, None, None, tr["leaf_size"], num_chunks=tr["num_chunks"],
                          blocks_per_sm=tr["blocks_per_sm"], model=model.blob)
        assert torch.equal(a, ref.adjacency) and torch.equal(o, ref.offsets) and torch.equal(s, ref.status)
