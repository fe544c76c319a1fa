"""GPU tests of the learned search radius: the feature, forward, gradient and
Adam kernels against the CPU oracle (oracle/pg_mlp_oracle.py), training on the
GPU, and builds with the model (identical diagrams, reported fallback rate).

Tolerances: features 2e-4 absolute (FP32 vs FP64 distances and logs) on all
but a few points whose 8th / 9th nearest window distances tie; network
outputs and gradients within 3e-2 (BF16 activations may round to the other
neighbour when FP32 and FP64 sums straddle a rounding boundary).
"""

import numpy as np
import pytest
import torch

from oracle import pg_mlp_oracle as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _cloud(seed, n=6000):
    from paragram_b200 import workloads as W

    return W.clustered(n, seed=seed)


def test_features_match_oracle(dev):
    import paragram_b200.cuda as pc
    from paragram_b200 import workloads as W

    for pts, w in ((_cloud(1), None), W.power_uniform(3000, seed=2)):
        t = torch.from_numpy(pts).to(dev)
        tw = None if w is None else torch.from_numpy(w).to(dev)[:, None]
        _, st = pc.build_with_stats(t, tw, features=True)
        order = st["order"].cpu().numpy()
        got = st["features"].cpu().numpy()[order]
        assert sorted(order.tolist()) == list(range(len(pts)))
        exp = M.features(pts[order], None if w is None else w[order], np.array([0, len(pts)]))
        bad = np.abs(got - exp).max(1) > 2e-4
        assert bad.mean() < 0.01, (bad.sum(), np.abs(got - exp).max(0))


def _model(dev, seed=0):
    from paragram_b200 import learned

    m = learned.Model(dev, seed=seed)
    rng = np.random.default_rng(seed)
    m._header(rng.normal(0, 0.5, 16).astype(np.float32), rng.uniform(0.5, 2, 16).astype(np.float32),
              np.array([0.3, 1.0], np.float32), np.array([2.0, 0.7], np.float32), 0.1)
    return m


def test_forward_matches_oracle(dev):
    m = _model(dev, 3)
    x = np.random.default_rng(4).normal(0, 1, (5000, 16)).astype(np.float32)
    got = m.predict(torch.from_numpy(x).to(dev)).cpu().numpy()
    exp = M.forward(x.astype(np.float64), m.params.cpu().numpy().astype(np.float64), m.feat_mean, m.feat_scale)
    err = np.abs(got - exp)
    assert err.max() < 3e-2 * (1 + np.abs(exp).max()), err.max()
    assert np.median(err) < 1e-3


@pytest.mark.parametrize("n", [64, 1000, 6001])
def test_gradient_matches_oracle(dev, n):
    """Gradient check of the training kernel (pg_mlp_grad) against the CPU oracle."""
    m = _model(dev, 5)
    rng = np.random.default_rng(n)
    x = rng.normal(0, 1, (n, 16)).astype(np.float32)
    t = rng.normal(0, 1, (n, 2)).astype(np.float32)
    sw = (rng.random(n) > 0.1).astype(np.float32)
    loss, g = m.loss_and_grad(torch.from_numpy(x).to(dev), torch.from_numpy(t).to(dev), torch.from_numpy(sw).to(dev))
    g = g.cpu().numpy().astype(np.float64)
    el, eg = M.loss_and_grads(x.astype(np.float64), t.astype(np.float64), sw.astype(np.float64),
                              m.params.cpu().numpy().astype(np.float64), m.feat_mean, m.feat_scale,
                              m.target_mean, m.target_scale)
    assert abs(float(loss[0]) - el) <= 1e-3 * el + 1e-6
    assert np.linalg.norm(g - eg) <= 3e-2 * np.linalg.norm(eg), np.linalg.norm(g - eg) / np.linalg.norm(eg)
    for name, lo, hi in (("w1", 0, 1024), ("b1", 1024, 1088), ("w2", 1088, 5184), ("b2", 5184, 5248),
                         ("w3", 5248, 5376), ("b3", 5376, 5378)):
        assert np.linalg.norm(g[lo:hi] - eg[lo:hi]) <= 5e-2 * np.linalg.norm(eg[lo:hi]) + 1e-7, name


def test_adam_step_matches_oracle(dev):
    m = _model(dev, 7)
    rng = np.random.default_rng(8)
    x = torch.from_numpy(rng.normal(0, 1, (512, 16)).astype(np.float32)).to(dev)
    t = torch.from_numpy(rng.normal(0, 1, (512, 2)).astype(np.float32)).to(dev)
    w = torch.ones(512, device=dev)
    p0 = m.params.cpu().numpy().astype(np.float64)
    m.loss_and_grad(x, t, w)
    g = m.grad.cpu().numpy().astype(np.float64)
    m.adam_step(1e-3)
    p1, mm, vv = M.adam(p0, g, np.zeros_like(p0), np.zeros_like(p0), 1, 1e-3)
    assert np.allclose(m.params.cpu().numpy(), p1, rtol=1e-5, atol=1e-7)
    assert np.allclose(m.m.cpu().numpy(), mm, rtol=1e-5, atol=1e-12)
    # the packed model holds the new weights
    y = m.predict(x).cpu().numpy()
    exp = M.forward(x.cpu().numpy().astype(np.float64), m.params.cpu().numpy().astype(np.float64), m.feat_mean,
                    m.feat_scale)
    assert np.abs(y - exp).max() < 3e-2 * (1 + np.abs(exp).max())


def test_training_and_learned_build(dev, oracle):
    """Training lowers the loss; a calibrated model predicts most radii; a build with it equals the
    plain build (and the oracle), and its fallback rate is what the calibration promised. An
    untrained model with the same margin falls back more often: what training gains (the cap saves
    no traversal work over the plain best-first search, which already stops at the final radius)."""
    import paragram_b200 as pg
    import paragram_b200.cuda as pc
    from paragram_b200 import learned

    train = [learned.collect(torch.from_numpy(_cloud(s, 30000)).to(dev)) for s in (11, 12)]
    log = []
    model = learned.train(train, epochs=6, batch=4096, log=log)
    assert log[-1] < 0.85 * log[0], log  # the targets' normalised variance is 1 per output
    margin = model.calibrate(train[0], quantile=0.97)
    held = learned.collect(torch.from_numpy(_cloud(13, 30000)).to(dev))
    assert model.hit_rate(held) > 0.9

    pts = _cloud(14, 20000)
    t = torch.from_numpy(pts).to(dev)
    plain = pg.voronoi_diagram(t)
    d = learned.voronoi_diagram(t, model)
    assert torch.equal(d.adjacency, plain.adjacency) and torch.equal(d.offsets, plain.offsets)
    assert torch.equal(d.status, plain.status)
    oa, oo, os_ = oracle.diagram(pts)
    assert np.array_equal(d.adjacency.cpu().numpy(), oa) and np.array_equal(d.status.cpu().numpy(), os_)

    _, st = pc.build_with_stats(t, model=model.blob)
    fallback = st["hint_misses"] / len(pts)
    assert fallback < 0.1, fallback
    untrained = learned.Model(dev, seed=99)
    untrained._header(model.feat_mean, model.feat_scale, model.target_mean, model.target_scale, margin)
    _, st0 = pc.build_with_stats(t, model=untrained.blob)
    # an untrained network with the same calibration predicts about a constant radius: it falls back more
    assert st0["hint_misses"] > 1.3 * st["hint_misses"], (st0["hint_misses"], st["hint_misses"])

    wpts, ww = __import__("paragram_b200.workloads", fromlist=["power_uniform"]).power_uniform(8000, seed=15)
    tw = torch.from_numpy(ww).to(dev)
    dp = learned.power_diagram(torch.from_numpy(wpts).to(dev), tw, model)
    pp = pg.power_diagram(torch.from_numpy(wpts).to(dev), tw)
    assert torch.equal(dp.adjacency, pp.adjacency) and torch.equal(dp.status, pp.status)


def test_learned_routing(dev, oracle):
    """The model's neighbour-count output routes work: with route_degree set, the cells predicted at
    or above it skip the first pass (64 vertex slots) and are built by the 128-slot tier. The diagram
    is unchanged; a threshold that would route every cell stops at the routing share of the deferred
    rows (4096 + N / 128) instead of exhausting them."""
    import paragram_b200.cuda as pc
    from paragram_b200 import learned
    from paragram_b200 import workloads as W

    rng = np.random.default_rng(21)
    train = [learned.collect(torch.from_numpy(W.surface_cloud(40_000, rng)).to(dev)) for _ in range(3)]
    model = learned.train(train, epochs=4, batch=4096)
    model.calibrate(train[0], quantile=0.97)
    held = learned.collect(torch.from_numpy(W.surface_cloud(40_000, rng)).to(dev))
    ok = held.weights > 0
    pred = model.predicted_degree(held.features[ok]).cpu().numpy()
    true = held.targets[ok, 1].double().cpu().numpy() * 16.0
    assert np.corrcoef(pred, true)[0, 1] > 0.2  # the count output carries signal (weak on surfaces)

    pts = W.surface_cloud(60_000, rng)
    n = len(pts)
    t = torch.from_numpy(pts).to(dev)
    (a0, o0, s0), _ = pc.build_with_stats(t)
    # deferred cells of the learned build without routing: the cells its first pass gives up on
    model.set_route(0.0)
    pc.build_with_stats(t, model=model.blob, profile=True)
    base_deferred = pc.last_profile()["deferred_cells"]
    route_cap = 4096 + n // 128
    # a threshold that routes about 1% of the cells, and one that would route all of them
    some = float(np.quantile(model.predicted_degree(learned.collect(t).features).cpu().numpy(), 0.99))
    for thr, expect in ((some, "some"), (0.5, "capped")):
        model.set_route(thr)
        (a, o, s), st = pc.build_with_stats(t, model=model.blob, profile=True)
        deferred = pc.last_profile()["deferred_cells"]
        assert torch.equal(a, a0) and torch.equal(o, o0) and torch.equal(s, s0), thr
        # deferred = routed cells + the unrouted ones the first pass gives up on
        assert deferred > base_deferred, (thr, deferred, base_deferred)
        routed = pc.last_profile()["routed_cells"]
        assert 0 < routed <= deferred
        if expect == "capped":
            assert routed == route_cap
            assert route_cap <= deferred <= route_cap + base_deferred, (deferred, route_cap)
    oa, oo, os_ = oracle.diagram(pts)
    assert np.array_equal(a.cpu().numpy(), oa) and np.array_equal(o.cpu().numpy(), oo)
