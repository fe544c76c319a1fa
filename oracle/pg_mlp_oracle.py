"""CPU restatement of the learned search-radius model (features, MLP, Adam).

TEST INFRASTRUCTURE ONLY: imported by ``tests/`` and never by the
``paragram_b200`` product, which runs these steps as CUDA kernels
(``paragram_b200/csrc/pg_mlp.cu``).

The learned model has no counterpart in the reference (it builds every cell
with a kNN warm start and a shrinking-radius traversal,
``csrc/laguerre/voronoi_ultra.cu:39-141``); this file is the specification the
kernels are checked against:

* ``features``: 16 features per point from its curve-order window (the 16
  points before and after it in the sorted order of its cloud);
* ``forward`` / ``loss_and_grads``: a 16 -> 64 -> 64 -> 2 MLP with BF16
  weights and activations (round to nearest even) and FP32 accumulation,
  gradients by the chain rule with the BF16 roundings passed straight through
  (the same rounding points as the kernels);
* ``adam``: one Adam step (Kingma and Ba, 2015) on FP32 master weights.
"""

from __future__ import annotations

import numpy as np

NFEAT = 16
HIDDEN = 64
NOUT = 2
HALF_WINDOW = 16
#: flat parameter layout: (name, shape) in order
LAYOUT = [("w1", (HIDDEN, NFEAT)), ("b1", (HIDDEN,)), ("w2", (HIDDEN, HIDDEN)), ("b2", (HIDDEN,)),
          ("w3", (NOUT, HIDDEN)), ("b3", (NOUT,))]
NPARAM = sum(int(np.prod(s)) for _, s in LAYOUT)


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(params: np.ndarray) -> dict:
    out, k = {}, 0
    for name, shape in LAYOUT:
        size = int(np.prod(shape))
        out[name] = params[k:k + size].reshape(shape)
        k += size
    return out


def features(sorted_pts: np.ndarray, sorted_w: np.ndarray | None, cloud_off: np.ndarray) -> np.ndarray:
    """Features [N, 16] per sorted slot (float64); rows of points without a distinct neighbour are 0."""
    p = sorted_pts.astype(np.float64)
    n = len(p)
    w = np.zeros(n) if sorted_w is None else sorted_w.astype(np.float64)
    out = np.zeros((n, NFEAT))
    for c in range(len(cloud_off) - 1):
        c0, c1 = int(cloud_off[c]), int(cloud_off[c + 1])
        if c1 <= c0:
            continue
        mn, mx = p[c0:c1].min(0), p[c0:c1].max(0)
        ext = np.maximum(mx - mn, 1e-20)
        ls = np.log(np.prod(ext) / (c1 - c0)) / 3.0
        for i in range(c0, c1):
            lo, hi = max(c0, i - HALF_WINDOW), min(c1 - 1, i + HALF_WINDOW)
            js = np.array([j for j in range(lo, hi + 1) if j != i], dtype=np.int64)
            if len(js) == 0:
                continue
            off = p[js] - p[i]
            d = np.sqrt((off * off).sum(1))
            ok = d > 0
            if not ok.any():
                continue
            dv, ov, wv = d[ok], off[ok], w[js][ok]
            order = np.argsort(dv, kind="stable")[:8]
            near = dv[order]
            m = len(near)
            near8 = np.concatenate([near, np.full(8 - m, near[-1])])
            logd = np.log(near8)
            lref = logd.mean()
            dref = np.exp(lref)
            f = out[i]
            f[:8] = logd - lref
            f[8] = lref - ls
            f[9] = (w[i] - wv.mean()) / (dref * dref)
            box = np.vstack([p[i][None], p[js]])
            e = np.sort(np.maximum(box.max(0) - box.min(0), 1e-6 * dref))
            f[10:13] = np.log(e) - lref
            f[13] = np.linalg.norm(ov[order].sum(0)) / (m * dref)
            face = min((p[i] - mn).min(), (mx - p[i]).min())
            f[14] = np.log(max(face, 1e-6 * dref)) - lref
            f[15] = np.count_nonzero(dv <= 2.0 * dref) / 32.0
    return out


def _r(x, rounding):
    return bf16(np.asarray(x, dtype=np.float32)).astype(np.float64) if rounding else np.asarray(x, np.float64)


def forward(x: np.ndarray, params: np.ndarray, mean: np.ndarray, scale: np.ndarray, keep: bool = False,
            rounding: bool = True):
    """Outputs [B, 2] (float64) of the MLP on raw features x [B, 16] (rounding=False: exact arithmetic)."""
    P = unpack(params)
    w1, w2, w3 = (_r(P[k], rounding) for k in ("w1", "w2", "w3"))
    xn = _r((x - mean) * scale, rounding)
    a1 = xn @ w1.T + P["b1"]
    h1 = _r(np.maximum(a1, 0.0), rounding)
    a2 = h1 @ w2.T + P["b2"]
    h2 = _r(np.maximum(a2, 0.0), rounding)
    y = h2 @ w3.T + P["b3"]
    if keep:
        return y, (xn, a1, h1, a2, h2, w2, w3)
    return y


def loss_and_grads(x, t, sw, params, mean, scale, tmean, tscale, total=None, rounding: bool = True):
    """Loss and flat gradient [NPARAM] of L = sum_s sw_s |y_s - t'_s|^2 / (2 total), t' = (t - tmean) * tscale,
    total = max(sum sw, 1) unless given."""
    y, (xn, a1, h1, a2, h2, w2, w3) = forward(x, params, mean, scale, keep=True, rounding=rounding)
    tn = (t - tmean) * tscale
    tot = max(float(sw.sum()), 1.0) if total is None else total
    r = y - tn
    loss = float((sw[:, None] * r * r).sum() / (2.0 * tot))
    dy = _r(sw[:, None] * r / tot, rounding)
    dh2 = _r((dy @ w3) * (a2 > 0), rounding)
    dh1 = _r((dh2 @ w2) * (a1 > 0), rounding)
    g = {
        "w3": dy.T @ h2, "b3": dy.sum(0),
        "w2": dh2.T @ h1, "b2": dh2.sum(0),
        "w1": dh1.T @ xn, "b1": dh1.sum(0),
    }
    return loss, np.concatenate([g[name].ravel() for name, _ in LAYOUT])


def adam(params, grad, m, v, step, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam step; returns (params, m, v) as float64 arrays."""
    m = beta1 * m + (1.0 - beta1) * grad
    v = beta2 * v + (1.0 - beta2) * grad * grad
    mh = m / (1.0 - beta1 ** step)
    vh = v / (1.0 - beta2 ** step)
    return params - lr * mh / (np.sqrt(vh) + eps), m, v
