"""Learned search radius: training data, training on the GPU, calibration, use.

A small MLP (16 -> 64 -> 64 -> 2, BF16 weights, FP32 accumulation) predicts,
from cheap features of a point's curve-order window, the certified radius of
its final cell and its neighbour count. The cell pass caps its first
traversal pass at the predicted radius and keeps the result only when the
final radius is within it (otherwise an unbounded pass completes the cell), so
the model changes the work, never the diagram. No reference counterpart: the
reference searches every cell with a kNN warm start and a shrinking radius
(csrc/laguerre/voronoi_ultra.cu:39-141).

All arithmetic runs in the library's kernels (include/paragram_b200.h:
features_out / radius_out of pg_build, pg_mlp_grad, pg_mlp_adam,
pg_mlp_forward, and the fused prediction of a build given a model); torch only
holds the device buffers and draws minibatches.

Typical use::

    data = [learned.collect(torch.from_numpy(W.clustered(1_000_000, seed=s)).cuda()) for s in (1, 2)]
    model = learned.train(data, epochs=4)
    model.calibrate(data[0], quantile=0.98)
    d = learned.voronoi_diagram(points, model)      # same Diagram as paragram_b200.voronoi_diagram
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._api import Diagram, _validate_initial_guesses, _validate_points, _validate_weights

NFEAT = 16
NPARAM = 5378
MODEL_BYTES = 11984
MAGIC = 0x314D4750
# byte offsets inside pg_model (include/paragram_b200.h)
_OFF_FEAT_MEAN, _OFF_FEAT_SCALE, _OFF_TMEAN, _OFF_TSCALE, _OFF_MARGIN, _OFF_ROUTE = 16, 80, 144, 152, 160, 164
_LAYOUT = [("w1", (64, 16)), ("b1", (64,)), ("w2", (64, 64)), ("b2", (64,)), ("w3", (2, 64)), ("b3", (2,))]


def _check(lib, rc):
    if rc != 0:
        raise RuntimeError(_lib.last_error(lib))


@dataclass
class Samples:
    """Training samples of one diagram: features [N, 16], targets [N, 2], weights [N] (device)."""

    features: torch.Tensor
    targets: torch.Tensor
    weights: torch.Tensor


def _log_spacing(points: torch.Tensor) -> float:
    """log of the cloud's mean spacing, (volume of its box / points)^(1/3) (feature f8's reference)."""
    p = points.double()
    ext = (p.max(0).values - p.min(0).values).clamp_min(1e-20)
    return float(torch.log(ext.prod() / points.shape[0]) / 3.0)


def collect(points: torch.Tensor, weights: Optional[torch.Tensor] = None) -> Samples:
    """Features and targets from one plain build (the method the model learns from).

    Targets: log(certified radius) - log(mean window distance) and degree / 16. Points without a
    distinct window neighbour and empty cells get weight 0.
    """
    from . import cuda as pc

    w = None if weights is None else weights.reshape(-1, 1)
    (a, o, s), st = pc.build_with_stats(points, w, diagnostics=True, features=True)
    f = st["features"]
    lref = f[:, 8].double() + _log_spacing(points)
    rad = st["radius"].double()
    ok = (rad > 0) & (f.abs().sum(1) > 0) & (s == 0)
    t0 = torch.where(ok, torch.log(rad.clamp_min(1e-30)) - lref, torch.zeros_like(rad))
    t1 = (o[1:] - o[:-1]).double() / 16.0
    return Samples(f.contiguous(), torch.stack([t0, t1], 1).float().contiguous(), ok.float().contiguous())


def _cat(samples: Sequence[Samples]) -> Samples:
    return Samples(torch.cat([s.features for s in samples]), torch.cat([s.targets for s in samples]),
                   torch.cat([s.weights for s in samples]))


class Model:
    """Master weights, Adam state and the packed device model (pg_model)."""

    def __init__(self, device: torch.device, seed: int = 0):
        self.device = torch.device(device)
        g = torch.Generator(device="cpu").manual_seed(seed)
        parts = []
        for name, shape in _LAYOUT:
            if name.startswith("w"):
                fan_in = shape[1]
                bound = math.sqrt(6.0 / fan_in) if name != "w3" else math.sqrt(1.0 / fan_in)
                parts.append((torch.rand(shape, generator=g) * 2 - 1).mul_(bound).reshape(-1))
            else:
                parts.append(torch.zeros(shape).reshape(-1))
        self.params = torch.cat(parts).to(self.device)
        self.m = torch.zeros(NPARAM, device=self.device)
        self.v = torch.zeros(NPARAM, device=self.device)
        self.grad = torch.zeros(NPARAM, device=self.device)
        self.loss_buf = torch.zeros(1, device=self.device)
        self.step = 0
        self.blob = torch.zeros(MODEL_BYTES, dtype=torch.uint8, device=self.device)
        self._header(np.zeros(16, np.float32), np.ones(16, np.float32), np.zeros(2, np.float32),
                     np.ones(2, np.float32), 0.0)
        lib = _lib.load()
        with torch.cuda.device(self.device):
            _check(lib, lib.pg_mlp_pack(self.params.data_ptr(), self.blob.data_ptr(), self._stream()))

    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def _header(self, mean, scale, tmean, tscale, margin, route_degree=None):
        if route_degree is None:
            route_degree = getattr(self, "route_degree", 0.0)
        head = np.zeros(176, dtype=np.uint8)
        head[0:16] = np.array([MAGIC, 16, 64, 0], dtype=np.uint32).view(np.uint8)
        head[_OFF_FEAT_MEAN:_OFF_FEAT_MEAN + 64] = np.asarray(mean, np.float32).view(np.uint8)
        head[_OFF_FEAT_SCALE:_OFF_FEAT_SCALE + 64] = np.asarray(scale, np.float32).view(np.uint8)
        head[_OFF_TMEAN:_OFF_TMEAN + 8] = np.asarray(tmean, np.float32).view(np.uint8)
        head[_OFF_TSCALE:_OFF_TSCALE + 8] = np.asarray(tscale, np.float32).view(np.uint8)
        head[_OFF_MARGIN:_OFF_MARGIN + 4] = np.asarray([margin], np.float32).view(np.uint8)
        head[_OFF_ROUTE:_OFF_ROUTE + 4] = np.asarray([route_degree], np.float32).view(np.uint8)
        self.blob[:176].copy_(torch.from_numpy(head))
        self.route_degree = float(route_degree)
        self.feat_mean, self.feat_scale = np.asarray(mean, np.float32), np.asarray(scale, np.float32)
        self.target_mean, self.target_scale = np.asarray(tmean, np.float32), np.asarray(tscale, np.float32)
        self.margin = float(margin)

    def set_normalization(self, data: Samples):
        """Feature and target normalisation (mean, 1 / std) from weighted samples."""
        wt = data.weights.double()
        tot = wt.sum().clamp_min(1.0)
        x = data.features.double()
        mean = (x * wt[:, None]).sum(0) / tot
        std = (((x - mean) ** 2 * wt[:, None]).sum(0) / tot).sqrt()
        scale = torch.where(std > 1e-6, 1.0 / std, torch.ones_like(std))
        t = data.targets.double()
        tmean = (t * wt[:, None]).sum(0) / tot
        tstd = (((t - tmean) ** 2 * wt[:, None]).sum(0) / tot).sqrt()
        tscale = torch.where(tstd > 1e-6, 1.0 / tstd, torch.ones_like(tstd))
        self._header(mean.float().cpu().numpy(), scale.float().cpu().numpy(), tmean.float().cpu().numpy(),
                     tscale.float().cpu().numpy(), self.margin)

    # ------------------------------------------------------------------ kernels
    def loss_and_grad(self, x: torch.Tensor, t: torch.Tensor, w: torch.Tensor, total: Optional[float] = None):
        """Loss and gradient [NPARAM] of a batch (pg_mlp_grad); the gradient is left in ``self.grad``."""
        lib = _lib.load()
        tot = float(w.sum()) if total is None else total
        self.grad.zero_()
        self.loss_buf.zero_()
        with torch.cuda.device(self.device):
            _check(lib, lib.pg_mlp_grad(x.shape[0], x.data_ptr(), t.data_ptr(), w.data_ptr(),
                                        1.0 / max(tot, 1.0), self.blob.data_ptr(), self.grad.data_ptr(),
                                        self.loss_buf.data_ptr(), self._stream()))
        return self.loss_buf, self.grad

    def adam_step(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8):
        lib = _lib.load()
        self.step += 1
        with torch.cuda.device(self.device):
            _check(lib, lib.pg_mlp_adam(self.params.data_ptr(), self.grad.data_ptr(), self.m.data_ptr(),
                                        self.v.data_ptr(), self.step, lr, beta1, beta2, eps, self.blob.data_ptr(),
                                        self._stream()))

    def predict(self, x: torch.Tensor) -> torch.Tensor:
        """Network outputs [N, 2] (normalised units) for raw features [N, 16] (pg_mlp_forward)."""
        lib = _lib.load()
        x = x.contiguous()
        out = torch.empty(max(x.shape[0], 1), 2, dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            _check(lib, lib.pg_mlp_forward(x.shape[0], x.data_ptr(), self.blob.data_ptr(), out.data_ptr(),
                                           self._stream()))
        return out[: x.shape[0]]

    def predicted_log_radius(self, x: torch.Tensor) -> torch.Tensor:
        """Predicted log(radius / window distance) without the margin."""
        y = self.predict(x)[:, 0].double()
        return y / float(self.target_scale[0]) + float(self.target_mean[0])

    def calibrate(self, data: Samples, quantile: float = 0.98) -> float:
        """Margin (added to the log radius) that covers ``quantile`` of the samples' radii."""
        ok = data.weights > 0
        res = (data.targets[ok, 0].double() - self.predicted_log_radius(data.features[ok]))
        margin = 0.0
        if res.numel():
            srt = torch.sort(res).values
            margin = float(srt[min(int(quantile * (srt.numel() - 1) + 0.5), srt.numel() - 1)])
        self._header(self.feat_mean, self.feat_scale, self.target_mean, self.target_scale, margin)
        return margin

    def set_route(self, degree: float = 0.0):
        """Route the cells whose predicted neighbour count is at least ``degree`` past the first pass
        (its 64 vertex slots) straight to the 128-slot tier; 0 turns routing off. A cell with more
        than 34 faces has more than 64 vertices, so thresholds in the mid thirties target the cells
        the first pass would give up on. The diagram never depends on it."""
        self._header(self.feat_mean, self.feat_scale, self.target_mean, self.target_scale, self.margin,
                     float(degree))

    def predicted_degree(self, x: torch.Tensor) -> torch.Tensor:
        """Predicted neighbour count for raw features [N, 16]."""
        y = self.predict(x)[:, 1].double()
        return (y / float(self.target_scale[1]) + float(self.target_mean[1])) * 16.0

    def hit_rate(self, data: Samples) -> float:
        """Fraction of cells whose certified radius lies within the calibrated prediction."""
        ok = data.weights > 0
        pred = self.predicted_log_radius(data.features[ok]) + self.margin
        return float((data.targets[ok, 0].double() <= pred).double().mean()) if ok.any() else 1.0

    def state_dict(self) -> dict:
        return {"params": self.params.cpu().numpy(), "feat_mean": self.feat_mean, "feat_scale": self.feat_scale,
                "target_mean": self.target_mean, "target_scale": self.target_scale, "margin": self.margin,
                "route_degree": self.route_degree}

    @classmethod
    def from_state(cls, state: dict, device) -> "Model":
        m = cls(device)
        m.params.copy_(torch.from_numpy(np.asarray(state["params"], np.float32)))
        m._header(state["feat_mean"], state["feat_scale"], state["target_mean"], state["target_scale"],
                  float(state["margin"]), float(state.get("route_degree", 0.0)))
        lib = _lib.load()
        with torch.cuda.device(m.device):
            _check(lib, lib.pg_mlp_pack(m.params.data_ptr(), m.blob.data_ptr(), m._stream()))
        return m


def train(data: Sequence[Samples] | Samples, *, epochs: int = 4, batch: int = 8192, lr: float = 2e-3,
          seed: int = 0, model: Optional[Model] = None, log: Optional[list] = None) -> Model:
    """Adam on the GPU (pg_mlp_grad + pg_mlp_adam) over shuffled minibatches; returns the model.

    ``log`` (a list) receives the mean minibatch loss of every epoch.
    """
    full = data if isinstance(data, Samples) else _cat(list(data))
    dev = full.features.device
    if model is None:
        model = Model(dev, seed=seed)
        model.set_normalization(full)
    gen = torch.Generator(device=dev).manual_seed(seed)
    n = full.features.shape[0]
    mean_w = float(full.weights.mean()) if n else 1.0  # minibatch loss normaliser without a host sync
    for ep in range(epochs):
        perm = torch.randperm(n, device=dev, generator=gen)
        tot_loss, nb = torch.zeros((), device=dev), 0
        for b0 in range(0, n, batch):
            idx = perm[b0:b0 + batch]
            x, t, w = full.features[idx], full.targets[idx], full.weights[idx]
            loss, _ = model.loss_and_grad(x, t, w, total=max(idx.numel() * mean_w, 1.0))
            model.adam_step(lr * (0.5 * (1 + math.cos(math.pi * (ep * n + b0) / (epochs * n)))))
            tot_loss += loss[0]
            nb += 1
        if log is not None:
            log.append(float(tot_loss) / max(nb, 1))
    return model


def _build(points, weights, model: Model, initial_guesses=None, initial_guesses_offsets=None):
    from . import cuda as pc

    w = None if weights is None else weights.reshape(-1, 1)
    g, go = _validate_initial_guesses(initial_guesses, initial_guesses_offsets, points.shape[0], points.device)
    return pc._run(points, w, 8, False, g, go, -1, model=model.blob)


def voronoi_diagram(points: torch.Tensor, model: Model, *, initial_guesses: Optional[torch.Tensor] = None,
                    initial_guesses_offsets: Optional[torch.Tensor] = None) -> Diagram:
    """``paragram_b200.voronoi_diagram`` with the learned search radius (identical result).

    ``initial_guesses`` / ``initial_guesses_offsets`` as in ``paragram_b200.voronoi_diagram`` (for
    instance the previous diagram of slightly moved points): the cells are clipped by them first,
    then searched with the learned radius."""
    points = _validate_points(points)
    a, o, s = _build(points, None, model, initial_guesses, initial_guesses_offsets)
    return Diagram(adjacency=a, offsets=o, status=s)


def power_diagram(points: torch.Tensor, weights: torch.Tensor, model: Model, *,
                  initial_guesses: Optional[torch.Tensor] = None,
                  initial_guesses_offsets: Optional[torch.Tensor] = None) -> Diagram:
    """``paragram_b200.power_diagram`` with the learned search radius (identical result)."""
    points = _validate_points(points)
    weights = _validate_weights(weights, points.shape[0], points.device)
    a, o, s = _build(points, weights, model, initial_guesses, initial_guesses_offsets)
    return Diagram(adjacency=a, offsets=o, status=s)
