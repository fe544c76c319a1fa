"""Benchmark: Mcells/s of 3D diagram construction on B200.

Default workload (the headline configuration): Voronoi diagram of N = 5,000,000
clustered points (90% from 64 truncated isotropic Gaussians, sigma log-uniform
in [0.005, 0.1], 10% uniform background), seeded synthetic data, built with the
learned search radius (a model trained before timing on two 1M-point clouds of
disjoint seeds) and FP32-filtered predicates; the plain build (no model) of the
same points is timed beside it. One step is one full build (LBVH, prediction,
cell clipping, CSR, adjacency) on device-resident points; ``e2e`` repeats the
step through the public API from pinned host memory, with the host->device
copy of the points and the device->host copy of the Diagram inside the timed
region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload NAME]

Workloads: clustered_voronoi_5m (default), clustered_voronoi_500k,
uniform_voronoi_100k, uniform_power_1m, lattice_power_310 (29.8M-point jittered
lattice, power: learned radius + batched CUDA-graph build, plain beside it;
``--plain`` for the single-cloud plain build), surface_batch_256 (256 surface
clouds in one CUDA-graph batch), moving_uniform_1m (iterations over 1M uniform
points that move by 1% of their spacing between steps, each rebuilt with the
previous step's diagram as initial guesses; the cold rebuild timed beside it).

For N > 1 (torch.distributed.run, one process per GPU) every rank builds its
own diagram of an equally sized, differently seeded point set (weak scaling;
cells shard without any data exchange) and the step time is the max over
ranks. ``--sharded`` times strong scaling instead: one diagram of the workload
built by all ranks together (point all-gather, a range of cells per rank, row
all-gather, the CSR on every rank). ``--impl reference`` times the reference's own CUDA extension
(``oracle/_ref``: its unmodified sources compiled with a project-written
stand-in for its absent cuBQL dependency) on the same workload, counting its
construction phase (cells + CSR) by its own timers; without that build or a
GPU (or with ``--reference-cpu``) it times the CPU restatement of the
reference's construction (the parity oracle, all host threads) on a bounded
sample of the workload.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
PROFILE_SUMMARY = os.path.join(ROOT, "profiles", "k_cells_fast_clustered5m.txt")

WORKLOADS = {
    "clustered_voronoi_5m": dict(kind="clustered", n=5_000_000, weighted=False),
    "clustered_voronoi_500k": dict(kind="clustered", n=500_000, weighted=False),
    "uniform_voronoi_100k": dict(kind="uniform", n=100_000, weighted=False),
    "uniform_power_1m": dict(kind="power", n=1_000_000, weighted=True),
    "lattice_power_310": dict(kind="lattice", n=310 ** 3, weighted=True),
    "surface_batch_256": dict(kind="surfaces", n=256, weighted=False),
    "surface_cloud_500k": dict(kind="surface", n=500_000, weighted=False),
    "moving_uniform_1m": dict(kind="moving", n=1_000_000, weighted=False),
}
#: workloads built with the learned search radius (plain build timed beside them)
LEARNED = {"clustered_voronoi_5m", "clustered_voronoi_500k"}


def make_points(spec: dict, seed: int):
    from paragram_b200 import workloads as W

    k = spec["kind"]
    if k == "clustered":
        return W.clustered(spec["n"], seed=seed), None
    if k == "uniform":
        return W.uniform(spec["n"], seed=seed), None
    if k == "power":
        return W.power_uniform(spec["n"], seed=seed)
    if k == "lattice":
        return W.jittered_lattice(round(spec["n"] ** (1 / 3)), seed=seed)
    if k == "surfaces":
        return W.surface_clouds(num_clouds=spec["n"], seed=seed), None
    if k == "surface":
        return W.surface_cloud(spec["n"], np.random.default_rng(seed)), None
    if k == "moving":
        return W.uniform(spec["n"], seed=seed), None
    raise ValueError(k)


def moved_points(pts, seed: int):
    """The moving workload's second point set: every point displaced by a Gaussian step of 1% of the
    mean spacing of a unit-cube cloud of that size."""
    rng = np.random.default_rng(7 + seed)
    step_len = 0.01 * (1.0 / pts.shape[0]) ** (1.0 / 3.0)
    return (pts + step_len * rng.standard_normal(pts.shape)).astype(np.float32)


def train_model(dev, seed: int):
    """Learned search radius trained on two 1M-point clustered clouds of other seeds (GPU kernels)."""
    import torch

    from paragram_b200 import learned
    from paragram_b200 import workloads as W

    t0 = time.perf_counter()
    data = [learned.collect(torch.from_numpy(W.clustered(1_000_000, seed=1000 + 2 * seed + k)).to(dev))
            for k in range(2)]
    log = []
    model = learned.train(data, epochs=4, batch=8192, log=log)
    margin = model.calibrate(data[0], quantile=0.98)
    torch.cuda.synchronize(dev)
    return model, {"train_s": time.perf_counter() - t0, "train_samples": sum(int(d.weights.sum()) for d in data),
                   "loss_per_epoch": [round(x, 4) for x in log], "margin": margin, "calibration_quantile": 0.98}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while active."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._first = threading.Event()
        self._thr = None

    def _run(self):
        try:
            p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                                  "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                 stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self._first.set()
            return
        try:
            while not self._stop.is_set():
                line = p.stdout.readline()
                if not line:
                    break
                self.samples.append([x.strip() for x in line.split(",")])
                self._first.set()
        finally:
            self._first.set()
            p.kill()
            p.wait()

    def __enter__(self):
        self._thr = threading.Thread(target=self._run, daemon=True)
        self._thr.start()
        # the sampler's start-up (driver initialisation) must not overlap the first timed step:
        # wait for its first sample and a moment more
        self._first.wait(timeout=10)
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._thr.join(timeout=5)

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                sm.append(float(s[1]))
                mx = float(s[2])
                for k, v in zip(names, s[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(k)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def algorithmic_work(offsets: np.ndarray, weighted: bool) -> tuple[float, float]:
    """(FP32 flops, compulsory bytes) of a diagram from its output degrees.

    Per cell with degree d: F = d * (20 + 8 * max(8, 2d - 4) + 6 * 38) flops (one
    clip per final face: bisector, side tests against 2d - 4 vertices, about six
    new vertices by 3x3 cofactors) and B = 12 + 4 [weighted] + 4 + 4 + 4d bytes
    (point in, weight in, status and offset out, adjacency out).
    """
    d = np.diff(offsets.astype(np.int64)).astype(np.float64)
    flops = float(np.sum(d * (20.0 + 8.0 * np.maximum(8.0, 2.0 * d - 4.0) + 6.0 * 38.0)))
    nbytes = float(len(d) * (12 + (4 if weighted else 0) + 8) + 4.0 * d.sum())
    return flops, nbytes


def fp32_peak_tflops(sm_max_mhz: float | None) -> float:
    """Nominal FP32 (FMA) peak: 148 SMs x 128 lanes x 2 flops x SM clock."""
    mhz = sm_max_mhz or 1965.0
    return 148 * 128 * 2 * mhz * 1e6 / 1e12


def read_traffic_per_launch() -> float | None:
    """DRAM bytes per cell-pass launch from the committed ncu summary, if present."""
    try:
        for line in open(PROFILE_SUMMARY):
            if line.startswith("dram_bytes_per_launch_full_size:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


def cpu_oracle_rate(pts, w, sample: int, threads: int = 0) -> dict:
    from oracle import pg_oracle

    n = pts.shape[0]
    m = min(sample, n)
    t0 = time.perf_counter()
    c = pg_oracle.cells(pts, w, mode="incremental", begin=0, end=m, threads=threads)
    wall = time.perf_counter() - t0
    per_cell = c.seconds / max(m, 1)
    full = c.tree_seconds + per_cell * n
    return {"value": n / full / 1e6, "cell_rate": m / c.seconds / 1e6, "cores": c.threads, "cells": m,
            "tree_s": c.tree_seconds, "cells_s": c.seconds, "wall_s": wall}


def cpu_oracle_rate_clouds(clouds, sample: int) -> dict:
    """Oracle rate over whole clouds taken in order until `sample` cells (each cloud its own diagram)."""
    from oracle import pg_oracle

    cells, secs, tree, threads, used = 0, 0.0, 0.0, 0, 0
    t0 = time.perf_counter()
    for c in clouds:
        if cells >= sample:
            break
        r = pg_oracle.cells(c, None, mode="incremental", threads=0)
        cells += len(c)
        secs += r.seconds + r.tree_seconds
        tree += r.tree_seconds
        threads = r.threads
        used += 1
    return {"value": cells / max(secs, 1e-9) / 1e6, "cores": threads, "cells": cells, "tree_s": tree,
            "cells_s": secs - tree, "wall_s": time.perf_counter() - t0, "clouds": used}


def run_reference_cuda(args, spec, world) -> bool:
    """The reference's own CUDA extension (oracle/_ref: its unmodified sources compiled with a
    project-written stand-in for its absent cuBQL dependency) on the same workload.

    A step is one reference call (paragram.voronoi_diagram / power_diagram's pybind function). Its
    value is cells / the reference's own "Construction time" (printed with debug=True: the cell
    kernel, the CSR gather, symmetrisation and cumsum, voronoi_ultra.cu:368-373), which leaves out
    its BVH build and kNN: the stand-in builds the BVH on the host, which would not be a fair
    stand-in for cuBQL's GPU builder. The full call's wall time is reported beside it.
    Returns False when the extension or a GPU is missing.
    """
    import torch

    from oracle import pg_ref

    if not (pg_ref.available() and torch.cuda.is_available()):
        return False
    dev = torch.device("cuda:0")
    pts, w = make_points(spec, seed=0)
    if spec["kind"] == "surfaces":
        # the reference has no batch API: one call per cloud, the clouds in order up to ~2M points
        take, tot = [], 0
        for c in pts:
            if tot >= 2_000_000:
                break
            take.append(torch.from_numpy(c).to(dev))
            tot += len(c)
        calls = [(lambda t=t, **kw: pg_ref.voronoi(t, **kw)) for t in take]
        sample = f"the first {len(take)} of {len(pts)} clouds ({tot} points), one reference call per cloud"
    elif spec["kind"] == "moving":
        # the moved points, warm-started with the reference's own diagram of the previous positions
        prev = pg_ref.voronoi(torch.from_numpy(pts).to(dev))
        t = torch.from_numpy(moved_points(pts, 0)).to(dev)
        g, go = prev[0].to(torch.int32).contiguous(), prev[1].to(torch.int32).contiguous()
        calls = [(lambda **kw: pg_ref.voronoi(t, initial_guesses=g, initial_guesses_offsets=go, **kw))]
        tot = len(pts)
        sample = (f"the whole {tot}-point workload per step, moved points rebuilt with the reference's diagram of "
                  "the previous positions as initial guesses")
    else:
        t = torch.from_numpy(pts).to(dev)
        tw = None if w is None else torch.from_numpy(w).to(dev)
        calls = [(lambda **kw: pg_ref.voronoi(t, **kw))] if tw is None else [(lambda **kw: pg_ref.power(t, tw, **kw))]
        tot = len(pts)
        sample = f"the whole {tot}-point workload per step"
    big = tot > 10_000_000  # the stand-in's host BVH build takes tens of seconds per call
    warm, steps = (min(args.warmup, 1), min(args.steps, 2)) if big else (args.warmup, args.steps)

    def one_step():
        cons, wall = 0.0, 0.0
        for fn in calls:
            t0 = time.perf_counter()
            ph = pg_ref.phase_ms(fn) or {}
            wall += time.perf_counter() - t0
            cons += sum(v for k, v in ph.items() if k.endswith("Construction"))
        return cons, wall

    for _ in range(warm):
        one_step()
    cons, walls = [], []
    for _ in range(steps):
        c, wl = one_step()
        cons.append(c)
        walls.append(wl)
    ms = statistics.median(cons)
    value = tot / (ms / 1e3) / 1e6
    line = {
        "impl": "reference", "metric": "Mcells/s", "value": value, "unit": "Mcells/s", "n_gpus": world,
        "steps": steps, "warmup": warm, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "n_points": tot, "weighted": spec["weighted"]},
        "cpu_baseline": {"value": value, "unit": "Mcells/s", "cores": 1, "kind": "reference",
                         "sample": sample + "; the reference's CUDA extension on the GPU, its construction phase "
                                   "(cells + CSR) timed by its own debug timers; the BVH comes from the "
                                   "stand-in's single-threaded host builder and is not counted"},
        "e2e": {"value": value, "unit": "Mcells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_full_call": {"ms_per_step": 1e3 * statistics.median(walls),
                                "note": "wall time of the whole call, including the stand-in's host BVH build"},
        "note": "the reference's own kernels (oracle/_ref); cuBQL replaced by a project-written stand-in",
    }
    print(json.dumps(line), flush=True)
    return True


def run_reference(args, spec, rank, world):
    """The reference on the same workload (rank 0 only): its CUDA extension where it is built and a
    GPU is present, else the CPU restatement of its construction on the host cores."""
    if rank != 0:
        return
    if not args.reference_cpu and run_reference_cuda(args, spec, world):
        return
    pts, w = make_points(spec, seed=0)
    sample = args.cpu_sample
    clouds = spec["kind"] == "surfaces"
    rate = (lambda m: cpu_oracle_rate_clouds(pts, m)) if clouds else (lambda m: cpu_oracle_rate(pts, w, m))
    for _ in range(args.warmup):
        rate(max(sample // 10, 1000))
    vals = []
    info = None
    for _ in range(args.steps):
        info = rate(sample)
        vals.append(info["value"])
    if clouds:
        spec = dict(spec, n=int(sum(len(c) for c in pts)))
    value = statistics.median(vals)
    line = {
        "impl": "reference",
        "metric": "Mcells/s",
        "value": value,
        "unit": "Mcells/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * info["wall_s"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": args.workload, "n_points": spec["n"], "weighted": spec["weighted"]},
        "cpu_baseline": {"value": value, "unit": "Mcells/s", "cores": info["cores"], "kind": "port",
                         "sample": f"{info['cells']} cells of the {spec['n']}-point workload per step; "
                                   f"kd-tree over all points ({info['tree_s']:.2f} s) + sampled cells "
                                   f"({info['cells_s']:.2f} s), extrapolated to all cells"},
        "e2e": {"value": value, "unit": "Mcells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "CPU restatement of the reference's construction (the oracle port) timed on the host",
    }
    print(json.dumps(line), flush=True)


def vertex_error(pts, w, count, rel, bound, planes, cells) -> dict:
    """Exported vertex positions of `cells` against their FP64 positions.

    Each vertex is the intersection of three planes; relative to its cell's point s the bisector
    with q is (q - s) . x = (|q - s|^2 - (w_q - w_s)) / 2 and a face of the reference's FP32 box
    (voronoi_ultra.cu:234-238) is x_axis = b - s_axis. The 3x3 systems are solved in FP64 from
    the FP32 inputs. Reported: max and median of |x - x64| / |x64|, the max absolute error, and
    how many vertices lie farther than their exported bound.
    """
    p = pts.astype(np.float64)
    wt = np.zeros(len(p)) if w is None else w.astype(np.float64)
    f = np.float32
    lo = ((pts.min(0) - f(1.0)).astype(f) - f(1e-5)).astype(np.float64)
    hi = ((pts.max(0) + f(1.0)).astype(f) + f(1e-5)).astype(np.float64)
    k = np.minimum(count[cells], rel.shape[1])
    cell = np.repeat(cells, k)
    slot = np.concatenate([np.arange(x) for x in k])
    x = rel[cell, slot].astype(np.float64)
    b = bound[cell, slot].astype(np.float64)
    pl = planes[cell, slot].astype(np.int64)
    s = p[cell]
    A = np.zeros((len(cell), 3, 3))
    rhs = np.zeros((len(cell), 3))
    for e in range(3):
        ids = pl[:, e]
        bis = ids >= 0
        q = np.where(bis, ids, 0)
        a = p[q] - s
        code = -1 - ids
        axis = np.where(bis, 0, code >> 1)
        A[:, e, :] = np.where(bis[:, None], a, np.eye(3)[axis])
        face = np.where(code & 1, hi[axis], lo[axis]) - s[np.arange(len(cell)), axis]
        rhs[:, e] = np.where(bis, 0.5 * ((a * a).sum(1) - (wt[q] - wt[cell])), face)
    x64 = np.linalg.solve(A, rhs[..., None])[..., 0]
    err = np.linalg.norm(x - x64, axis=1)
    rel_err = err / np.maximum(np.linalg.norm(x64, axis=1), 1e-300)
    return {"vertices": int(err.size), "cells": int(len(cells)), "max_rel": float(rel_err.max()),
            "median_rel": float(np.median(rel_err)), "max_abs": float(err.max()),
            "beyond_bound": int((err > b + 1e-12 * np.linalg.norm(x64, axis=1)).sum()),
            "reference": "FP64 solve of each vertex's three planes from the FP32 inputs"}


def _timed(fn, steps, dev, flush):
    """Run fn `steps` times, L2 flushed before each, timed with CUDA events on the current stream."""
    import torch

    import paragram_b200.cuda as pc

    times, cell_ms, launches, out = [], [], 0, None
    for _ in range(steps):
        flush.fill_(1.0)
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize(dev)
        times.append(e0.elapsed_time(e1))
        prof = pc.last_profile()
        cell_ms.append(prof["cells_ms"])
        launches += int(prof["launches"])
    return times, cell_ms, launches, out


class _PinnedOut:
    """Reusable pinned host buffers for the Diagram's device->host copies (full PCIe rate, asynchronous)."""

    def __init__(self):
        import torch

        self._torch = torch
        self.bufs = {}

    def copy(self, key, t):
        buf = self.bufs.get(key)
        if buf is None or buf.numel() < t.numel() or buf.dtype != t.dtype:
            buf = self._torch.empty(max(t.numel(), 1), dtype=t.dtype, pin_memory=True)
            self.bufs[key] = buf
        out = buf[: t.numel()]
        out.copy_(t, non_blocking=True)
        return out


def _peaks():
    try:
        return json.load(open(MEASURED_PEAKS))
    except (OSError, ValueError):
        return {}


def _roofline(flops, nbytes, cell_s, csum, kernel, traffic):
    peaks = _peaks()
    peak = fp32_peak_tflops(peaks.get("sm_max_mhz") or csum.get("sm_max_mhz"))
    achieved = flops / cell_s / 1e12 if cell_s > 0 else None
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    return {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": (achieved / peak) if achieved else None, "traffic": traffic,
            "kernel": kernel, "cell_pass_ms": cell_s * 1e3,
            "algorithmic_flops": flops, "algorithmic_bytes": nbytes,
            "hbm_frac": (nbytes / cell_s / 1e9) / hbm_peak if cell_s > 0 else None,
            "peak_note": "nominal FP32 FMA peak 148 SM x 128 lanes x 2 x max SM clock "
                         "(MEASURED_PEAKS has no FP32 figure)"}


def _cpu_baseline(args, world, pts, w, n):
    if world != 1 or args.no_cpu_baseline:
        return None
    try:
        cb = cpu_oracle_rate(pts, w, args.cpu_sample)
        return {"value": cb["value"], "unit": "Mcells/s", "cores": cb["cores"], "kind": "port",
                "sample": f"{cb['cells']} of {n} cells; kd-tree {cb['tree_s']:.2f} s + cells "
                          f"{cb['cells_s']:.2f} s on {cb['cores']} threads, extrapolated to all cells"}
    except Exception as exc:  # the baseline must not hide the GPU number
        return {"value": None, "unit": "Mcells/s", "cores": 0, "kind": "port", "sample": f"failed: {exc}"}


def _cpu_baseline_clouds(args, world, clouds):
    if world != 1 or args.no_cpu_baseline:
        return None
    try:
        cb = cpu_oracle_rate_clouds(clouds, args.cpu_sample)
        return {"value": cb["value"], "unit": "Mcells/s", "cores": cb["cores"], "kind": "port",
                "sample": f"the first {cb['clouds']} clouds ({cb['cells']} cells), each its own diagram, on "
                          f"{cb['cores']} threads"}
    except Exception as exc:
        return {"value": None, "unit": "Mcells/s", "cores": 0, "kind": "port", "sample": f"failed: {exc}"}


def run_gpu(args, spec, rank, world, local):
    import torch

    import paragram_b200 as pg
    import paragram_b200.cuda as pc
    from paragram_b200 import dist, learned

    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    if spec["kind"] == "surfaces":
        return run_batch_gpu(args, spec, rank, world, local, dev)
    if spec["kind"] == "lattice" and not args.plain:
        return run_lattice_gpu(args, spec, rank, world, local, dev)
    if spec["kind"] == "moving":
        return run_moving_gpu(args, spec, rank, world, local, dev)
    if args.sharded:
        return run_sharded_gpu(args, spec, rank, world, local, dev)
    pts, w = make_points(spec, seed=rank)
    n = pts.shape[0]
    h_pts = torch.from_numpy(pts).pin_memory()
    h_w = torch.from_numpy(w).pin_memory() if w is not None else None
    d_pts = h_pts.to(dev)
    d_w = h_w.to(dev)[:, None] if h_w is not None else None
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2
    use_model = args.workload in LEARNED and not args.plain
    model = train_info = None
    if use_model:
        model, train_info = train_model(dev, rank)
    blob = model.blob if model is not None else None

    def step_device(with_model=True, profile=False):
        return pc._run(d_pts, d_w, 8, False, None, None, -1, profile=profile,
                       model=blob if with_model else None)

    phases = {}

    def cell_pass_ms(with_model=True):
        # phase times come from a separate profiled build: the timed steps carry no per-phase events
        ms, prs = [], []
        for _ in range(3):
            flush.fill_(1.0)
            step_device(with_model, profile=True)
            pr = pc.last_profile()
            prs.append(pr)
            ms.append(pr["cells_ms"] + pr["deferred_ms"])  # both cell launches
        if with_model or not use_model:
            phases.update({k: round(statistics.median(p[k] for p in prs), 3)
                           for k in ("lbvh_ms", "cells_ms", "deferred_ms", "csr_ms")})
        return statistics.median(ms)

    host_out = _PinnedOut()

    def step_e2e():
        x = h_pts.to(dev, non_blocking=True)
        if h_w is None:
            d = learned.voronoi_diagram(x, model) if model is not None else pg.voronoi_diagram(x)
        else:
            d = pg.power_diagram(x, h_w.to(dev, non_blocking=True))
        return host_out.copy("a", d.adjacency), host_out.copy("o", d.offsets), host_out.copy("s", d.status)

    for _ in range(args.warmup):
        step_device()
        if use_model:
            step_device(False)
    torch.cuda.synchronize(dev)
    dist.barrier()
    with ClockSampler(local) as clocks:
        # learned and plain steps interleaved, so that neither gets the warmer half of the run
        times, cell_ms, launches, plain = [], [], 0, ([], [], 0, None) if use_model else None
        for _ in range(args.steps):
            t, c, l_, out = _timed(step_device, 1, dev, flush)
            times += t
            cell_ms += c
            launches += l_
            (adj, off, st) = out
            if use_model:
                pt = _timed(lambda: step_device(False), 1, dev, flush)
                plain = (plain[0] + pt[0], plain[1] + pt[1], plain[2] + pt[2], pt[3])
    dist.barrier()
    torch.cuda.synchronize(dev)
    total_ms = dist.reduce_max(sum(times), dev)
    total_cells = dist.reduce_sum(float(n) * args.steps, dev)
    value = total_cells / (total_ms / 1e3) / 1e6
    plain_value = None
    if plain is not None:
        plain_value = total_cells / (dist.reduce_max(sum(plain[0]), dev) / 1e3) / 1e6

    # end-to-end through the public API from pinned host memory
    for _ in range(max(1, args.warmup // 2)):
        step_e2e()
    torch.cuda.synchronize(dev)
    dist.barrier()
    e2e_times, _, _, (a, o, s) = _timed(step_e2e, args.steps, dev, flush)
    d2h = a.numel() * 4 + o.numel() * 4 + s.numel() * 4
    e2e_ms = dist.reduce_max(sum(e2e_times), dev)
    e2e_value = total_cells / (e2e_ms / 1e3) / 1e6
    h2d = n * 12 + (n * 4 if h_w is not None else 0)
    # counters of one more (untimed) build: escalations, fallback rate, traversal work; the cell pass alone
    _, cnt = pc.build_with_stats(d_pts, d_w, model=blob)
    fp32_only = None
    if args.fp32_only_too:
        # the same build with FP32-only side tests (the reference's arithmetic: no escalation)
        def step_fp32():
            return pc._run(d_pts, d_w, 8, False, None, None, -1, fp32_only=True)
        step_fp32()
        ft, _, _, (fa, fo, fs) = _timed(step_fp32, args.steps, dev, flush)
        fv = total_cells / (dist.reduce_max(sum(ft), dev) / 1e3) / 1e6
        dd = (fo[1:] - fo[:-1]) != (off[1:] - off[:-1])
        fp32_only = {"value": fv, "unit": "Mcells/s", "ms_per_step": statistics.mean(ft),
                     "identical_to_exact": bool(torch.equal(fa, adj) and torch.equal(fo, off) and torch.equal(fs, st)),
                     "cells_with_other_degree_or_status": int((dd | (fs != st)).sum())}
    cells_main = cell_pass_ms(True)
    cells_plain = cell_pass_ms(False) if use_model else None
    vtx_err = None
    if rank == 0:
        # the position error of the builder's vertices, on the first 200k cells of one more build
        _, vst = pc.build_with_stats(d_pts, d_w, vertices=64)
        m = min(n, 200_000)
        vtx_err = vertex_error(pts[: n], w, vst["vertex_count"].cpu().numpy(), vst["vertices"][:m].cpu().numpy(),
                               vst["vertex_bound"][:m].cpu().numpy(), vst["vertex_planes"][:m].cpu().numpy(),
                               np.arange(m))
        del vst

    if rank == 0:
        off_np = off.cpu().numpy()
        flops, nbytes = algorithmic_work(off_np, spec["weighted"])
        cell_s = cells_main / 1e3
        csum = clocks.summary()
        config = {"workload": args.workload, "n_points": n, "weighted": spec["weighted"],
                  "l2": "flushed between steps (256 MiB write)",
                  "parallelism": f"independent diagram per GPU x{world}",
                  "predicates": "FP32 filtered, FP64 / exact escalation",
                  "escalation": {"fp32_tests_per_cell": cnt["tests"] / n,
                                 "fp64_fraction": cnt["fp64_escalations"] / max(cnt["tests"], 1),
                                 "exact_fraction": cnt["exact_escalations"] / max(cnt["tests"], 1),
                                 "fp64_vertices_per_cell": cnt["vertex64"] / n,
                                 "vertex_error": vtx_err},
                  "work_per_cell": {k: round(cnt[k] / n, 3) for k in ("nodes", "leaves", "candidates", "clips",
                                                                       "deferred_cells")},
                  "phases_ms": dict(phases, note="one profiled build: LBVH (+ prediction), first cell pass, "
                                                 "deferred-cell pass, CSR count + scan; the CSR fill runs in "
                                                 "the adjacency emission")}
        if fp32_only is not None:
            config["fp32_only_predicates"] = fp32_only
        if use_model:
            config["search_radius"] = "learned (MLP 16-64-64-2, BF16, trained before timing)"
            config["learned"] = dict(train_info, fallback_rate=cnt["hint_misses"] / n,
                                     capped_cells=(cnt["hint_hits"] + cnt["hint_misses"]) / n)
            config["plain"] = {"value": plain_value, "unit": "Mcells/s", "ms_per_step": statistics.mean(plain[0]),
                               "step_ms": [round(t, 2) for t in plain[0]],
                               "cell_pass_ms": cells_plain}
            config["learned_over_plain"] = value / plain_value if plain_value else None
            # the same ratio from the median step times (robust to an occasional slow step)
            config["learned_over_plain_median"] = statistics.median(plain[0]) / statistics.median(times)
        line = {
            "metric": "Mcells/s",
            "value": value,
            "unit": "Mcells/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": statistics.mean(times),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "step_ms": [round(t, 2) for t in times],
            "config": config,
            "e2e": {"value": e2e_value, "unit": "Mcells/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": _roofline(flops, nbytes, cell_s, csum, "k_cells_fast (cell pass)",
                                  read_traffic_per_launch() if args.workload == "clustered_voronoi_5m" else None),
            "cpu_baseline": _cpu_baseline(args, world, pts, w, n),
            "clocks": csum,
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)


def run_lattice_gpu(args, spec, rank, world, local, dev):
    """The jittered 310^3 power lattice as its configuration states it: learned search radius (a model
    trained before timing on two 100^3 jittered lattices of other seeds), FP32-filtered predicates
    with FP64 / exact escalation, and the batched path (one cloud, CUDA-graph replay), unchunked;
    the plain batched build is timed beside it."""
    import torch

    import paragram_b200.cuda as pc
    from paragram_b200 import dist, learned
    from paragram_b200 import workloads as W
    from paragram_b200.batch import build_batch

    pts, w = make_points(spec, seed=rank)
    n = pts.shape[0]
    h_pts, h_w = torch.from_numpy(pts).pin_memory(), torch.from_numpy(w).pin_memory()
    d_pts, d_w = h_pts.to(dev), h_w.to(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    t0 = time.perf_counter()
    data = [learned.collect(*[torch.from_numpy(a).to(dev) for a in W.jittered_lattice(100, seed=1000 + 2 * rank + k)])
            for k in range(2)]
    log = []
    model = learned.train(data, epochs=4, batch=8192, log=log)
    margin = model.calibrate(data[0], quantile=0.98)
    del data
    torch.cuda.synchronize(dev)
    train_info = {"train_s": time.perf_counter() - t0, "loss_per_epoch": [round(x, 4) for x in log],
                  "margin": margin, "calibration_quantile": 0.98, "trained_on": "two 100^3 jittered lattices"}

    def step(with_model=True):
        return build_batch([d_pts], [d_w], graph=True, model=model if with_model else None)

    host_out = _PinnedOut()

    def step_e2e():
        d = build_batch([h_pts.to(dev, non_blocking=True)], [h_w.to(dev, non_blocking=True)], graph=True,
                        model=model)[0]
        return host_out.copy("a", d.adjacency), host_out.copy("o", d.offsets), host_out.copy("s", d.status)

    for _ in range(args.warmup):
        step()
        step(False)
    torch.cuda.synchronize(dev)
    dist.barrier()
    times, plain_times = [], []
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            t, _, _, out = _timed(step, 1, dev, flush)
            times += t
            t, _, _, _ = _timed(lambda: step(False), 1, dev, flush)
            plain_times += t
    dist.barrier()
    total_cells = dist.reduce_sum(float(n) * args.steps, dev)
    value = total_cells / (dist.reduce_max(sum(times), dev) / 1e3) / 1e6
    plain_value = total_cells / (dist.reduce_max(sum(plain_times), dev) / 1e3) / 1e6
    for _ in range(max(1, args.warmup // 2)):
        step_e2e()
    e2e_times, _, _, (a, o, s) = _timed(step_e2e, args.steps, dev, flush)
    e2e_value = total_cells / (dist.reduce_max(sum(e2e_times), dev) / 1e3) / 1e6
    d2h = a.numel() * 4 + o.numel() * 4 + s.numel() * 4
    # counters and phase times of the same build through the single-cloud entry point (untimed)
    _, cnt = pc.build_with_stats(d_pts, d_w, model=model.blob, profile=True)
    prof = pc.last_profile()
    if rank == 0:
        d = out[0]
        off_np = d.offsets.cpu().numpy()
        flops, nbytes = algorithmic_work(off_np, True)
        cell_s = (prof["cells_ms"] + prof["deferred_ms"]) / 1e3
        csum = clocks.summary()
        line = {
            "metric": "Mcells/s", "value": value, "unit": "Mcells/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": statistics.mean(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "step_ms": [round(t, 2) for t in times],
            "config": {"workload": args.workload, "n_points": n, "weighted": True,
                       "l2": "flushed between steps (256 MiB write)", "launch": "batched build, CUDA graph replay",
                       "chunks": int(prof["chunks"]), "parallelism": f"independent diagram per GPU x{world}",
                       "predicates": "FP32 filtered, FP64 / exact escalation",
                       "escalation": {"fp32_tests_per_cell": cnt["tests"] / n,
                                      "fp64_fraction": cnt["fp64_escalations"] / max(cnt["tests"], 1),
                                      "exact_fraction": cnt["exact_escalations"] / max(cnt["tests"], 1),
                                      "fp64_vertices_per_cell": cnt["vertex64"] / n},
                       "search_radius": "learned (MLP 16-64-64-2, BF16, trained before timing)",
                       "learned": dict(train_info, fallback_rate=cnt["hint_misses"] / n,
                                       hit_rate=cnt["hint_hits"] / n),
                       "plain": {"value": plain_value, "unit": "Mcells/s",
                                 "ms_per_step": statistics.mean(plain_times)},
                       "learned_over_plain": value / plain_value,
                       "learned_over_plain_median": statistics.median(plain_times) / statistics.median(times),
                       "status_counts": np.bincount(d.status.cpu().numpy(), minlength=6)[:6].tolist(),
                       "phases_ms": {k: round(prof[k], 3) for k in ("lbvh_ms", "cells_ms", "deferred_ms", "csr_ms")}},
            "e2e": {"value": e2e_value, "unit": "Mcells/s", "h2d_bytes_per_step": n * 16, "d2h_bytes_per_step": d2h},
            "roofline": _roofline(flops, nbytes, cell_s, csum, "k_cells_fast (cell pass)", None),
            "cpu_baseline": _cpu_baseline(args, world, pts, w, n),
            "clocks": csum,
            "gpu_launches": int(prof["launches"]) * args.steps,
        }
        print(json.dumps(line), flush=True)


def run_sharded_gpu(args, spec, rank, world, local, dev):
    """One diagram over all ranks (strong scaling, ``--sharded``): the workload's one point set
    (seed 0 on every rank) split into contiguous shards, rank r passing the r-th; every step is
    ``paragram_b200.sharded.voronoi_diagram`` / ``power_diagram`` (point all-gather, the rank's
    range of cells, row all-gather, CSR assembly), which returns the full Diagram on every rank.
    The plain build (no learned radius)."""
    import torch

    import paragram_b200.cuda as pc
    from paragram_b200 import dist, sharded

    pts, w = make_points(spec, seed=0)
    n = pts.shape[0]
    b, e = n * rank // world, n * (rank + 1) // world
    h_pts = torch.from_numpy(np.ascontiguousarray(pts[b:e])).pin_memory()
    h_w = None if w is None else torch.from_numpy(np.ascontiguousarray(w[b:e])).pin_memory()
    d_pts = h_pts.to(dev)
    d_w = None if h_w is None else h_w.to(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def build(p, wt):
        return sharded.voronoi_diagram(p) if wt is None else sharded.power_diagram(p, wt)

    host_out = _PinnedOut()

    def step_e2e():
        d = build(h_pts.to(dev, non_blocking=True), None if h_w is None else h_w.to(dev, non_blocking=True))
        return host_out.copy("a", d.adjacency), host_out.copy("o", d.offsets), host_out.copy("s", d.status)

    for _ in range(args.warmup):
        build(d_pts, d_w)
    torch.cuda.synchronize(dev)
    dist.barrier()
    with ClockSampler(local) as clocks:
        times, _, launches, d = _timed(lambda: build(d_pts, d_w), args.steps, dev, flush)
    dist.barrier()
    total_ms = dist.reduce_max(sum(times), dev)
    value = float(n) * args.steps / (total_ms / 1e3) / 1e6
    step_e2e()
    e2e_times, _, _, (a, o, s) = _timed(step_e2e, args.steps, dev, flush)
    e2e_value = float(n) * args.steps / (dist.reduce_max(sum(e2e_times), dev) / 1e3) / 1e6
    d2h = a.numel() * 4 + o.numel() * 4 + s.numel() * 4
    if rank == 0:
        off_np = d.offsets.cpu().numpy()
        flops, nbytes = algorithmic_work(off_np, spec["weighted"])
        csum = clocks.summary()
        line = {
            "metric": "Mcells/s", "value": value, "unit": "Mcells/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "step_ms": [round(t, 2) for t in times],
            "config": {"workload": args.workload, "n_points": n, "weighted": spec["weighted"],
                       "parallelism": f"one diagram sharded over {world} GPU(s): point all-gather, a range of "
                                      "the curve order per rank, row all-gather, CSR on every rank",
                       "l2": "flushed between steps (256 MiB write)"},
            "e2e": {"value": e2e_value, "unit": "Mcells/s", "h2d_bytes_per_step": h_pts.numel() * 4 +
                    (0 if h_w is None else h_w.numel() * 4), "d2h_bytes_per_step": d2h},
            "roofline": _roofline(flops / world, nbytes / world, total_ms / args.steps / 1e3, csum,
                                  "whole sharded step (this rank's share of the cells)", None),
            "cpu_baseline": None,
            "clocks": csum,
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)


def run_moving_gpu(args, spec, rank, world, local, dev):
    """Warm start across iterations: the points move by 1% of their mean spacing between steps (a
    fixed displacement field, applied forwards then backwards, so the steps alternate between two
    point sets A and B), and each step rebuilds the diagram with the previous step's diagram as
    initial guesses; the cold rebuild of the same points is timed beside it. Both give the same
    diagram (checked here)."""
    import torch

    import paragram_b200 as pg
    import paragram_b200.cuda as pc
    from paragram_b200 import dist

    pts, _ = make_points(spec, seed=rank)
    n = pts.shape[0]
    moved = moved_points(pts, rank)
    h_sets = [torch.from_numpy(pts).pin_memory(), torch.from_numpy(moved).pin_memory()]
    d_sets = [h.to(dev) for h in h_sets]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    diagrams = [pg.voronoi_diagram(d) for d in d_sets]  # each set's diagram, the guesses of the other
    state = {"k": 0}

    def step_warm():
        k = state["k"] = 1 - state["k"]
        prev = diagrams[1 - k]
        return pc._run(d_sets[k], None, 8, False, prev.adjacency, prev.offsets, -1)

    def step_cold():
        return pc._run(d_sets[state["k"]], None, 8, False, None, None, -1)

    host_out = _PinnedOut()

    def step_e2e():
        k = state["k"] = 1 - state["k"]
        prev = diagrams[1 - k]
        d = pg.voronoi_diagram(h_sets[k].to(dev, non_blocking=True), initial_guesses=prev.adjacency,
                               initial_guesses_offsets=prev.offsets)
        return host_out.copy("a", d.adjacency), host_out.copy("o", d.offsets), host_out.copy("s", d.status)

    for _ in range(args.warmup):
        step_warm()
        step_cold()
    torch.cuda.synchronize(dev)
    dist.barrier()
    times, cold_times, same = [], [], True
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            t, _, _, (a, o, s) = _timed(step_warm, 1, dev, flush)
            times += t
            t, _, _, (a0, o0, s0) = _timed(step_cold, 1, dev, flush)
            cold_times += t
            same = same and torch.equal(a, a0) and torch.equal(o, o0) and torch.equal(s, s0)
    dist.barrier()
    total_cells = dist.reduce_sum(float(n) * args.steps, dev)
    value = total_cells / (dist.reduce_max(sum(times), dev) / 1e3) / 1e6
    cold_value = total_cells / (dist.reduce_max(sum(cold_times), dev) / 1e3) / 1e6
    for _ in range(max(1, args.warmup // 2)):
        step_e2e()
    e2e_times, _, _, (a, o, s) = _timed(step_e2e, args.steps, dev, flush)
    e2e_value = total_cells / (dist.reduce_max(sum(e2e_times), dev) / 1e3) / 1e6
    d2h = a.numel() * 4 + o.numel() * 4 + s.numel() * 4
    k = 1 - state["k"]
    prev = diagrams[1 - k]
    _, cw = pc.build_with_stats(d_sets[k], initial_guesses=prev.adjacency, initial_guesses_offsets=prev.offsets,
                                profile=True)
    prof = pc.last_profile()
    _, cc = pc.build_with_stats(d_sets[k])
    if rank == 0:
        off_np = diagrams[k].offsets.cpu().numpy()
        flops, nbytes = algorithmic_work(off_np, False)
        cell_s = (prof["cells_ms"] + prof["deferred_ms"]) / 1e3
        csum = clocks.summary()
        work = ("nodes", "leaves", "candidates", "clips")
        line = {
            "metric": "Mcells/s", "value": value, "unit": "Mcells/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": statistics.mean(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "step_ms": [round(t, 2) for t in times],
            "config": {"workload": args.workload, "n_points": n, "weighted": False,
                       "motion": "1% of the mean spacing per step (Gaussian), alternating between two point sets",
                       "warm_start": "the previous step's diagram as initial_guesses",
                       "l2": "flushed between steps (256 MiB write)",
                       "parallelism": f"independent diagram per GPU x{world}",
                       "cold": {"value": cold_value, "unit": "Mcells/s", "ms_per_step": statistics.mean(cold_times)},
                       "warm_over_cold": value / cold_value, "identical_to_cold": bool(same),
                       "work_per_cell_warm": {k_: round(cw[k_] / n, 3) for k_ in work},
                       "work_per_cell_cold": {k_: round(cc[k_] / n, 3) for k_ in work},
                       "phases_ms": {k_: round(prof[k_], 3) for k_ in ("lbvh_ms", "cells_ms", "deferred_ms",
                                                                       "csr_ms")}},
            "e2e": {"value": e2e_value, "unit": "Mcells/s", "h2d_bytes_per_step": n * 12, "d2h_bytes_per_step": d2h},
            "roofline": _roofline(flops, nbytes, cell_s, csum, "k_cells_fast (cell pass)", None),
            "cpu_baseline": _cpu_baseline(args, world, pts, None, n),
            "clocks": csum,
            "gpu_launches": int(prof["launches"]) * args.steps,
        }
        print(json.dumps(line), flush=True)


def run_batch_gpu(args, spec, rank, world, local, dev):
    """256 surface clouds of uneven size in one build (CUDA graph replay), per-cloud Diagrams."""
    import torch

    import paragram_b200.cuda as pc
    from paragram_b200 import dist
    from paragram_b200.batch import build_batch

    clouds, _ = make_points(spec, seed=rank)
    n = int(sum(len(c) for c in clouds))
    h_clouds = [torch.from_numpy(c).pin_memory() for c in clouds]
    d_clouds = [c.to(dev) for c in h_clouds]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    build_batch(d_clouds, graph=False)
    launches_per_build = int(pc.last_profile()["launches"]) + 1  # + adjacency emission

    def step():
        return build_batch(d_clouds, graph=True)

    host_out = _PinnedOut()

    def step_e2e():
        ds = build_batch([c.to(dev, non_blocking=True) for c in h_clouds], graph=True)
        return [(host_out.copy(("a", k), d.adjacency), host_out.copy(("o", k), d.offsets),
                 host_out.copy(("s", k), d.status)) for k, d in enumerate(ds)]

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    dist.barrier()
    with ClockSampler(local) as clocks:
        times, _, _, ds = _timed(step, args.steps, dev, flush)
    dist.barrier()
    total_ms = dist.reduce_max(sum(times), dev)
    total_cells = dist.reduce_sum(float(n) * args.steps, dev)
    value = total_cells / (total_ms / 1e3) / 1e6
    for _ in range(max(1, args.warmup // 2)):
        step_e2e()
    e2e_times, _, _, res = _timed(step_e2e, args.steps, dev, flush)
    e2e_value = total_cells / (dist.reduce_max(sum(e2e_times), dev) / 1e3) / 1e6
    d2h = sum(a.numel() * 4 + o.numel() * 4 + s.numel() * 4 for a, o, s in res)
    # phase times of one more (untimed, not captured) build of the same batch
    build_batch(d_clouds, graph=False, profile=True)
    prof = pc.last_profile()
    if rank == 0:
        flops = nbytes = 0.0
        status = np.zeros(6, np.int64)
        for d in ds:
            f, b = algorithmic_work(d.offsets.cpu().numpy(), False)
            flops += f
            nbytes += b
            status += np.bincount(d.status.cpu().numpy(), minlength=6)[:6]
        csum = clocks.summary()
        step_s = statistics.mean(times) / 1e3
        line = {
            "metric": "Mcells/s", "value": value, "unit": "Mcells/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": statistics.mean(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "clouds": len(clouds), "n_points": n,
                       "cloud_sizes": [int(min(len(c) for c in clouds)), int(max(len(c) for c in clouds))],
                       "l2": "flushed between steps (256 MiB write)", "launch": "one CUDA graph per batch shape",
                       "status_counts": status.tolist(), "parallelism": f"independent batch per GPU x{world}",
                       "phases_ms": {k: round(prof[k], 3) for k in ("lbvh_ms", "cells_ms", "deferred_ms", "csr_ms",
                                                                     "deferred_cells")}},
            "e2e": {"value": e2e_value, "unit": "Mcells/s", "h2d_bytes_per_step": n * 12, "d2h_bytes_per_step": d2h},
            "roofline": _roofline(flops, nbytes, step_s, csum, "whole batched build (graph replay)", None),
            "cpu_baseline": _cpu_baseline_clouds(args, world, clouds),
            "clocks": csum,
            "gpu_launches": launches_per_build * args.steps,
        }
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="clustered_voronoi_5m", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-sample", type=int, default=200_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--reference-cpu", action="store_true",
                    help="with --impl reference: time the CPU restatement even where the reference's CUDA "
                         "extension is built")
    ap.add_argument("--plain", action="store_true", help="time the plain build only (no learned radius)")
    ap.add_argument("--sharded", action="store_true",
                    help="strong scaling: one diagram of the workload built by all ranks together")
    ap.add_argument("--fp32-only-too", action="store_true",
                    help="also time the build with FP32-only side tests (no FP64 / exact escalation)")
    args = ap.parse_args()
    spec = WORKLOADS[args.workload]
    from paragram_b200 import dist

    if args.impl == "reference":
        rank, world, _ = dist.env_world()
        run_reference(args, spec, rank, world)
        return
    rank, world, local = dist.init("nccl" if int(os.environ.get("WORLD_SIZE", 1)) > 1 else "gloo", timeout_s=300)
    try:
        run_gpu(args, spec, rank, world, local)
    finally:
        dist.finalize()


if __name__ == "__main__":
    main()
