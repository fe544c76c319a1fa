"""Where the cell kernel's time goes: SM cycles per cell by phase.

Runs the plain build of a few workloads through the instrumented library
(``python -m paragram_b200.build --phase-cycles`` compiles it with
``-DPG_PHASE_CYCLES``: every phase of a cell brackets itself with
``clock64()`` and adds the difference to the warp's counters) and prints one
JSON line per workload with the per-cell averages of the work counters and of
the cycles per phase, and each phase's share of the whole cell:

* ``nodes``: popping BVH node entries, the node's empty-sphere vertex mask,
  queueing its children;
* ``leaves``: leaf batches (loading the points, the security-radius and
  FP32 pre-checks), including ``clips``;
* ``clips``: clipping the cell by the candidates that pass the pre-check;
* ``out``: writing the row;
* ``other``: the rest of the cell (box init, the path walk from the seed's
  leaf, radius updates after clips are in ``leaves``).

The counters are per warp: a phase's cycles include the cycles other warps of
the SM issued meanwhile, so the figures are latencies as one cell sees them,
and the shares are the meaningful part. The instrumented kernel runs slower
than the product's (the counters live in shared memory).

Usage: ``PARAGRAM_B200_LIB=paragram_b200/libparagram_b200_phase.so
python -m paragram_b200.phase_cycles [--workloads clustered_5m,power_1m,...]``
"""

from __future__ import annotations

import argparse
import json
import os

import numpy as np
import torch


def _workloads():
    from . import workloads as W

    def surface_big():
        clouds = W.surface_clouds(num_clouds=256, seed=0)
        return clouds[int(np.argmax([len(c) for c in clouds]))], None

    return {
        "uniform_100k": lambda: (W.uniform(100_000, seed=0), None),
        "power_1m": lambda: W.power_uniform(1_000_000, seed=0),
        "clustered_500k": lambda: (W.clustered(500_000, seed=0), None),
        "clustered_5m": lambda: (W.clustered(5_000_000, seed=0), None),
        "surface_largest_of_256": surface_big,
    }


def main(argv=None):
    from . import _lib
    from . import cuda as pc

    table = _workloads()
    ap = argparse.ArgumentParser()
    ap.add_argument("--workloads", default="clustered_5m,power_1m,surface_largest_of_256")
    args = ap.parse_args(argv)
    if not torch.cuda.is_available():
        raise SystemExit("phase_cycles needs a CUDA device")
    dev = torch.device("cuda:0")
    for name in args.workloads.split(","):
        pts, w = table[name]()
        t = torch.from_numpy(pts).to(dev)
        tw = None if w is None else torch.from_numpy(w).to(dev)
        n = len(pts)
        for _ in range(2):  # the second build is the one reported
            _, st = pc.build_with_stats(t, tw, profile=True)
        if st["cyc_cell"] == 0:
            raise SystemExit(f"{_lib.LIB_PATH} was built without PG_PHASE_CYCLES "
                             "(python -m paragram_b200.build --phase-cycles)")
        prof = pc.last_profile()
        cyc = {k[4:]: st[k] / n for k in ("cyc_cell", "cyc_warm", "cyc_nodes", "cyc_leaves", "cyc_clips", "cyc_out")}
        cyc["other"] = cyc["cell"] - cyc["warm"] - cyc["nodes"] - cyc["leaves"] - cyc["out"]
        share = {k: round(v / cyc["cell"], 4) for k, v in cyc.items() if k != "cell"}
        work = {k: round(st[k] / n, 2) for k in ("nodes", "leaves", "candidates", "clips", "tests", "fp64_escalations")}
        print(json.dumps({"workload": name, "n": n, "library": os.path.basename(_lib.LIB_PATH),
                          "phases_ms": {k: round(v, 2) for k, v in prof.items()},
                          "per_cell": work, "cycles_per_cell": {k: round(v) for k, v in cyc.items()},
                          "share_of_cell": share,
                          "deferred_tier_cycles_per_deferred_cell": round(st["cyc_big"] / max(1, prof["deferred_cells"]))}),
              flush=True)


if __name__ == "__main__":
    main()
