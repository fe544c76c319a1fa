"""Build recipe of libparagram_b200.so (sm_100a, in-tree).

Every ``csrc/*.cu`` file is compiled by nvcc for ``sm_100a`` and linked into
``paragram_b200/libparagram_b200.so`` next to this file, so the library
travels with the source tree. Object files go to ``paragram_b200/_build/``.
"""

from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD_DIR = os.path.join(HERE, "_build")
LIB_PATH = os.path.join(HERE, "libparagram_b200.so")
SOURCES = ["pg_api.cu", "pg_lbvh.cu", "pg_cells.cu", "pg_csr.cu", "pg_scan.cu", "pg_noalloc.cu", "pg_mlp.cu",
           "pg_faces.cu", "pg_knn.cu"]
#: The instrumented variant (per-phase SM cycle counters in the cell kernel, -DPG_PHASE_CYCLES): a
#: separate library for profiling only; ``PARAGRAM_B200_LIB`` selects it at load time.
PHASE_BUILD_DIR = os.path.join(HERE, "_build_phase")
PHASE_LIB_PATH = os.path.join(HERE, "libparagram_b200_phase.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps() -> list[str]:
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".h"))] + [
        os.path.join(HERE, "..", "include", "paragram_b200.h")
    ]


def up_to_date(lib: str = LIB_PATH) -> bool:
    if not os.path.exists(lib):
        return False
    t = os.path.getmtime(lib)
    return all(os.path.getmtime(d) <= t for d in _deps() if os.path.exists(d))


def _compile(src: str, ptxas_verbose: bool, phase_cycles: bool = False) -> tuple[str, str]:
    obj = os.path.join(PHASE_BUILD_DIR if phase_cycles else BUILD_DIR, os.path.splitext(src)[0] + ".o")
    cmd = [nvcc(), *ARCH, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
    if phase_cycles:
        cmd.append("-DPG_PHASE_CYCLES")
    if ptxas_verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False, phase_cycles: bool = False) -> str:
    """Compile the CUDA library for sm_100a if it is missing or stale (``phase_cycles``: the
    instrumented variant, ``libparagram_b200_phase.so``)."""
    lib_path = PHASE_LIB_PATH if phase_cycles else LIB_PATH
    if not force and up_to_date(lib_path):
        return lib_path
    os.makedirs(PHASE_BUILD_DIR if phase_cycles else BUILD_DIR, exist_ok=True)
    with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(lambda s: _compile(s, ptxas_verbose, phase_cycles), SOURCES))
    if verbose or ptxas_verbose:
        for _, log in results:
            if log:
                print(log, file=sys.stderr)
    objs = [o for o, _ in results]
    tmp = lib_path + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed:\n{r.stderr}")
    os.replace(tmp, lib_path)
    return lib_path


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, ptxas_verbose="--ptxas" in sys.argv,
                phase_cycles="--phase-cycles" in sys.argv))
