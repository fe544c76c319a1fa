"""Compile the reference's own CUDA extension into ``oracle/_ref/`` (test infrastructure).

TEST INFRASTRUCTURE ONLY: the result is a parity and timing baseline, loaded
by ``oracle/pg_ref.py`` from ``tests/`` and ``bench.py``; the paragram_b200
product never loads it.

The reference (zenseact/paragram) JIT-compiles ``paragram/csrc/laguerre/*.cu``
and ``paragram/csrc/ext.cpp`` into a torch extension (paragram/_backend.py:147-192)
against its cuBQL submodule, which is empty in the reference tree (pinned
version unknown). This recipe compiles those unmodified source files where
they lie, with the reference's own flags for a compute-capability-10 device
(``-O3 --extended-lambda -Xptxas -dlcm=ca --maxrregcount=128
-DMODERN_CUDA_CARDS -use_fast_math``, _backend.py:160-165) for sm_100a, and
replaces cuBQL by the project-written headers of ``oracle/cubql_standin/``
(types, a host-built median-split BVH, a BVH kNN query, a rounded-down box
distance). Object files go to a temporary directory; only
``oracle/_ref/paragram_ref.so`` is written into the tree.

    python oracle/build_ref.py [REFERENCE_ROOT]    # default: /root/reference
"""

from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
OUT = os.path.join(OUT_DIR, "paragram_ref.so")
STANDIN = os.path.join(HERE, "cubql_standin")
NAME = "paragram_ref"


def _torch_flags():
    import torch
    import torch.utils.cpp_extension as ce

    inc = [f"-I{p}" for p in ce.include_paths("cuda")]
    libs = [f"-L{p}" for p in ce.library_paths("cuda")]
    abi = f"-D_GLIBCXX_USE_CXX11_ABI={int(torch._C._GLIBCXX_USE_CXX11_ABI)}"
    defs = [f"-DTORCH_EXTENSION_NAME={NAME}", "-DTORCH_API_INCLUDE_EXTENSION_H", abi]
    return inc, libs, defs, list(ce.COMMON_NVCC_FLAGS)


def build(ref_root: str = "/root/reference", force: bool = False) -> str:
    src = os.path.join(ref_root, "paragram", "csrc")
    if not os.path.isdir(src):
        raise FileNotFoundError(f"reference sources not found under {src}")
    cu = sorted(os.path.join(src, "laguerre", f) for f in os.listdir(os.path.join(src, "laguerre"))
                if f.endswith(".cu"))
    cpp = [os.path.join(src, "ext.cpp")]
    deps = cu + cpp + [os.path.join(dp, f) for dp, _, fs in os.walk(STANDIN) for f in fs]
    if not force and os.path.exists(OUT) and all(os.path.getmtime(d) <= os.path.getmtime(OUT) for d in deps):
        return OUT
    import sysconfig

    inc, libs, defs, nv_common = _torch_flags()
    inc += [f"-I{src}", f"-I{STANDIN}", f"-I{sysconfig.get_paths()['include']}"]
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    tmp = tempfile.mkdtemp(prefix="paragram_ref_")
    cuda_flags = ["-O3", "--extended-lambda", "-Xptxas", "-dlcm=ca", "--maxrregcount=128", "-DMODERN_CUDA_CARDS",
                  "-use_fast_math", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17",
                  "-Xcompiler", "-fPIC", *nv_common]
    cxx_flags = ["-O3", "-Wno-attributes", "-fPIC", "-std=c++17"]

    def compile_one(path: str) -> str:
        obj = os.path.join(tmp, os.path.basename(path) + ".o")
        if path.endswith(".cu"):
            cmd = [nvcc, *cuda_flags, *defs, *inc, "-c", path, "-o", obj]
        else:
            cmd = ["g++", *cxx_flags, *defs, *inc, "-c", path, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compiling {path} failed:\n{r.stderr[-4000:]}")
        return obj

    try:
        with concurrent.futures.ThreadPoolExecutor(len(cu) + len(cpp)) as ex:
            objs = list(ex.map(compile_one, cu + cpp))
        os.makedirs(OUT_DIR, exist_ok=True)
        stubs = "/usr/local/cuda/lib64/stubs"
        cmd = ["g++", "-shared", "-o", OUT + ".tmp", *objs, *libs, f"-L{stubs}", "-lc10", "-lc10_cuda", "-ltorch_cpu",
               "-ltorch_cuda", "-ltorch", "-ltorch_python", "-lcudart", "-lcuda"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"linking failed:\n{r.stderr[-4000:]}")
        os.replace(OUT + ".tmp", OUT)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return OUT


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else "/root/reference", force="--force" in sys.argv))
