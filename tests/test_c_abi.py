"""The C ABI library loads, exports every symbol of include/paragram_b200.h and
rejects bad arguments before touching a GPU."""

import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    from paragram_b200 import _lib

    return _lib.load()


def test_header_symbols_exported(lib):
    from paragram_b200 import _lib

    header = open(os.path.join(ROOT, "include", "paragram_b200.h")).read()
    declared = set(re.findall(r"^\s*(?:int|size_t|const char \*)\s*(pg_\w+)\s*\(", header, re.M))
    assert declared == set(_lib.EXPORTED)
    for name in declared:
        assert hasattr(lib, name), name


def test_version(lib):
    assert lib.pg_version() >= 100


def test_workspace_size(lib):
    n = ctypes.c_size_t(0)
    assert lib.pg_workspace_size(1000, ctypes.byref(n)) == 0
    small = n.value
    assert lib.pg_workspace_size(1_000_000, ctypes.byref(n)) == 0
    assert n.value > small > 0
    assert lib.pg_workspace_size(-1, ctypes.byref(n)) == -1
    assert lib.pg_workspace_size(1 << 26, ctypes.byref(n)) == -1


def _build(lib, n, points=1, weights=None, guesses=None, goff=None, ws=256, ws_bytes=1 << 40, offsets=256,
           status=256, options=None):
    from paragram_b200 import _lib

    e = ctypes.c_int64(0)
    opt = options if options is not None else _lib.PgOptions(8, -1, 0, 0)
    return lib.pg_build(n, points, weights, guesses, goff, ctypes.byref(opt), ws, ws_bytes, offsets, status,
                        ctypes.byref(e), None)


def test_build_rejects_bad_arguments(lib):
    from paragram_b200 import _lib

    assert _build(lib, -5) == -1
    assert _build(lib, 10, points=None) == -1
    assert _build(lib, 10, ws=None) == -1
    assert _build(lib, 10, ws=257) == -1  # not 256-byte aligned
    assert _build(lib, 10, guesses=512) == -1  # guesses without offsets
    assert _build(lib, 10, ws_bytes=16) == -1  # workspace too small
    assert _build(lib, 10, options=_lib.PgOptions(8, 64, 0, 0)) == -1  # leaf too large
    assert "leaf_size" in _lib.last_error(lib)
    opt = _lib.PgOptions(8, -1, 0, 0)
    opt.geometry_out = 264  # centroid + volume rows need 16-byte alignment
    assert _build(lib, 10, options=opt) == -1
    assert "geometry_out" in _lib.last_error(lib)


def test_emit_rejects_bad_arguments(lib):
    assert lib.pg_emit_adjacency(10, None, None, None, None) == -1


def test_mlp_entry_points_without_gpu(lib):
    """Sizes of the learned-radius model and argument checks (no kernel runs)."""
    assert lib.pg_mlp_num_params() == 5378
    assert lib.pg_mlp_model_bytes() == 11984
    assert lib.pg_mlp_forward(-1, None, None, None, None) == -1
    assert lib.pg_mlp_forward(0, None, None, None, None) == 0
    assert lib.pg_mlp_grad(10, None, None, None, 1.0, None, None, None, None) == -1
    assert lib.pg_mlp_adam(None, None, None, None, 1, 1e-3, 0.9, 0.999, 1e-8, None, None) == -1
    assert lib.pg_mlp_adam(256, 256, 256, 256, 0, 1e-3, 0.9, 0.999, 1e-8, 256, None) == -1  # step must be >= 1
    assert lib.pg_mlp_pack(None, None, None) == -1


def test_vertex_export_arguments(lib):
    from paragram_b200 import _lib

    opt = _lib.PgOptions(8, -1, 0, 0)
    opt.vertices_out = 256  # vertex_cap 0 with an output
    assert _build(lib, 10, options=opt) == -1
    assert "vertex_cap" in _lib.last_error(lib)
    opt.vertex_cap = 8
    opt.vertices_out = 264  # float4 rows need 16-byte alignment
    assert _build(lib, 10, options=opt) == -1
    assert "vertices_out" in _lib.last_error(lib)
    opt.vertex_cap = -1
    opt.vertices_out = None
    assert _build(lib, 10, options=opt) == -1


def test_options_layout_matches_header(tmp_path):
    """The ctypes mirror of pg_options has the header's size and field offsets."""
    import shutil
    import subprocess

    from paragram_b200 import _lib

    if shutil.which("gcc") is None:
        pytest.skip("needs gcc")
    fields = [f for f, _ in _lib.PgOptions._fields_]
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "paragram_b200.h"\nint main(void){\n'
                   '  printf("%zu\\n", sizeof(pg_options));\n' +
                   "".join(f'  printf("%zu\\n", offsetof(pg_options, {f}));\n' for f in fields) + "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", f"-I{os.path.join(ROOT, 'include')}", str(src), "-o", str(exe)], check=True)
    vals = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert vals[0] == ctypes.sizeof(_lib.PgOptions)
    assert vals[1:] == [getattr(_lib.PgOptions, f).offset for f in fields]


def test_workspace_tree_offsets(lib):
    out = (ctypes.c_int64 * 5)()
    for n, clouds in ((1000, 1), (250_000, 1), (250_000, 37)):
        size = ctypes.c_size_t(0)
        if clouds == 1:
            assert lib.pg_workspace_size(n, ctypes.byref(size)) == 0
        else:
            assert lib.pg_batch_workspace_size(n, clouds, ctypes.byref(size)) == 0
        assert lib.pg_workspace_tree(n, clouds, out, 5) == 0
        offs = list(out)
        assert all(o % 256 == 0 for o in offs)
        # points, order and records are N-sized; the per-cloud roots and boxes come last
        assert offs[0] + 16 * n <= offs[1] and offs[1] + 4 * n <= offs[2] < offs[3]
        assert offs[3] + 4 * clouds <= size.value and offs[4] + 32 * clouds <= size.value
    assert lib.pg_workspace_tree(1000, 0, out, 5) == -1
    assert lib.pg_workspace_tree(-1, 1, out, 5) == -1
    assert lib.pg_workspace_tree(1000, 1, None, 5) == -1
