"""ctypes binding of libparagram_b200.so (the C ABI declared in include/paragram_b200.h)."""

from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
#: The library loaded by ``load()``; ``PARAGRAM_B200_LIB`` names another build of the same sources
#: (the phase-cycle instrumented one, ``python -m paragram_b200.build --phase-cycles``).
LIB_PATH = os.environ.get("PARAGRAM_B200_LIB") or os.path.join(_HERE, "libparagram_b200.so")

_lock = threading.Lock()
_lib = None


class PgOptions(ctypes.Structure):
    """Mirror of ``pg_options`` (include/paragram_b200.h)."""

    _fields_ = [
        ("knn", ctypes.c_int32),
        ("leaf_size", ctypes.c_int32),
        ("debug", ctypes.c_int32),
        ("num_chunks", ctypes.c_int32),
        ("blocks_per_sm", ctypes.c_int32),
        ("predicates", ctypes.c_int32),
        ("model", ctypes.c_void_p),
        ("radius_hint", ctypes.c_void_p),
        ("radius_out", ctypes.c_void_p),
        ("work_out", ctypes.c_void_p),
        ("features_out", ctypes.c_void_p),
        ("order_out", ctypes.c_void_p),
        ("geometry_out", ctypes.c_void_p),
        ("vertex_cap", ctypes.c_int32),
        ("vertices_out", ctypes.c_void_p),
        ("vertex_planes_out", ctypes.c_void_p),
        ("vertex_count_out", ctypes.c_void_p),
    ]


#: Symbols declared in include/paragram_b200.h.
EXPORTED = ["pg_version", "pg_last_error", "pg_workspace_size", "pg_build", "pg_emit_adjacency", "pg_stats",
            "pg_last_profile", "pg_degrees_to_offsets_noalloc", "pg_batch_workspace_size", "pg_build_batch",
            "pg_batch_check", "pg_mlp_num_params", "pg_mlp_model_bytes", "pg_mlp_forward", "pg_mlp_grad",
            "pg_mlp_adam", "pg_mlp_pack", "pg_face_areas", "pg_workspace_tree", "pg_knn", "pg_build_range",
            "pg_range_pack", "pg_range_unpack", "pg_range_finish"]


def load() -> ctypes.CDLL:
    """Load the CUDA library; raise ImportError when it has not been built."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                "paragram_b200 CUDA library is missing (libparagram_b200.so); build it with "
                "`python -m paragram_b200.build` (nvcc with sm_100a support is required)"
            )
        lib = ctypes.CDLL(LIB_PATH)
        vp, i64, i32, sz = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_size_t
        lib.pg_version.restype = ctypes.c_int
        lib.pg_last_error.restype = ctypes.c_char_p
        lib.pg_workspace_size.argtypes = [i64, ctypes.POINTER(sz)]
        lib.pg_workspace_size.restype = ctypes.c_int
        lib.pg_build.argtypes = [i64, vp, vp, vp, vp, ctypes.POINTER(PgOptions), vp, sz, vp, vp,
                                 ctypes.POINTER(i64), vp]
        lib.pg_build.restype = ctypes.c_int
        lib.pg_emit_adjacency.argtypes = [i64, vp, vp, vp, vp]
        lib.pg_emit_adjacency.restype = ctypes.c_int
        lib.pg_stats.argtypes = [vp, i64, ctypes.POINTER(ctypes.c_uint64), i32, vp]
        lib.pg_stats.restype = ctypes.c_int
        lib.pg_build_range.argtypes = [i64, vp, vp, ctypes.POINTER(PgOptions), vp, sz, i64, i64, vp, vp]
        lib.pg_build_range.restype = ctypes.c_int
        lib.pg_range_pack.argtypes = [i64, vp, vp, i64, i64, vp, i64, ctypes.POINTER(i64), vp]
        lib.pg_range_pack.restype = ctypes.c_int
        lib.pg_range_unpack.argtypes = [i64, vp, vp, vp, i64, i64, vp]
        lib.pg_range_unpack.restype = ctypes.c_int
        lib.pg_range_finish.argtypes = [i64, vp, vp, ctypes.POINTER(i64), vp]
        lib.pg_range_finish.restype = ctypes.c_int
        lib.pg_knn.argtypes = [i64, vp, i32, vp, sz, vp, vp]
        lib.pg_knn.restype = ctypes.c_int
        lib.pg_workspace_tree.argtypes = [i64, i32, ctypes.POINTER(i64), i32]
        lib.pg_workspace_tree.restype = ctypes.c_int
        lib.pg_last_profile.argtypes = [ctypes.POINTER(ctypes.c_double), i32]
        lib.pg_last_profile.restype = ctypes.c_int
        lib.pg_batch_workspace_size.argtypes = [i64, i32, ctypes.POINTER(sz)]
        lib.pg_batch_workspace_size.restype = ctypes.c_int
        lib.pg_build_batch.argtypes = [i64, i32, vp, vp, vp, ctypes.POINTER(PgOptions), vp, sz, vp, vp,
                                       ctypes.POINTER(i64), vp]
        lib.pg_build_batch.restype = ctypes.c_int
        lib.pg_batch_check.argtypes = [vp, i64, i32, vp]
        lib.pg_batch_check.restype = ctypes.c_int
        lib.pg_mlp_num_params.restype = ctypes.c_int
        lib.pg_mlp_model_bytes.restype = sz
        lib.pg_mlp_forward.argtypes = [i64, vp, vp, vp, vp]
        lib.pg_mlp_forward.restype = ctypes.c_int
        lib.pg_mlp_grad.argtypes = [i64, vp, vp, vp, ctypes.c_float, vp, vp, vp, vp]
        lib.pg_mlp_grad.restype = ctypes.c_int
        lib.pg_mlp_adam.argtypes = [vp, vp, vp, vp, i64, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                    ctypes.c_float, vp, vp]
        lib.pg_mlp_adam.restype = ctypes.c_int
        lib.pg_mlp_pack.argtypes = [vp, vp, vp]
        lib.pg_mlp_pack.restype = ctypes.c_int
        lib.pg_face_areas.argtypes = [i64, i32, vp, vp, vp, vp, vp, vp, vp, vp]
        lib.pg_face_areas.restype = ctypes.c_int
        lib.pg_degrees_to_offsets_noalloc.argtypes = [i64, vp, vp, vp]
        lib.pg_degrees_to_offsets_noalloc.restype = ctypes.c_int
        _lib = lib
        return lib


def last_error(lib: ctypes.CDLL) -> str:
    msg = lib.pg_last_error()
    return msg.decode() if msg else ""
