"""ctypes binding of the C ABI in ``include/ccc_b200.h`` and ``include/ccc_engine.h``
(``libccc_b200.so``).

There is no fallback: if the library is missing or fails to load, every operation raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libccc_b200.so")

# return codes / status bits (mirrors include/ccc_b200.h)
CCC_OK = 0
CCC_ERR_INVALID_ARG = 1
CCC_ERR_WORKSPACE = 2
CCC_ERR_CUDA = 3
CCC_ERR_TOO_LARGE = 4
LIB_REFERENCE = 0
LIB_PORTABLE = 1
CCC_ST_CAND_OVERFLOW = 1
CCC_ST_OUT_OVERFLOW = 2
CCC_ST_STACK_OVERFLOW = 4
CCC_ST_MALFORMED_TREE = 8

OP_BVH, OP_FIND_COLLISIONS, OP_CONTINUOUS, OP_PROXIMITY, OP_IMPULSES, OP_MINCOL = range(6)

# every symbol the header declares, with (restype, argtypes)
_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_D = ctypes.c_double
SIGNATURES = {
    "ccc_version": (_I, []),
    "ccc_error_string": (ctypes.c_char_p, [_I]),
    "ccc_kernel_launches": (_I64, []),
    "ccc_debug_math": (_I, [_I, _P, _P, _I64, _P]),
    "ccc_debug_stage": (_I, [_I, _I, _P, _I, _P, _I, _I64, _P]),
    "ccc_set_math_library": (_I, [_I]),
    "ccc_get_math_library": (_I, []),
    "ccc_timing_begin": (_I, []),
    "ccc_timing_end": (_I, [_I, _P, _I, _P, _P]),
    "ccc_workspace_size": (_I64, [_I, _I64, _I64, _I64]),
    "ccc_read_status": (_I, [_P, _I64, _P, _P]),
    "ccc_read_counters": (_I, [_P, _P, _P]),
    "ccc_bvh": (_I, [_I, _P, _P, _I64, _I64, _P, _P, _P, _I64, _P]),
    "ccc_find_collisions": (_I, [_I, _P, _P, _P, _I64, _I64, _D, _I64, _P, _P, _I64, _P]),
    "ccc_find_collisions_continuous": (_I, [_I, _P, _P, _P, _P, _P, _I64, _I64, _I64, _I64, _P, _P, _P, _I64, _P]),
    "ccc_find_mincol_cand": (_I, [_I, _P, _P, _P, _P, _I64, _I64, _I64, _P, _P, _I64, _P]),
    "ccc_find_proximity": (_I, [_I, _P, _P, _P, _I64, _I64, _D, _I64, _P, _P, _I64, _P]),
    "ccc_find_triangle_edge_collisions": (_I, [_I, _P, _P, _P, _I64, _I64, _I64, _P, _P, _P, _I64, _P]),
    "ccc_find_triangle_edge_candidates": (_I, [_I, _P, _P, _P, _I64, _I64, _I64, _P, _P, _I64, _P]),
    "ccc_find_triangle_edge_candidates2": (_I, [_I, _P, _P, _P, _I64, _I64, _I64, _P, _P, _P, _I64, _P]),
    "ccc_compute_impulses": (_I, [_I, _P, _P, _P, _P, _P, _P, _I64, _I64, _I64, _I64, _P, _P, _P, _P, _I64, _P]),
    "ccc_static_scratch_bytes": (_I64, []),
    "ccc_find_collisions_continuous_static": (_I, [_I, _P, _P, _P, _P, _P, _I64, _I64, _I64, _I64, _P, _P, _P]),
    "ccc_static_scratch_read_status": (_I, [_I64, _P, _P]),
    "ccc_static_scratch_read_counters": (_I, [_P, _P]),
    "ccc_compute_impulses_from_collisions": (_I, [_I, _P, _P, _I64, _I64, _P, _P, _P, _I64, _P, _P, _P, _P, _I64,
                                                 _P]),
    # resident engine (include/ccc_engine.h)
    "ccc_engine_bytes": (_I64, [_I, _I64, _I64, _I64, _I64, _I64]),
    "ccc_engine_create": (_I, [_I, _I64, _I64, _I64, _I64, _I64, _P, _I64, _P, _P]),
    "ccc_engine_destroy": (_I, [_P]),
    "ccc_engine_add_mesh": (_I, [_P, _I64, _I64, _P]),
    "ccc_engine_remove_mesh": (_I, [_P, ctypes.c_int32]),
    "ccc_engine_mesh_view": (_I, [_P, ctypes.c_int32, _P]),
    "ccc_engine_free_slots": (_I, [_P, _P, _P]),
    "ccc_engine_set_active": (_I, [_P, _P, _I64, _P]),
    "ccc_engine_build": (_I, [_P, _P, _I64, _P]),
    "ccc_engine_ccd": (_I, [_P, _P]),
    "ccc_engine_loop_prepare": (_I, [_P, _P, _I64, _P]),
    "ccc_engine_loop_step": (_I, [_P, ctypes.c_int32, _P]),
    "ccc_engine_capture": (_I, [_P, _I, ctypes.c_int32, _P]),
    "ccc_engine_replay": (_I, [_P, _I, _P]),
    "ccc_engine_autotune": (_I, [_P, _P, _P]),
    "ccc_engine_schedule_count": (_I, []),
    "ccc_engine_schedule_info": (_I, [ctypes.c_int32, _P]),
    "ccc_engine_set_schedule": (_I, [_P, ctypes.c_int32]),
    "ccc_engine_read_state": (_I, [_P, _P, _I64, _P, _P, _P, _P, _P, _P]),
    "ccc_engine_pack_rows": (_I, [_P, _P, _P, _I64, _P, _P]),
    "ccc_engine_counters": (_I, [_P, _P, _P]),
}

# engine constants (mirrors include/ccc_engine.h)
CCC_MESH_DONE = 1
CCC_MESH_CONVERGED = 2
CCC_ST_NONFINITE = 16
ENGINE_OP_CCD = 0
ENGINE_OP_LOOP_STEP = 1


class MeshView(ctypes.Structure):
    """ccc_mesh_view"""
    _fields_ = [("F", ctypes.c_int64), ("V", ctypes.c_int64), ("x0", ctypes.c_void_p), ("x1", ctypes.c_void_p),
                ("masses", ctypes.c_void_p), ("faces", ctypes.c_void_p), ("verts0", ctypes.c_void_p),
                ("verts1", ctypes.c_void_p), ("vel", ctypes.c_void_p), ("rows", ctypes.c_void_p),
                ("times", ctypes.c_void_p)]


_lib = None


class NativeLibraryError(RuntimeError):
    pass


def lib():
    """Load libccc_b200.so (raises NativeLibraryError when it is absent)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise NativeLibraryError(
                f"{LIB_PATH} is not built; run `python -m cccollisions_b200.build` (nvcc, sm_100a)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int, what: str):
    if rc != CCC_OK:
        msg = lib().ccc_error_string(rc).decode()
        raise RuntimeError(f"{what} failed: {msg} (code {rc})")


def kernel_launches() -> int:
    return int(lib().ccc_kernel_launches())


def timing_begin():
    lib().ccc_timing_begin()


def timing_end(max_kernels: int = 64):
    """{kernel name: (total ms, launches)} for the launches since timing_begin()."""
    name_len = 64
    names = ctypes.create_string_buffer(max_kernels * name_len)
    ms = (ctypes.c_float * max_kernels)()
    cnt = (ctypes.c_int32 * max_kernels)()
    n = lib().ccc_timing_end(max_kernels, names, name_len, ms, cnt)
    if n < 0:
        raise RuntimeError("kernel timing failed")
    out = {}
    for i in range(n):
        nm = names.raw[i * name_len:(i + 1) * name_len].split(b"\0", 1)[0].decode()
        out[nm] = (float(ms[i]), int(cnt[i]))
    return out


class math_library:
    """Context manager selecting the solver's elementary functions (LIB_REFERENCE: CUDA's,
    as the reference; LIB_PORTABLE: the library's own, shared bit for bit with the oracle)."""

    def __init__(self, lib_id: int):
        self.lib_id = lib_id
        self.prev = None

    def __enter__(self):
        self.prev = lib().ccc_get_math_library()
        check(lib().ccc_set_math_library(self.lib_id), "ccc_set_math_library")
        return self

    def __exit__(self, *exc):
        lib().ccc_set_math_library(self.prev)
        return False
