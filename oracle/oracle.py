"""ctypes front end of the CPU oracle (oracle/ccc_oracle.cpp).

TEST INFRASTRUCTURE ONLY: the test suite, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` use this module as the checker.  The product package never imports it.

All functions take numpy arrays in the reference's tensor layouts for ONE mesh
(``triangles`` (F, 3, 3), ``bboxes`` (2F-1, 6), ``tree`` (2F-1, 4) int64) and return numpy
arrays.  ``dtype`` follows the triangle array (float32 or float64).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libccc_oracle.so")
_SRC = os.path.join(_HERE, "ccc_oracle.cpp")
_LIBM = os.path.join(_HERE, "..", "cccollisions_b200", "csrc", "ccc_libm.h")
_DDMUL = os.path.join(_HERE, "..", "cccollisions_b200", "csrc", "ccc_ddmul.h")

_P = ctypes.c_void_p
_I64 = ctypes.c_int64


def build(force: bool = False) -> str:
    """Compile the oracle shared library (g++, no FP contraction, OpenMP)."""
    deps = [_SRC, _LIBM, _DDMUL]
    if not force and os.path.exists(_LIB_PATH):
        t = os.path.getmtime(_LIB_PATH)
        if all(os.path.getmtime(d) <= t for d in deps):
            return _LIB_PATH
    os.makedirs(os.path.dirname(_LIB_PATH), exist_ok=True)
    cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC",
           "-shared", "-o", _LIB_PATH, _SRC]
    # explicit fma() calls become single instructions where the CPU has FMA (results are
    # identical either way: fma is correctly rounded in hardware and in libm)
    try:
        if " fma " in open("/proc/cpuinfo").read().replace("\n", " "):
            cmd.insert(1, "-mfma")
    except OSError:
        pass
    subprocess.check_call(cmd)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _LIB_PATH if os.path.exists(_LIB_PATH) else build()
        L = ctypes.CDLL(path)
        L.orc_bvh.argtypes = [ctypes.c_int, _P, _P, ctypes.c_int, ctypes.c_int, _P, _P, _P]
        L.orc_bvh.restype = ctypes.c_int
        L.orc_candidates.argtypes = [ctypes.c_int, _P, _P, ctypes.c_int, ctypes.c_double, _P, _P, _I64,
                                     ctypes.c_int]
        L.orc_candidates.restype = _I64
        L.orc_find_collisions.argtypes = [ctypes.c_int, _P, _P, _P, ctypes.c_int, ctypes.c_double, _P, _I64,
                                          ctypes.c_int]
        L.orc_find_collisions.restype = _I64
        L.orc_ccd.argtypes = [ctypes.c_int, _P, _P, _P, _P, ctypes.c_int, _P, _P, _P, _I64, ctypes.c_int]
        L.orc_ccd.restype = _I64
        L.orc_mincol.argtypes = [ctypes.c_int, _P, _P, _P, _P, ctypes.c_int, _P, _I64]
        L.orc_mincol.restype = _I64
        L.orc_impulses_from_rows.argtypes = [ctypes.c_int, _P, _P, _P, ctypes.c_int, _P, _P, _I64, _P, _P, _P]
        L.orc_impulses_from_rows.restype = ctypes.c_int
        L.orc_impulses.argtypes = [ctypes.c_int, _P, _P, _P, _P, _P, ctypes.c_int, _P, _P, _P, _P, ctypes.c_int]
        L.orc_impulses.restype = _I64
        L.orc_proximity.argtypes = [ctypes.c_int, _P, _P, _P, ctypes.c_int, ctypes.c_double, _P, _P, _I64]
        L.orc_proximity.restype = _I64
        L.orc_solve_cubic.argtypes = [ctypes.c_double] * 4 + [_P]
        L.orc_morton.argtypes = [ctypes.c_double] * 3
        L.orc_morton.restype = ctypes.c_uint32
        L.orc_morton_f.argtypes = [ctypes.c_float] * 3
        L.orc_morton_f.restype = ctypes.c_uint32
        L.orc_certmul.argtypes = [_P, ctypes.c_int, ctypes.c_double, _P]
        for f in ("orc_cbrt", "orc_acos", "orc_cos", "orc_sin"):
            getattr(L, f).argtypes = [ctypes.c_double]
            getattr(L, f).restype = ctypes.c_double
        L.orc_cubic_coeffs.argtypes = [_P, _P]
        L.orc_filter.argtypes = [_P, ctypes.c_int, ctypes.c_double]
        L.orc_filter.restype = ctypes.c_int
        L.orc_contact.argtypes = [_P, ctypes.c_int, ctypes.c_double, _P, _P]
        L.orc_sat.argtypes = [ctypes.c_int, _P, _P, ctypes.c_double]
        L.orc_sat.restype = ctypes.c_int
        L.orc_num_threads.restype = ctypes.c_int
        L.orc_triangle_edge.argtypes = [ctypes.c_int, _P, _P, _P, ctypes.c_int, ctypes.c_int, _P, _P, _P, _I64,
                                        ctypes.c_int]
        L.orc_triangle_edge.restype = _I64
        L.orc_ddmul_check.argtypes = [_I64, ctypes.c_uint64, ctypes.c_int, _P]
        L.orc_ddmul_check.restype = ctypes.c_int
        L.orc_impulse_loop.argtypes = [ctypes.c_int, _P, _P, _P, _P, _P, _I64, _I64, ctypes.c_int, _P, ctypes.c_int,
                                       _P]
        L.orc_impulse_loop.restype = ctypes.c_int
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _dt(a):
    if a.dtype == np.float32:
        return 0
    if a.dtype == np.float64:
        return 1
    raise TypeError(f"unsupported dtype {a.dtype}")


def _c(a, dtype=None):
    return np.ascontiguousarray(a if dtype is None else a.astype(dtype, copy=False))


def num_threads() -> int:
    return lib().orc_num_threads()


def bvh(triangles, triangles_next=None, spatial=False, return_codes=False):
    """bvh / bvh_motion for one mesh: (bboxes (2F-1, 6), tree (2F-1, 4) int64)."""
    t = _c(triangles)
    n = t.shape[0]
    tn = None if triangles_next is None else _c(triangles_next, t.dtype)
    bb = np.full((2 * n - 1, 6), -1, dtype=t.dtype)
    tr = np.full((2 * n - 1, 4), -1, dtype=np.int64)
    codes = np.zeros(n, dtype=np.uint32)
    rc = lib().orc_bvh(_dt(t), _ptr(t), _ptr(tn), n, 1 if spatial else 0, _ptr(bb), _ptr(tr), _ptr(codes))
    if rc != 0:
        raise RuntimeError("oracle bvh failed")
    return (bb, tr, codes) if return_codes else (bb, tr)


def candidates(bboxes, tree, threshold=0.0, mask=None, nthreads=1):
    bb = _c(bboxes)
    tr = _c(tree, np.int64)
    n = (bb.shape[0] + 1) // 2
    m = None if mask is None else _c(mask, np.uint8)
    cnt = lib().orc_candidates(_dt(bb), _ptr(bb), _ptr(tr), n, float(threshold), _ptr(m), None, 0, nthreads)
    if cnt < 0:
        raise RuntimeError("oracle traversal failed (malformed tree or stack overflow)")
    out = np.zeros((max(cnt, 1), 2), dtype=np.int64)
    cnt = lib().orc_candidates(_dt(bb), _ptr(bb), _ptr(tr), n, float(threshold), _ptr(m), _ptr(out), cnt, nthreads)
    return out[:cnt]


def find_collisions(bboxes, tree, triangles, threshold=0.0, nthreads=1):
    """Intersecting pairs (i, j), i < j, as an (N, 2) int64 array (emission order)."""
    bb = _c(bboxes)
    tr = _c(tree, np.int64)
    t = _c(triangles, bb.dtype)
    n = t.shape[0]
    cap = 1 << 22
    out = np.zeros((cap, 2), dtype=np.int64)
    cnt = lib().orc_find_collisions(_dt(bb), _ptr(bb), _ptr(tr), _ptr(t), n, float(threshold), _ptr(out), cap,
                                    nthreads)
    if cnt < 0 or cnt > cap:
        raise RuntimeError("oracle find_collisions failed")
    return out[:cnt].copy()


def _triangle_edge(bboxes, tree, triangles, op, nthreads):
    bb = _c(bboxes)
    tr = _c(tree, np.int64)
    t = _c(triangles, bb.dtype)
    n = t.shape[0]
    L = lib()
    cnt = L.orc_triangle_edge(_dt(bb), _ptr(bb), _ptr(tr), _ptr(t), n, op, None, None, None, 0, nthreads)
    if cnt < 0:
        raise RuntimeError("oracle triangle-edge query failed (malformed tree or stack overflow)")
    w = 2 if op == 2 else 4
    rows = np.zeros((max(cnt, 1), w), dtype=np.int64)
    coefs = np.zeros(max(cnt, 1), dtype=bb.dtype) if op == 0 else None
    masks = np.zeros((max(cnt, 1), 2), dtype=np.int32) if op == 2 else None
    cnt = L.orc_triangle_edge(_dt(bb), _ptr(bb), _ptr(tr), _ptr(t), n, op, _ptr(rows), _ptr(coefs), _ptr(masks), cnt,
                              nthreads)
    return rows[:cnt], (coefs[:cnt] if op == 0 else masks[:cnt] if op == 2 else None)


def triangle_edge_collisions(bboxes, tree, triangles, nthreads=1):
    """find_triangle_edge_collisions for one mesh: rows (N, 4) int64 (i, j, cid, flag) and
    the edge coefficients (N,)."""
    return _triangle_edge(bboxes, tree, triangles, 0, nthreads)


def triangle_edge_candidates(bboxes, tree, triangles, nthreads=1):
    """find_triangle_edge_candidates for one mesh: rows (N, 4) int64 (i, j, cid, flag)."""
    return _triangle_edge(bboxes, tree, triangles, 1, nthreads)[0]


def triangle_edge_candidates2(bboxes, tree, triangles, nthreads=1):
    """find_triangle_edge_candidates2 for one mesh: pairs (N, 2) int64 and their masks (N, 2) int32."""
    return _triangle_edge(bboxes, tree, triangles, 2, nthreads)


def ccd(bboxes, tree, triangles, triangles_next, mask=None, nthreads=1):
    """Continuous collisions: rows (N, 3) int64 (i, j, k) and times (N,) float64."""
    bb = _c(bboxes)
    tr = _c(tree, np.int64)
    x0 = _c(triangles, bb.dtype)
    x1 = _c(triangles_next, bb.dtype)
    n = x0.shape[0]
    m = None if mask is None else _c(mask, np.uint8)
    cnt = lib().orc_ccd(_dt(bb), _ptr(bb), _ptr(tr), _ptr(x0), _ptr(x1), n, _ptr(m), None, None, 0, nthreads)
    if cnt < 0:
        raise RuntimeError("oracle ccd failed")
    rows = np.zeros((max(cnt, 1), 3), dtype=np.int64)
    times = np.zeros(max(cnt, 1), dtype=np.float64)
    cnt = lib().orc_ccd(_dt(bb), _ptr(bb), _ptr(tr), _ptr(x0), _ptr(x1), n, _ptr(m), _ptr(rows), _ptr(times), cnt,
                        nthreads)
    return rows[:cnt], times[:cnt]


def mincol_cand(bboxes, tree, triangles, triangles_next):
    bb = _c(bboxes)
    tr = _c(tree, np.int64)
    x0 = _c(triangles, bb.dtype)
    x1 = _c(triangles_next, bb.dtype)
    n = x0.shape[0]
    cnt = lib().orc_mincol(_dt(bb), _ptr(bb), _ptr(tr), _ptr(x0), _ptr(x1), n, None, 0)
    rows = np.zeros((max(cnt, 1), 3), dtype=np.int64)
    cnt = lib().orc_mincol(_dt(bb), _ptr(bb), _ptr(tr), _ptr(x0), _ptr(x1), n, _ptr(rows), cnt)
    return rows[:cnt]


def impulses_from_rows(triangles, triangles_next, masses, rows, times):
    x0 = _c(triangles)
    x1 = _c(triangles_next, x0.dtype)
    m = _c(masses, x0.dtype)
    r = _c(rows, np.int64).reshape(-1, 3)
    t = _c(times, np.float64).reshape(-1)
    n = x0.shape[0]
    dv = np.zeros((n, 3, 3), dtype=x0.dtype)
    dx = np.zeros((n, 3, 3), dtype=x0.dtype)
    cnt = np.zeros((n, 3), dtype=np.int32)
    lib().orc_impulses_from_rows(_dt(x0), _ptr(x0), _ptr(x1), _ptr(m), n, _ptr(r), _ptr(t), r.shape[0], _ptr(dv),
                                 _ptr(dx), _ptr(cnt))
    return dv, dx, cnt


def impulses(bboxes, tree, triangles, triangles_next, masses, mask=None, nthreads=1):
    """compute_impulses for one mesh: dv (F,3,3), dx (F,3,3), counter (F,3) int32, contacts."""
    bb = _c(bboxes)
    tr = _c(tree, np.int64)
    x0 = _c(triangles, bb.dtype)
    x1 = _c(triangles_next, bb.dtype)
    m = _c(masses, bb.dtype)
    n = x0.shape[0]
    mk = None if mask is None else _c(mask, np.uint8)
    dv = np.zeros((n, 3, 3), dtype=bb.dtype)
    dx = np.zeros((n, 3, 3), dtype=bb.dtype)
    cnt = np.zeros((n, 3), dtype=np.int32)
    c = lib().orc_impulses(_dt(bb), _ptr(bb), _ptr(tr), _ptr(x0), _ptr(x1), _ptr(m), n, _ptr(mk), _ptr(dv), _ptr(dx),
                           _ptr(cnt), nthreads)
    if c < 0:
        raise RuntimeError("oracle impulses failed")
    return dv, dx, cnt, c


def impulse_loop(verts0, verts1, vel, faces, masses, max_iter=50, nthreads=0):
    """The resident engine's impulse loop on one mesh (vertices (V,3), faces (F,3), per-corner
    masses (F,3)): returns (verts1, vel, iterations, converged, contacts per check)."""
    v0 = _c(verts0)
    v1 = _c(verts1, v0.dtype).copy()
    vl = _c(vel, v0.dtype).copy()
    fc = _c(faces, np.int32)
    m = _c(masses, v0.dtype)
    conv = ctypes.c_int(0)
    per = np.zeros(max_iter + 1, dtype=np.int32)
    it = lib().orc_impulse_loop(_dt(v0), _ptr(v0), _ptr(v1), _ptr(vl), _ptr(fc), _ptr(m), fc.shape[0], v0.shape[0],
                                int(max_iter), _ptr(per), int(nthreads), ctypes.byref(conv))
    if it < 0:
        raise RuntimeError("oracle impulse loop failed")
    return v1, vl, it, bool(conv.value), per[:it + (1 if conv.value else 0)]


def proximity(bboxes, tree, triangles, threshold):
    bb = _c(bboxes)
    tr = _c(tree, np.int64)
    t = _c(triangles, bb.dtype)
    n = t.shape[0]
    cnt = lib().orc_proximity(_dt(bb), _ptr(bb), _ptr(tr), _ptr(t), n, float(threshold), None, None, 0)
    rows = np.zeros((max(cnt, 1), 3), dtype=np.int64)
    dist = np.zeros(max(cnt, 1), dtype=np.float64)
    cnt = lib().orc_proximity(_dt(bb), _ptr(bb), _ptr(tr), _ptr(t), n, float(threshold), _ptr(rows), _ptr(dist), cnt)
    return rows[:cnt], dist[:cnt]


# ---- primitives -------------------------------------------------------------------------

def solve_cubic(a, b, c, d):
    r = np.zeros(3, dtype=np.float64)
    lib().orc_solve_cubic(float(a), float(b), float(c), float(d), _ptr(r))
    return r


def morton(x, y, z, single=False):
    if single:
        return lib().orc_morton_f(x, y, z)
    return lib().orc_morton(x, y, z)


def ddmul_check(n, seed, family):
    """(mismatches, short-path uses) of the double-double short paths against the bin
    algorithm on n generated operand sets (orc_ddmul_check)."""
    out = np.zeros(2, dtype=np.int64)
    lib().orc_ddmul_check(int(n), int(seed), int(family), _ptr(out))
    return int(out[0]), int(out[1])


def certmul(x, y):
    xs = np.ascontiguousarray(np.atleast_1d(np.asarray(x, dtype=np.float64)))
    r = np.zeros(2, dtype=np.float64)
    lib().orc_certmul(_ptr(xs), xs.shape[0], float(y), _ptr(r))
    return r


def cbrt(x):
    return lib().orc_cbrt(float(x))


def acos(x):
    return lib().orc_acos(float(x))


def cos(x):
    return lib().orc_cos(float(x))


def sin(x):
    return lib().orc_sin(float(x))


def cubic_coeffs(tet24):
    t = np.ascontiguousarray(np.asarray(tet24, dtype=np.float64).reshape(24))
    c = np.zeros(4, dtype=np.float64)
    lib().orc_cubic_coeffs(_ptr(t), _ptr(c))
    return c


def ccd_filter(tet24, k, root):
    t = np.ascontiguousarray(np.asarray(tet24, dtype=np.float64).reshape(24))
    return bool(lib().orc_filter(_ptr(t), int(k), float(root)))


def contact(tet24, k, root, masses4):
    """(normal (3), normal velocity, mass pair (2)) of one contact."""
    t = np.ascontiguousarray(np.asarray(tet24, dtype=np.float64).reshape(24))
    q = np.ascontiguousarray(np.asarray(masses4, dtype=np.float64).reshape(4))
    o = np.zeros(6)
    lib().orc_contact(_ptr(t), int(k), float(root), _ptr(q), _ptr(o))
    return o


def sat(tri_a, tri_b, threshold=0.0):
    a = _c(tri_a)
    b = _c(tri_b, a.dtype)
    return bool(lib().orc_sat(_dt(a), _ptr(a), _ptr(b), float(threshold)))


# ---- comparison helpers -----------------------------------------------------------------

def row_multiset(rows, times=None, ndigits=None):
    """Sorted list of row tuples (optionally with times) for multiset comparison."""
    rows = np.asarray(rows).reshape(len(rows), -1)
    if times is None:
        return sorted(map(tuple, rows.tolist()))
    t = np.asarray(times).reshape(-1)
    return sorted((tuple(r), float(x)) for r, x in zip(rows.tolist(), t.tolist()))
