"""Drop-in Python API of the reference torch extension ``cccollisions``.

Same function names, argument names, defaults, output shapes and dtypes as the
reference's pybind module (Dolorousrtur/CCCollisions src/cccollisions.cpp:426-468).  Each
function checks its tensors like the reference's CHECK_INPUT (CUDA + contiguous, raising
RuntimeError), allocates the outputs exactly as the reference does (-1 filled rows, zeroed
impulses), and calls the native library through its C ABI on the current CUDA stream.

Capacity overflows print the reference's warnings (as ``warnings.warn``) and truncate like
the reference; set ``cccollisions_b200.api.STRICT = True`` to raise instead.  Set
``CHECK_STATUS = False`` to skip the status read-back (one small synchronising copy per
call) when running inside CUDA graphs or tight loops.
"""
from __future__ import annotations

import ctypes
import warnings

import torch

from . import _native as N

STRICT = False
CHECK_STATUS = True

_MSG_CAND = ("Number of candidate collisions exceeds maximal allowed number. "
             "Some of the candidate collisions are omitted.")
_MSG_OUT = "Number of actual collisions exceeds maximal allowed number. Some of the collisions are omitted."


def _check_input(t, name):
    if not isinstance(t, torch.Tensor):
        raise RuntimeError(f"{name} must be a torch.Tensor")
    if not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise RuntimeError(f"{name} must be contiguous")


def _dtype_code(t):
    if t.dtype == torch.float32:
        return 0
    if t.dtype == torch.float64:
        return 1
    raise RuntimeError(f"unsupported floating type {t.dtype} (float32 or float64)")


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _workspace(op, B, F, maxc, device):
    n = N.lib().ccc_workspace_size(op, B, F, maxc)
    if n < 0:
        raise RuntimeError("invalid sizes for workspace")
    return torch.empty(int(n), dtype=torch.uint8, device=device)


def _report(ws, device, B, what):
    if not CHECK_STATUS:
        return 0
    out = (ctypes.c_int32 * 2)()
    N.check(N.lib().ccc_read_status(_ptr(ws), 0, out, _stream(device)), what)
    st = int(out[0])
    if st & (N.CCC_ST_STACK_OVERFLOW | N.CCC_ST_MALFORMED_TREE):
        raise RuntimeError(f"{what}: traversal failed (status {st}: "
                           f"{'stack overflow' if st & N.CCC_ST_STACK_OVERFLOW else 'malformed tree'})")
    if st & N.CCC_ST_CAND_OVERFLOW or st & N.CCC_ST_OUT_OVERFLOW:
        msg = _MSG_CAND if st & N.CCC_ST_CAND_OVERFLOW else _MSG_OUT
        if STRICT:
            raise RuntimeError(msg)
        warnings.warn(msg, RuntimeWarning, stacklevel=3)
    return st


def _num_tris_from_bboxes(bboxes):
    return (bboxes.size(1) + 1) // 2


def _mask_ptr(mask):
    if mask is None:
        return None
    _check_input(mask, "triangles_to_check")
    if mask.dtype not in (torch.bool, torch.uint8):
        raise RuntimeError("triangles_to_check must be a bool tensor")
    return _ptr(mask)


def _with_device(t):
    return torch.cuda.device(t.device)


def bvh(triangles):
    """bvh(triangles) -> [bboxes (B, 2F-1, 6), tree (B, 2F-1, 4) int64] (cccollisions.cpp:102-116)."""
    _check_input(triangles, "triangles")
    return _bvh(triangles, None)


def bvh_motion(triangles, triangles_next):
    """bvh_motion(triangles, triangles_next) -> [bboxes, tree] over swept boxes (cccollisions.cpp:118-132)."""
    _check_input(triangles, "triangles")
    _check_input(triangles_next, "triangles_next")
    if triangles_next.shape != triangles.shape or triangles_next.dtype != triangles.dtype:
        raise RuntimeError("triangles_next must match triangles in shape and dtype")
    return _bvh(triangles, triangles_next)


def _bvh(triangles, triangles_next):
    B, F = triangles.size(0), triangles.size(1)
    dev = triangles.device
    bboxes = -1 * torch.ones((B, 2 * F - 1, 6), dtype=triangles.dtype, device=dev)
    tree = -1 * torch.ones((B, 2 * F - 1, 4), dtype=torch.int64, device=dev)
    with _with_device(triangles):
        ws = _workspace(N.OP_BVH, B, F, 0, dev)
        rc = N.lib().ccc_bvh(_dtype_code(triangles), _ptr(triangles), _ptr(triangles_next), B, F, _ptr(bboxes),
                             _ptr(tree), _ptr(ws), ws.numel(), _stream(dev))
        N.check(rc, "bvh")
        _report(ws, dev, B, "bvh")
    return [bboxes, tree]


def find_collisions(bboxes, tree, triangles, threshold=0., max_collisions=16):
    """Static triangle-triangle intersections (cccollisions.cpp:134-148): (B, F*max_collisions, 2) int64."""
    for t, nme in ((bboxes, "bboxes"), (tree, "tree"), (triangles, "triangles")):
        _check_input(t, nme)
    B, F = bboxes.size(0), _num_tris_from_bboxes(bboxes)
    dev = bboxes.device
    out = -1 * torch.ones((B, F * max_collisions, 2), dtype=torch.int64, device=dev)
    with _with_device(bboxes):
        ws = _workspace(N.OP_FIND_COLLISIONS, B, F, max_collisions, dev)
        rc = N.lib().ccc_find_collisions(_dtype_code(bboxes), _ptr(bboxes), _ptr(tree), _ptr(triangles), B, F,
                                         float(threshold), max_collisions, _ptr(out), _ptr(ws), ws.numel(),
                                         _stream(dev))
        N.check(rc, "find_collisions")
        _report(ws, dev, B, "find_collisions")
    return out


def _continuous(bboxes, tree, triangles, triangles_next, mask, maxc, maxcol, what):
    for t, nme in ((bboxes, "bboxes"), (tree, "tree"), (triangles, "triangles"), (triangles_next, "triangles_next")):
        _check_input(t, nme)
    B, F = bboxes.size(0), _num_tris_from_bboxes(bboxes)
    dev = bboxes.device
    rows = -1 * torch.ones((B, F * maxcol, 3), dtype=torch.int64, device=dev)
    times = -1 * torch.ones((B, F * maxcol, 1), dtype=bboxes.dtype, device=dev)
    with _with_device(bboxes):
        ws = _workspace(N.OP_CONTINUOUS, B, F, maxc, dev)
        rc = N.lib().ccc_find_collisions_continuous(_dtype_code(bboxes), _ptr(bboxes), _ptr(tree), _ptr(triangles),
                                                    _ptr(triangles_next), _mask_ptr(mask), B, F, maxc, maxcol,
                                                    _ptr(rows), _ptr(times), _ptr(ws), ws.numel(), _stream(dev))
        N.check(rc, what)
        _report(ws, dev, B, what)
    return [rows, times]


def find_collisions_continuous(bboxes, tree, triangles, triangles_next, max_candidates_per_triangle=16,
                               max_collisions_per_triangle=16):
    """Continuous collisions (cccollisions.cpp:220-245): [(B, F*mc, 3) int64 (i, j, type), (B, F*mc, 1) TOI]."""
    return _continuous(bboxes, tree, triangles, triangles_next, None, max_candidates_per_triangle,
                       max_collisions_per_triangle, "find_collisions_continuous")


def find_collisions_continuous_partial(bboxes, tree, triangles, triangles_next, triangles_to_check,
                                       max_candidates_per_triangle=16, max_collisions_per_triangle=16):
    """Masked continuous collisions (cccollisions.cpp:247-273)."""
    return _continuous(bboxes, tree, triangles, triangles_next, triangles_to_check, max_candidates_per_triangle,
                       max_collisions_per_triangle, "find_collisions_continuous_partial")


def find_proximity(bboxes, tree, triangles, threshold, max_candidates_per_triangle=16):
    """Pairs of features closer than threshold (cccollisions.cpp:276-296): [(B, F*mc, 3) int64]."""
    for t, nme in ((bboxes, "bboxes"), (tree, "tree"), (triangles, "triangles")):
        _check_input(t, nme)
    B, F = bboxes.size(0), _num_tris_from_bboxes(bboxes)
    dev = bboxes.device
    rows = -1 * torch.ones((B, F * max_candidates_per_triangle, 3), dtype=torch.int64, device=dev)
    with _with_device(bboxes):
        ws = _workspace(N.OP_PROXIMITY, B, F, max_candidates_per_triangle, dev)
        rc = N.lib().ccc_find_proximity(_dtype_code(bboxes), _ptr(bboxes), _ptr(tree), _ptr(triangles), B, F,
                                        float(threshold), max_candidates_per_triangle, _ptr(rows), _ptr(ws),
                                        ws.numel(), _stream(dev))
        N.check(rc, "find_proximity")
        _report(ws, dev, B, "find_proximity")
    return [rows]


def find_mincol_cand(bboxes, tree, triangles, triangles_next, max_collisions=16):
    """Sub-tests whose swept sub-boxes overlap (cccollisions.cpp:405-423): (B, F*mc*15, 3) int64."""
    for t, nme in ((bboxes, "bboxes"), (tree, "tree"), (triangles, "triangles"), (triangles_next, "triangles_next")):
        _check_input(t, nme)
    B, F = bboxes.size(0), _num_tris_from_bboxes(bboxes)
    dev = bboxes.device
    rows = -1 * torch.ones((B, F * max_collisions * 15, 3), dtype=torch.int64, device=dev)
    with _with_device(bboxes):
        ws = _workspace(N.OP_MINCOL, B, F, max_collisions, dev)
        rc = N.lib().ccc_find_mincol_cand(_dtype_code(bboxes), _ptr(bboxes), _ptr(tree), _ptr(triangles),
                                          _ptr(triangles_next), B, F, max_collisions, _ptr(rows), _ptr(ws),
                                          ws.numel(), _stream(dev))
        N.check(rc, "find_mincol_cand")
        _report(ws, dev, B, "find_mincol_cand")
    return rows


def _impulse_outputs(B, F, dtype, dev):
    dv = torch.zeros((B, F, 3, 3), dtype=dtype, device=dev)
    dx = torch.zeros((B, F, 3, 3), dtype=dtype, device=dev)
    cnt = torch.zeros((B, F, 3), dtype=torch.int32, device=dev)
    return dv, dx, cnt


def _impulses(bboxes, tree, triangles, triangles_next, triangles_mass, mask, maxc, maxcol, what):
    for t, nme in ((bboxes, "bboxes"), (tree, "tree"), (triangles, "triangles"), (triangles_next, "triangles_next"),
                   (triangles_mass, "triangles_masses")):
        _check_input(t, nme)
    B, F = bboxes.size(0), _num_tris_from_bboxes(bboxes)
    dev = bboxes.device
    dv, dx, cnt = _impulse_outputs(B, F, bboxes.dtype, dev)
    with _with_device(bboxes):
        ws = _workspace(N.OP_IMPULSES, B, F, maxc, dev)
        rc = N.lib().ccc_compute_impulses(_dtype_code(bboxes), _ptr(bboxes), _ptr(tree), _ptr(triangles),
                                          _ptr(triangles_next), _ptr(triangles_mass), _mask_ptr(mask), B, F, maxc,
                                          maxcol, _ptr(dv), _ptr(dx), _ptr(cnt), _ptr(ws), ws.numel(), _stream(dev))
        N.check(rc, what)
        _report(ws, dev, B, what)
    return [dv, dx, cnt]


def compute_impulses(bboxes, tree, triangles, triangles_next, triangles_mass, max_candidates_per_triangle=16,
                     max_collisions_per_triangle=16):
    """Per-corner impulses of all continuous collisions (cccollisions.cpp:299-333): [dv, dx, counter]."""
    return _impulses(bboxes, tree, triangles, triangles_next, triangles_mass, None, max_candidates_per_triangle,
                     max_collisions_per_triangle, "compute_impulses")


def compute_impulses_partial(bboxes, tree, triangles, triangles_next, triangles_mass, triangles_to_check,
                             max_candidates_per_triangle=16, max_collisions_per_triangle=16):
    """Masked variant of compute_impulses (cccollisions.cpp:336-370)."""
    return _impulses(bboxes, tree, triangles, triangles_next, triangles_mass, triangles_to_check,
                     max_candidates_per_triangle, max_collisions_per_triangle, "compute_impulses_partial")


def compute_impulses_from_collisions(collisions, roots, triangles, triangles_next, triangles_mass):
    """Impulses from given (collisions (B,N,3), roots (B,N,1)) rows (cccollisions.cpp:374-403).

    Rows whose indices are out of range (e.g. the -1 padding of find_collisions_continuous)
    are skipped instead of being read out of bounds.
    """
    for t, nme in ((collisions, "collisions"), (roots, "roots"), (triangles, "triangles"),
                   (triangles_next, "triangles_next"), (triangles_mass, "triangles_masses")):
        _check_input(t, nme)
    B, F = triangles.size(0), triangles.size(1)
    Nr = collisions.size(1)
    dev = triangles.device
    dv, dx, cnt = _impulse_outputs(B, F, triangles.dtype, dev)
    with _with_device(triangles):
        ws = _workspace(N.OP_BVH, B, F, 0, dev)
        rc = N.lib().ccc_compute_impulses_from_collisions(_dtype_code(triangles), _ptr(collisions), _ptr(roots), B,
                                                          Nr, _ptr(triangles), _ptr(triangles_next),
                                                          _ptr(triangles_mass), F, _ptr(dv), _ptr(dx), _ptr(cnt),
                                                          _ptr(ws), ws.numel(), _stream(dev))
        N.check(rc, "compute_impulses_from_collisions")
    return [dv, dx, cnt]


def _triangle_edge(bboxes, tree, triangles):
    for t, nme in ((bboxes, "bboxes"), (tree, "tree"), (triangles, "triangles")):
        _check_input(t, nme)
    return bboxes.size(0), _num_tris_from_bboxes(bboxes), bboxes.device


def find_triangle_edge_collisions(bboxes, tree, triangles, threshold=0., max_collisions=16):
    """Edges crossing triangles of intersecting pairs (cccollisions.cpp:151-173):
    [(B, F*mc, 4) int64 (i, j, cid, flag), (B, F*mc, 1) edge coefficients].

    ``threshold`` is accepted and unused, as in the reference (its queries use 0)."""
    B, F, dev = _triangle_edge(bboxes, tree, triangles)
    rows = -1 * torch.ones((B, F * max_collisions, 4), dtype=torch.int64, device=dev)
    coefs = -1 * torch.ones((B, F * max_collisions, 1), dtype=bboxes.dtype, device=dev)
    with _with_device(bboxes):
        ws = _workspace(N.OP_FIND_COLLISIONS, B, F, max_collisions, dev)
        rc = N.lib().ccc_find_triangle_edge_collisions(_dtype_code(bboxes), _ptr(bboxes), _ptr(tree), _ptr(triangles),
                                                       B, F, max_collisions, _ptr(rows), _ptr(coefs), _ptr(ws),
                                                       ws.numel(), _stream(dev))
        N.check(rc, "find_triangle_edge_collisions")
        _report(ws, dev, B, "find_triangle_edge_collisions")
    return [rows, coefs]


def find_triangle_edge_candidates(bboxes, tree, triangles, threshold=0., max_collisions=16):
    """Edge / face sub-tests of the pairs sharing at most one vertex (cccollisions.cpp:176-194):
    (B, F*mc, 4) int64 (i, j, cid, flag).  ``threshold`` is unused, as in the reference."""
    B, F, dev = _triangle_edge(bboxes, tree, triangles)
    rows = -1 * torch.ones((B, F * max_collisions, 4), dtype=torch.int64, device=dev)
    with _with_device(bboxes):
        ws = _workspace(N.OP_FIND_COLLISIONS, B, F, max_collisions, dev)
        rc = N.lib().ccc_find_triangle_edge_candidates(_dtype_code(bboxes), _ptr(bboxes), _ptr(tree), _ptr(triangles),
                                                       B, F, max_collisions, _ptr(rows), _ptr(ws), ws.numel(),
                                                       _stream(dev))
        N.check(rc, "find_triangle_edge_candidates")
        _report(ws, dev, B, "find_triangle_edge_candidates")
    return rows


def find_triangle_edge_candidates2(bboxes, tree, triangles, threshold=0., max_collisions=16):
    """The pairs of find_triangle_edge_candidates with their sub-test bit masks
    (cccollisions.cpp:197-218): [(B, F*mc, 2) int64 pairs, (B, F*mc, 2) int32 masks].
    ``threshold`` is unused, as in the reference."""
    B, F, dev = _triangle_edge(bboxes, tree, triangles)
    pairs = -1 * torch.ones((B, F * max_collisions, 2), dtype=torch.int64, device=dev)
    masks = torch.zeros((B, F * max_collisions, 2), dtype=torch.int32, device=dev)
    with _with_device(bboxes):
        ws = _workspace(N.OP_FIND_COLLISIONS, B, F, max_collisions, dev)
        rc = N.lib().ccc_find_triangle_edge_candidates2(_dtype_code(bboxes), _ptr(bboxes), _ptr(tree),
                                                        _ptr(triangles), B, F, max_collisions, _ptr(pairs),
                                                        _ptr(masks), _ptr(ws), ws.numel(), _stream(dev))
        N.check(rc, "find_triangle_edge_candidates2")
        _report(ws, dev, B, "find_triangle_edge_candidates2")
    return [pairs, masks]
