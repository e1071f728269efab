"""The C ABI library builds, loads without a GPU and exports every declared symbol."""
import os
import re

import pytest

from conftest import ROOT


def _declared_functions():
    names = set()
    for h in ("ccc_b200.h", "ccc_engine.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(ccc_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_header_declares_the_reference_entry_points():
    names = _declared_functions()
    for n in ("ccc_bvh", "ccc_find_collisions", "ccc_find_collisions_continuous", "ccc_find_proximity",
              "ccc_find_mincol_cand", "ccc_compute_impulses", "ccc_compute_impulses_from_collisions",
              "ccc_workspace_size", "ccc_read_status"):
        assert n in names


def _declarations():
    """(name, [parameter text]) of every function the headers declare."""
    out = []
    for h in ("ccc_b200.h", "ccc_engine.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(ccc_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", src):
            args = m.group(2).strip()
            out.append((m.group(1), [] if args in ("", "void") else args.split(",")))
    return out


def _c_kind(param):
    if "*" in param:
        return "pointer"
    if "int64_t" in param:
        return "int64"
    if "double" in param:
        return "double"
    if re.search(r"\b(int|int32_t)\b", param):
        return "int32"
    return "unknown: " + param


def _ctypes_kind(t):
    import ctypes
    if t in (ctypes.c_void_p, ctypes.c_char_p) or isinstance(getattr(t, "_type_", None), type):
        return "pointer"
    return {ctypes.c_int64: "int64", ctypes.c_int32: "int32", ctypes.c_double: "double"}.get(t, str(t))


def test_ctypes_signatures_match_the_headers():
    """Every ctypes signature the package binds has the header's parameter count and, per
    parameter, the same kind (pointer, 64-bit integer, 32-bit integer, double)."""
    from cccollisions_b200 import _native
    decls = _declarations()
    assert len(decls) == len(_declared_functions())
    for name, params in decls:
        sig = _native.SIGNATURES[name][1]
        assert len(sig) == len(params), name
        for i, (p, t) in enumerate(zip(params, sig)):
            assert _c_kind(p) == _ctypes_kind(t), (name, i, p, t)


def test_library_exports_every_declared_symbol(native_lib):
    from cccollisions_b200 import _native
    for name in _declared_functions():
        assert hasattr(native_lib, name), name
        assert name in _native.SIGNATURES, name


def test_pure_host_calls(native_lib):
    from cccollisions_b200 import _native as N
    assert native_lib.ccc_version() >= 1
    assert native_lib.ccc_error_string(N.CCC_OK) == b"ok"
    for op in range(6):
        a = native_lib.ccc_workspace_size(op, 1, 1000, 16)
        b = native_lib.ccc_workspace_size(op, 2, 1000, 16)
        assert 0 < a <= b
    assert native_lib.ccc_workspace_size(0, 1, 1, 16) == -1      # F >= 2 is required
    # argument errors are reported before any device work (no GPU touched)
    rc = native_lib.ccc_bvh(7, None, None, 1, 10, None, None, None, 0, None)
    assert rc == 1
    rc = native_lib.ccc_find_collisions(0, None, None, None, 1, 1, 0.0, 16, None, None, 0, None)
    assert rc == 1


def test_engine_sizes_are_pure_host(native_lib):
    small = native_lib.ccc_engine_bytes(1, 1000, 500, 4, 16, 16)
    big = native_lib.ccc_engine_bytes(1, 2000, 500, 4, 16, 16)
    assert 0 < small < big
    assert native_lib.ccc_engine_bytes(0, 1000, 500, 4, 16, 16) < small      # fp32 positions
    assert native_lib.ccc_engine_bytes(2, 1000, 0, 4, 16, 16) == -1          # dtype
    assert native_lib.ccc_engine_bytes(1, 1, 0, 4, 16, 16) == -1             # F >= 2
    assert native_lib.ccc_engine_bytes(1, 1 << 27, 0, 4, 16, 16) == -1       # candidate slots > 2^31
    # argument errors before any device work
    assert native_lib.ccc_engine_create(1, 1000, 0, 4, 16, 16, None, 0, None, None) == 1
    assert native_lib.ccc_engine_ccd(None, None) == 1
    assert native_lib.ccc_engine_pack_rows(None, None, None, 0, None, None) == 1
    # triangle-edge queries: bad dtype, too few triangles, missing outputs
    te = (native_lib.ccc_find_triangle_edge_collisions, native_lib.ccc_find_triangle_edge_candidates2)
    assert native_lib.ccc_find_triangle_edge_collisions(7, None, None, None, 1, 4, 16, None, None, None, 0, None) == 1
    assert native_lib.ccc_find_triangle_edge_candidates(1, None, None, None, 1, 1, 16, None, None, 0, None) == 1
    for f in te:
        assert f(1, None, None, None, 1, 4, 16, None, None, None, 0, None) == 1


def test_api_mirrors_reference_signatures():
    import inspect
    import cccollisions_b200 as C
    sig = lambda f: list(inspect.signature(f).parameters.items())
    p = sig(C.find_collisions)
    assert [k for k, _ in p] == ["bboxes", "tree", "triangles", "threshold", "max_collisions"]
    assert p[3][1].default == 0.0 and p[4][1].default == 16
    p = sig(C.find_collisions_continuous)
    assert [k for k, _ in p] == ["bboxes", "tree", "triangles", "triangles_next", "max_candidates_per_triangle",
                                 "max_collisions_per_triangle"]
    p = sig(C.compute_impulses_partial)
    assert [k for k, _ in p][:6] == ["bboxes", "tree", "triangles", "triangles_next", "triangles_mass",
                                     "triangles_to_check"]
    assert [k for k, _ in sig(C.find_proximity)] == ["bboxes", "tree", "triangles", "threshold",
                                                    "max_candidates_per_triangle"]
    assert [k for k, _ in sig(C.compute_impulses_from_collisions)] == ["collisions", "roots", "triangles",
                                                                      "triangles_next", "triangles_mass"]
    for f in (C.find_triangle_edge_collisions, C.find_triangle_edge_candidates, C.find_triangle_edge_candidates2):
        p = sig(f)
        assert [k for k, _ in p] == ["bboxes", "tree", "triangles", "threshold", "max_collisions"]
        assert p[3][1].default == 0.0 and p[4][1].default == 16
        with pytest.raises(RuntimeError, match="torch.Tensor"):
            f(None, None, None)


def test_api_rejects_cpu_tensors():
    import torch
    import cccollisions_b200 as C
    t = torch.zeros((1, 4, 3, 3))
    with pytest.raises(RuntimeError, match="CUDA"):
        C.bvh(t)


def test_served_engine_capacity_fits_the_budget(native_lib):
    """The server sizes its engine block from a device-memory budget (pure host): the
    largest triangle capacity whose block fits beside the library's fixed module-data
    array, so one triangle more does not fit (or exceeds the engine's limits)."""
    import torch
    from cccollisions_b200.serve import engine_capacity
    fixed = native_lib.ccc_static_scratch_bytes()
    assert fixed == 64 << 20
    prev = 0
    for gb in (1, 2, 40):
        budget = gb << 30
        tc, vc = engine_capacity(budget, torch.float64, mesh_capacity=4096, vert_ratio=0.75, maxc=16)
        assert tc > prev
        prev = tc
        assert vc == int(tc * 0.75) + 16
        assert 0 < native_lib.ccc_engine_bytes(1, tc, vc, 4096, 16, 1) <= budget - fixed
        over = native_lib.ccc_engine_bytes(1, tc + 1, int((tc + 1) * 0.75) + 16, 4096, 16, 1)
        assert over > budget - fixed or over == -1


def test_size_checks_cannot_wrap(native_lib):
    """Capacity checks divide rather than multiply, so per-triangle capacities near 2^63
    (whose products with B * F would wrap to small numbers) are argument errors, before
    any pointer is touched; so are batch and triangle counts whose product would wrap."""
    from cccollisions_b200 import _native as N
    huge = 1 << 44
    assert native_lib.ccc_workspace_size(N.OP_CONTINUOUS, 1, 1 << 20, huge) == -1
    assert native_lib.ccc_workspace_size(N.OP_CONTINUOUS, 1 << 40, 1 << 40, 16) == -1
    assert native_lib.ccc_workspace_size(N.OP_CONTINUOUS, 1, 1 << 20, 16) > 0
    args = (None, None, None, None, None, 1, 1 << 20, huge, 16, None, None)
    assert native_lib.ccc_find_collisions_continuous(1, *args, None, 0, None) == N.CCC_ERR_INVALID_ARG
    assert native_lib.ccc_find_collisions_continuous_static(1, *args, None) == N.CCC_ERR_INVALID_ARG
    assert native_lib.ccc_find_collisions_continuous_static(1, None, None, None, None, None, 1 << 40, 1 << 40, 16, 16,
                                                            None, None, None) == N.CCC_ERR_INVALID_ARG
    assert native_lib.ccc_compute_impulses(1, None, None, None, None, None, None, 1, 1 << 20, huge, 16, None, None,
                                           None, None, 0, None) == N.CCC_ERR_INVALID_ARG
    assert native_lib.ccc_find_mincol_cand(1, None, None, None, None, 1, 1 << 20, huge, None, None, 0,
                                           None) == N.CCC_ERR_INVALID_ARG


def test_reference_module_name_imports_the_drop_in(native_lib):
    """``import cccollisions`` (the reference's module name) gives this library's functions,
    with the reference's argument names and defaults."""
    import inspect

    import cccollisions
    import cccollisions_b200
    assert sorted(cccollisions.__all__) == sorted(cccollisions_b200.__all__)
    for name in cccollisions_b200.__all__:
        assert getattr(cccollisions, name) is getattr(cccollisions_b200, name)
    sig = inspect.signature(cccollisions.find_collisions_continuous)
    assert list(sig.parameters) == ["bboxes", "tree", "triangles", "triangles_next", "max_candidates_per_triangle",
                                    "max_collisions_per_triangle"]
    assert sig.parameters["max_candidates_per_triangle"].default == 16
    sig = inspect.signature(cccollisions.compute_impulses)
    assert list(sig.parameters)[:5] == ["bboxes", "tree", "triangles", "triangles_next", "triangles_mass"]


def test_engine_schedules_are_described(native_lib):
    """The autotuner's candidates cover both traversal forms, 0-2 tree levels staged in
    shared memory and both narrow batch sizes; out-of-range choices are argument errors (no
    engine or device needed)."""
    import ctypes

    from cccollisions_b200 import _native as N
    n = native_lib.ccc_engine_schedule_count()
    assert n >= 2
    forms, stages, batches = set(), set(), set()
    for i in range(n):
        a = (ctypes.c_int32 * 5)()
        assert native_lib.ccc_engine_schedule_info(i, a) == 0
        assert a[0] > 0 and a[1] > 0 and a[2] in (0, 1) and a[3] in (0, 1, 2) and a[4] in (1, 2)
        assert a[3] == 0 or a[2] == 0
        forms.add(a[2])
        stages.add(a[3])
        batches.add(a[4])
    assert forms == {0, 1} and stages == {0, 1, 2} and batches == {1, 2}
    a = (ctypes.c_int32 * 5)()
    assert native_lib.ccc_engine_schedule_info(n, a) == N.CCC_ERR_INVALID_ARG
    assert native_lib.ccc_engine_set_schedule(None, 0) == N.CCC_ERR_INVALID_ARG
