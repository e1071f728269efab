"""The sm_100a path against the reference extension's own outputs (tests/golden).

In its default mode (CCC_LIB_REFERENCE: CUDA's cbrt / acos / cos / sin / pow / rsqrt, as the
reference calls them, plus the reference's fused multiply-adds written out) the GPU path
reproduces the reference bit for bit: stage outputs of the reference's kernels on sampled
tetrahedra, and the full continuous-collision rows and times of the golden soups.  In the
portable mode it reproduces the CPU oracle bit for bit instead.
"""
import ctypes
import os
from collections import Counter

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
STAGES = ["stages_soup_20_float64", "stages_soup_21_float64", "stages_soup_23_float64", "stages_cloth_sphere"]
SOUPS = ["soup_20_float64", "soup_21_float64", "soup_22_float32", "soup_23_float64"]


def _load(name):
    p = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(p):
        pytest.skip(f"missing fixture {name}")
    return np.load(p)


def _tets(name, d):
    if "tets" in d:
        return d["tets"]
    import sys
    sys.path.insert(0, GOLDEN)
    from make_stage_golden import tets_of
    s = _load(name.replace("stages_", ""))
    return tets_of(s["x0"], s["x1"], d["items"])


def _stage(op, lib, rows, out_w):
    from cccollisions_b200 import _native as N
    x = torch.from_numpy(np.ascontiguousarray(rows, dtype=np.float64)).cuda()
    out = torch.zeros((x.shape[0], out_w), dtype=torch.float64, device="cuda")
    rc = N.lib().ccc_debug_stage(op, lib, ctypes.c_void_p(x.data_ptr()), x.shape[1], ctypes.c_void_p(out.data_ptr()),
                                 out_w, x.shape[0], ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _bits(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return (a.view(np.int64) == b.view(np.int64)) | (np.isnan(a) & np.isnan(b))


@pytest.mark.parametrize("name", STAGES)
def test_stages_bit_exact_with_reference_kernels(cuda, name):
    from cccollisions_b200 import _native as N
    d = _load(name)
    tets = _tets(name, d)
    items = d["items"]
    assert _bits(_stage(0, N.LIB_REFERENCE, tets, 4), d["coefs"]).all()
    roots = _stage(1, N.LIB_REFERENCE, d["coefs"], 3)
    assert _bits(roots, d["roots"]).all(), np.mean(_bits(roots, d["roots"]).all(axis=1))
    fi = d["flt_item"]
    rows = np.concatenate([tets[fi], items[fi][:, 2:3].astype(np.float64), d["flt_root"][:, None]], axis=1)
    flt = _stage(2, N.LIB_REFERENCE, rows, 1)[:, 0] > 0.5
    assert (flt == d["flt_valid"].astype(bool)).all()
    rows_c = np.concatenate([rows, d["ct_mass_quads"]], axis=1)
    ct = _stage(3, N.LIB_REFERENCE, rows_c, 6)
    assert _bits(ct[:, :3], d["ct_normals"]).all()
    assert _bits(ct[:, 3], d["ct_vn"]).all()
    assert _bits(ct[:, 4:6], d["ct_mass_pairs"]).all()


@pytest.mark.parametrize("name", STAGES)
def test_portable_stages_bit_exact_with_oracle(cuda, oracle, name):
    from cccollisions_b200 import _native as N
    d = _load(name)
    tets = _tets(name, d)
    assert _bits(_stage(0, N.LIB_PORTABLE, tets, 4), [oracle.cubic_coeffs(t) for t in tets]).all()
    roots = _stage(1, N.LIB_PORTABLE, d["coefs"], 3)
    assert _bits(roots, [oracle.solve_cubic(*c) for c in d["coefs"]]).all()
    items = d["items"]
    fi = d["flt_item"]
    rows = np.concatenate([tets[fi], items[fi][:, 2:3].astype(np.float64), d["flt_root"][:, None],
                           d["ct_mass_quads"]], axis=1)
    ct = _stage(3, N.LIB_PORTABLE, rows, 6)
    exp = np.array([oracle.contact(tets[i], int(items[i][2]), r, q)
                    for i, r, q in zip(fi, d["flt_root"], d["ct_mass_quads"])])
    assert _bits(ct, exp).all()


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("name", SOUPS + ["cloth_sphere_small"])
def test_continuous_rows_bit_exact_with_reference(cuda, oracle, name):
    import cccollisions_b200 as C
    from cccollisions_b200 import _native as N
    d = _load(name)
    x0, x1 = d["x0"], d["x1"]
    bb, tr = oracle.bvh(x0, x1)     # the reference was fed the same reference-order tree
    with N.math_library(N.LIB_REFERENCE):
        rows, times = C.find_collisions_continuous(_t(bb[None]), _t(tr[None]), _t(x0[None]), _t(x1[None]), 16, 16)
    r = rows[0].cpu().numpy()
    n = int((r[:, 0] >= 0).sum())
    t = times[0, :n, 0].cpu().numpy().astype(np.float64)
    got = Counter(zip(map(tuple, r[:n].tolist()), t.tolist()))
    ref = Counter(zip(map(tuple, d["ccd_rows"].tolist()), d["ccd_times"].astype(np.float64).tolist()))
    assert got == ref, (sum((got - ref).values()), sum((ref - got).values()))


@pytest.mark.parametrize("name", SOUPS)
def test_impulses_match_reference(cuda, oracle, name):
    import cccollisions_b200 as C
    from cccollisions_b200 import _native as N
    d = _load(name)
    x0, x1, m = d["x0"], d["x1"], d["masses"]
    bb, tr = oracle.bvh(x0, x1)
    with N.math_library(N.LIB_REFERENCE):
        dv, dx, cnt = C.compute_impulses(_t(bb[None]), _t(tr[None]), _t(x0[None]), _t(x1[None]), _t(m[None]))
    assert (cnt[0].cpu().numpy() == d["imp_cnt"]).all()
    tol = 1e-6 if x0.dtype == np.float64 else 1e-4
    for got, ref in ((dv, d["imp_dv"]), (dx, d["imp_dx"])):
        g = got[0].cpu().numpy().astype(np.float64)
        r = ref.astype(np.float64)
        assert np.abs(g - r).max() <= tol * np.abs(r).max()


@pytest.mark.parametrize("name", SOUPS)
def test_partial_variants_bit_exact_with_reference(cuda, oracle, name):
    """find_collisions_continuous_partial and compute_impulses_partial in the default mode
    against the reference's own outputs under the fixture's mask, including its mask
    indexing (sorted leaf position on the query side, triangle id on the other,
    src/collisions_continuous.cu:1090, 174-175): equal row multisets with bit-equal times,
    equal counters, dv / dx within 1e-6 (fp64) / 1e-4 (fp32) of the largest."""
    import cccollisions_b200 as C
    from cccollisions_b200 import _native as N
    d = _load(name)
    x0, x1, m, mask = d["x0"], d["x1"], d["masses"], d["mask"]
    bb, tr = oracle.bvh(x0, x1)
    args = (_t(bb[None]), _t(tr[None]), _t(x0[None]), _t(x1[None]))
    with N.math_library(N.LIB_REFERENCE):
        rows, times = C.find_collisions_continuous_partial(*args, _t(mask[None]), 16, 16)
        dv, dx, cnt = C.compute_impulses_partial(*args, _t(m[None]), _t(mask[None]), 16, 16)
    r = rows[0].cpu().numpy()
    n = int((r[:, 0] >= 0).sum())
    t = times[0, :n, 0].cpu().numpy().astype(np.float64)
    got = Counter(zip(map(tuple, r[:n].tolist()), t.tolist()))
    ref = Counter(zip(map(tuple, d["ccdp_rows"].tolist()), d["ccdp_times"].astype(np.float64).tolist()))
    assert n > 0 and got == ref, (sum((got - ref).values()), sum((ref - got).values()))
    assert (cnt[0].cpu().numpy() == d["impp_cnt"]).all()
    tol = 1e-6 if x0.dtype == np.float64 else 1e-4
    for g, want in ((dv, d["impp_dv"]), (dx, d["impp_dx"])):
        g = g[0].cpu().numpy().astype(np.float64)
        want = want.astype(np.float64)
        assert np.abs(g - want).max() <= tol * np.abs(want).max()


def test_static_and_proximity_match_reference(cuda, oracle):
    import cccollisions_b200 as C
    d = _load("static_fold")
    x = d["x"]
    bb, tr = oracle.bvh(x)
    B, T, X = _t(bb[None]), _t(tr[None]), _t(x[None])
    for th in (0.0, 0.005):
        out = C.find_collisions(B, T, X, th, 16)[0].cpu().numpy()
        n = int((out[:, 0] >= 0).sum())
        assert Counter(map(tuple, out[:n].tolist())) == Counter(map(tuple, d[f"static_{th}"].tolist()))
    if "prox_rows" in d:
        (p,) = C.find_proximity(B, T, X, 0.002, 16)
        p = p[0].cpu().numpy()
        n = int((p[:, 0] >= 0).sum())
        assert Counter(map(tuple, p[:n].tolist())) == Counter(map(tuple, d["prox_rows"].tolist()))


TE_CASES = ["te_fold_60_float64", "te_fold_61_float32", "te_fold_70_float32", "te_fold_75_float32",
            "te_fold_75_float64", "te_static_fold"]


@pytest.mark.parametrize("name", TE_CASES)
def test_triangle_edge_queries_match_reference(cuda, name):
    """find_triangle_edge_collisions / _candidates / _candidates2 in the default mode
    (CUDA's rsqrt in the face normal, as the reference) against the reference's own rows:
    equal multisets, edge coefficients bit for bit.  Many crossings of these folds pass
    exactly through a triangle edge (a barycentric coordinate of exactly 0), so the rows
    depend on every rounding of the reference's expressions."""
    import cccollisions_b200 as C
    from cccollisions_b200 import _native as N
    d = _load(name)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    Bb, Tr, X = T(d["bboxes"][None]), T(d["tree"][None]), T(d["x"][None])
    assert N.lib().ccc_get_math_library() == N.LIB_REFERENCE
    rows, coefs = C.find_triangle_edge_collisions(Bb, Tr, X, 0.0, 32)
    r = rows[0].cpu().numpy()
    n = int((r[:, 0] >= 0).sum())
    got = Counter(zip(map(tuple, r[:n].tolist()), coefs[0, :n, 0].cpu().tolist()))
    assert got == Counter(zip(map(tuple, d["te_rows"].tolist()), d["te_coefs"].tolist()))
    c = C.find_triangle_edge_candidates(Bb, Tr, X, 0.0, 32)[0].cpu().numpy()
    c = c[c[:, 0] >= 0]
    assert Counter(map(tuple, c.tolist())) == Counter(map(tuple, d["cand_rows"].tolist()))
    pairs, masks = C.find_triangle_edge_candidates2(Bb, Tr, X, 0.0, 32)
    p, m = pairs[0].cpu().numpy(), masks[0].cpu().numpy()
    k = p[:, 0] >= 0
    assert Counter(zip(map(tuple, p[k].tolist()), map(tuple, m[k].tolist()))) == \
        Counter(zip(map(tuple, d["cand2_pairs"].tolist()), map(tuple, d["cand2_masks"].tolist())))
