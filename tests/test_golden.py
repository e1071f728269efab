"""The CPU oracle against outputs of the reference extension itself.

tests/golden/*.npz were written by tests/golden/make_golden.py, which ran the reference's
own compiled extension (built from its sources by oracle/build_ref.py) on a B200 with
seeded inputs.  The trees fed to it are the oracle's reference-order builds.

Bars:
  * candidate sub-tests (find_mincol_cand), static intersections (find_collisions, fp32
    and fp64, two thresholds) and proximity rows: equal as multisets;
  * impulses from the reference's own collision rows (compute_impulses_from_collisions):
    counters equal, dv / dx within 1e-12 relative (fp64) / 1e-3 relative (fp32);
  * continuous-collision rows: the oracle writes out the fused multiply-adds that nvcc's
    default contraction puts into the reference (coefficients, discriminant, roots), so its
    arithmetic matches the reference's except in the elementary functions: its own cbrt /
    acos / cos / sin differ from CUDA's by an ulp on part of the inputs, which moves a root
    by an ulp and, near t = 0 or at a filter boundary, a row (bounded below).  The GPU
    path in its default mode calls CUDA's functions and matches bit for bit (GPU tests).
"""
import os
from collections import Counter

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SOUPS = ["soup_20_float64", "soup_21_float64", "soup_22_float32", "soup_23_float64"]


def _ms(a):
    return Counter(map(tuple, np.asarray(a).reshape(len(a), -1).tolist()))


def _load(name):
    p = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(p):
        pytest.skip(f"missing fixture {name}")
    return np.load(p)


@pytest.mark.parametrize("name", SOUPS)
def test_mincol_static_proximity_match_reference(oracle, name):
    d = _load(name)
    x0, x1 = d["x0"], d["x1"]
    bb, tr = oracle.bvh(x0, x1)
    bbs, trs = oracle.bvh(x0)
    assert _ms(d["mincol_rows"]) == _ms(oracle.mincol_cand(bb, tr, x0, x1))
    for th in (0.0, 0.005):
        assert _ms(d[f"static_{th}"]) == _ms(oracle.find_collisions(bbs, trs, x0, threshold=th))
    assert _ms(d["prox_rows"]) == _ms(oracle.proximity(bbs, trs, x0, 0.02)[0])


def test_static_fold_matches_reference(oracle):
    d = _load("static_fold")
    x = d["x"]
    bb, tr = oracle.bvh(x)
    for th in (0.0, 0.005):
        ref = d[f"static_{th}"]
        assert len(ref) > 1000
        assert _ms(ref) == _ms(oracle.find_collisions(bb, tr, x, threshold=th))
    if "prox_rows" in d:
        assert _ms(d["prox_rows"]) == _ms(oracle.proximity(bb, tr, x, 0.002)[0])


@pytest.mark.parametrize("name", SOUPS)
def test_impulses_from_reference_rows(oracle, name):
    d = _load(name)
    x0, x1, m = d["x0"], d["x1"], d["masses"]
    dv, dx, cnt = oracle.impulses_from_rows(x0, x1, m, d["ccd_rows"], d["ccd_times"])
    assert (cnt == d["impr_cnt"]).all()
    tol = 1e-12 if x0.dtype == np.float64 else 1e-3
    for got, ref in ((dv, d["impr_dv"]), (dx, d["impr_dx"])):
        scale = np.abs(ref).max()
        assert np.abs(got - ref).max() <= tol * scale


@pytest.mark.parametrize("name", SOUPS + ["cloth_sphere_small"])
def test_continuous_rows_close_to_reference(oracle, name):
    d = _load(name)
    x0, x1 = d["x0"], d["x1"]
    bb, tr = oracle.bvh(x0, x1)
    er, et = oracle.ccd(bb, tr, x0, x1)
    ref, orc = _ms(d["ccd_rows"]), _ms(er)
    differing = sum((ref - orc).values()) + sum((orc - ref).values())
    total = max(len(d["ccd_rows"]), 1)
    if name == "cloth_sphere_small":
        # flat cloth: coplanar pairs give roots within a few ulps of t = 0, whose sign
        # decides the row; every row the reference reports is also found by the oracle
        assert not (ref - orc)
    else:
        assert differing <= 0.1 * total, (differing, total)


@pytest.mark.parametrize("name", SOUPS)
def test_partial_variants_match_reference(oracle, name):
    """find_collisions_continuous_partial / compute_impulses_partial of the reference under
    the fixture's mask (``ccdp_*``, ``impp_*``).  The reference indexes the mask by sorted
    leaf position on the query side and by triangle id on the other
    (src/collisions_continuous.cu:1090, 174-175): every pair of its rows is a candidate of
    the oracle's masked traversal, which restates that quirk, and the rows agree as closely
    as the unmasked ones (elementary-function ulps).  Its impulses are those of its own
    partial rows: counters equal, dv / dx within 1e-12 (fp64) / 1e-6 (fp32) of the largest."""
    d = _load(name)
    x0, x1, m = d["x0"], d["x1"], d["masses"]
    mask = d["mask"].astype(np.uint8)
    assert 0 < mask.sum() < len(mask)
    bb, tr = oracle.bvh(x0, x1)
    cand = set(map(tuple, oracle.candidates(bb, tr, mask=mask).tolist()))
    full = set(map(tuple, oracle.candidates(bb, tr).tolist()))
    assert len(cand) < len(full)
    ref_pairs = {(a, b) for a, b, _ in d["ccdp_rows"].tolist()}
    assert ref_pairs and ref_pairs <= cand
    er, _ = oracle.ccd(bb, tr, x0, x1, mask=mask)
    ref, orc = _ms(d["ccdp_rows"]), _ms(er)
    differing = sum((ref - orc).values()) + sum((orc - ref).values())
    assert differing <= 0.1 * max(len(d["ccdp_rows"]), 1), differing
    dv, dx, cnt = oracle.impulses_from_rows(x0, x1, m, d["ccdp_rows"], d["ccdp_times"])
    assert (cnt == d["impp_cnt"]).all()
    tol = 1e-12 if x0.dtype == np.float64 else 1e-6
    for got, want in ((dv, d["impp_dv"]), (dx, d["impp_dx"])):
        assert np.abs(got - want).max() <= tol * np.abs(want).max()


# ------------------------------------------------------------------ stage by stage
# tests/golden/stages_*.npz hold, for sampled (i, j, type) sub-tests, the outputs of the
# reference's own kernels (getCubicCoeffs, solveCubic, filterCollisions,
# compute_coeficients_and_directions), recorded by tests/golden/make_stage_golden.py.

STAGES = ["stages_soup_20_float64", "stages_soup_21_float64", "stages_soup_23_float64", "stages_cloth_sphere"]


def _stage_tets(name, d):
    if "tets" in d:
        return d["tets"]
    import sys
    sys.path.insert(0, GOLDEN)
    from make_stage_golden import tets_of
    s = _load(name.replace("stages_", ""))
    return tets_of(s["x0"], s["x1"], d["items"])


@pytest.mark.parametrize("name", STAGES)
def test_cubic_coefficients_bit_exact_with_reference(oracle, name):
    # the oracle's fma model of nvcc's contraction reproduces the reference's coefficients
    d = _load(name)
    tets = _stage_tets(name, d)
    got = np.array([oracle.cubic_coeffs(t) for t in tets])
    assert (got.view(np.int64) == d["coefs"].view(np.int64)).all()


@pytest.mark.parametrize("name", STAGES)
def test_root_filter_bit_exact_with_reference(oracle, name):
    d = _load(name)
    tets = _stage_tets(name, d)
    items = d["items"]
    got = [oracle.ccd_filter(tets[i], int(items[i][2]), r) for i, r in zip(d["flt_item"], d["flt_root"])]
    assert list(map(bool, got)) == list(map(bool, d["flt_valid"]))


@pytest.mark.parametrize("name", STAGES)
def test_contact_kinematics_close_to_reference(oracle, name):
    # normals use the reference's rsqrt on the GPU and 1/sqrt here: agreement to 1e-14
    d = _load(name)
    tets = _stage_tets(name, d)
    items = d["items"]
    for n, (i, r) in enumerate(zip(d["flt_item"], d["flt_root"])):
        o = oracle.contact(tets[i], int(items[i][2]), r, d["ct_mass_quads"][n])
        ref_n = d["ct_normals"][n]
        if not np.isfinite(ref_n).all():
            continue
        assert np.allclose(o[:3], ref_n, rtol=0, atol=1e-14)
        assert np.allclose(o[4:6], d["ct_mass_pairs"][n], rtol=1e-15, atol=0)
        assert abs(o[3] - d["ct_vn"][n]) <= 1e-13 * max(abs(d["ct_vn"][n]), 1e-3)


@pytest.mark.parametrize("name", STAGES)
def test_cubic_roots_against_reference(oracle, name):
    # same coefficients in; the oracle's portable cbrt / acos / cos / sin differ from CUDA's
    # by an ulp on part of the inputs, so roots agree to 1e-9 relative (the declared TOI
    # tolerance) where they are in [0, 1]; the GPU's reference mode is bit-exact (GPU test)
    d = _load(name)
    got = np.array([oracle.solve_cubic(*c) for c in d["coefs"]])
    ref = d["roots"]
    inside = (ref >= 0) & (ref <= 1)
    rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-12)
    assert np.median(rel[inside]) < 1e-13
    assert (got == ref).mean() > 0.5


TE_CASES = ["te_fold_60_float64", "te_fold_61_float32", "te_fold_70_float32", "te_fold_75_float32",
            "te_fold_75_float64", "te_static_fold"]


@pytest.mark.parametrize("name", TE_CASES)
def test_triangle_edge_oracle_against_reference(oracle, name):
    """Triangle-edge queries (tests/golden/make_te_golden.py).  The candidate queries involve
    no rounding and are equal as multisets.  The crossings take the face normal through
    rsqrt in the reference and through 1 / sqrt in the oracle.  The edge coefficient divides
    a difference of nearly equal dot products, which magnifies that one-ulp difference: the
    coefficients of the common rows agree within 1e4 ulps relative (measured up to about
    2e3 on the folded sheet), and rows differ only where the crossing lies on a triangle edge
    (a barycentric coordinate exactly 0 in exact arithmetic), at most 10 % of them.  The GPU
    path in its default mode calls rsqrt and matches bit for bit (GPU tests)."""
    d = _load(name)
    x, bb, tr = d["x"], d["bboxes"], d["tree"]
    assert _ms(oracle.triangle_edge_candidates(bb, tr, x)) == _ms(d["cand_rows"])
    pairs, masks = oracle.triangle_edge_candidates2(bb, tr, x)
    assert Counter(zip(map(tuple, pairs.tolist()), map(tuple, masks.tolist()))) == \
        Counter(zip(map(tuple, d["cand2_pairs"].tolist()), map(tuple, d["cand2_masks"].tolist())))
    rows, coefs = oracle.triangle_edge_collisions(bb, tr, x)
    got = {tuple(r): c for r, c in zip(rows.tolist(), coefs.tolist())}
    ref = {tuple(r): c for r, c in zip(d["te_rows"].tolist(), d["te_coefs"].tolist())}
    assert len(got) == len(rows) and len(ref) == len(d["te_rows"])
    assert len(set(got) ^ set(ref)) <= 0.1 * len(ref)
    eps = np.finfo(x.dtype).eps
    for k in set(got) & set(ref):
        assert abs(got[k] - ref[k]) <= 1e4 * eps * max(abs(ref[k]), 1e-3)
