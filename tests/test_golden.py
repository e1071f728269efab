"""The CPU oracle against outputs of the reference extension itself.

tests/golden/*.npz were written by tests/golden/make_golden.py, which ran the reference's
own compiled extension (built from its sources by oracle/build_ref.py) on a B200 with
seeded inputs.  The trees fed to it are the oracle's reference-order builds.

Bars:
  * candidate sub-tests (find_mincol_cand), static intersections (find_collisions, fp32
    and fp64, two thresholds) and proximity rows: equal as multisets;
  * impulses from the reference's own collision rows (compute_impulses_from_collisions):
    counters equal, dv / dx within 1e-12 relative (fp64) / 1e-3 relative (fp32);
  * continuous-collision rows: the reference is compiled with nvcc's default fused
    multiply-add contraction, which moves cubic roots of near-degenerate tetrahedra; the
    oracle evaluates the same expressions without contraction, so a small fraction of
    rows differs (bounded below), and every differing row is a near-degenerate case.
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
