"""Known-answer and brute-force pins of the CPU oracle (no GPU needed).

The reference ships no tests or golden vectors, so the oracle's restatement is pinned by
hand-derived values: Morton interleaving, the Karras topology over all-equal keys, the
reference's unbounded-scene-box quirk, each branch of the cubic solver, analytic times of
impact, the separating-axis test and proximity on known configurations, CAMPARY products
against exact rational arithmetic, and O(F^2) brute force for candidate pairs.
"""
import math
from fractions import Fraction

import numpy as np
import pytest

from conftest import random_mesh_soup


# ----------------------------------------------------------------------------- primitives

def test_morton_known_values(oracle):
    # expandBits interleaves x*4 + y*2 + z over 10 bits per axis (bvh.cu:29-62)
    assert oracle.morton(0.0, 0.0, 0.0) == 0
    assert oracle.morton(1.0, 1.0, 1.0) == (1 << 30) - 1        # clamps to 1023 on each axis
    # x = 1/1024 -> cell 1 -> bit 2
    assert oracle.morton(1.0 / 1024, 0.0, 0.0) == 4
    assert oracle.morton(0.0, 1.0 / 1024, 0.0) == 2
    assert oracle.morton(0.0, 0.0, 1.0 / 1024) == 1
    assert oracle.morton(2.0 / 1024, 0.0, 0.0) == 32
    # negative and NaN clamp to 0 (fmax semantics)
    assert oracle.morton(-5.0, float("nan"), 0.0) == 0
    assert oracle.morton(0.5, 0.5, 0.5, single=True) == oracle.morton(0.5, 0.5, 0.5)


def test_karras_identity_topology_n8(oracle):
    # all-equal keys with ids 0..7: delta(i, j) = 32 + clz(i ^ j), i.e. the radix tree of
    # the indices
    tri = np.zeros((8, 3, 3), dtype=np.float64)
    tri[:, :, 0] = np.arange(8)[:, None] + np.array([0.0, 0.5, 0.0])
    tri[:, 2, 1] = 1.0
    bb, tr = oracle.bvh(tri)
    expect = np.array([[-1, 3, 4, -1], [3, 7, 8, -1], [3, 9, 10, -1], [0, 1, 2, -1], [0, 5, 6, -1],
                       [4, 11, 12, -1], [4, 13, 14, -1]])
    assert (tr[:7] == expect).all()
    assert (tr[7:, 0] == [1, 1, 2, 2, 5, 5, 6, 6]).all()
    assert (tr[7:, 1:3] == -1).all()
    assert (tr[7:, 3] == np.arange(8)).all()
    # internal boxes are unions of their children
    for k in range(7):
        l, r = tr[k, 1], tr[k, 2]
        assert (bb[k, :3] == np.minimum(bb[l, :3], bb[r, :3])).all()
        assert (bb[k, 3:] == np.maximum(bb[l, 3:], bb[r, 3:])).all()


def test_reference_scene_box_gives_zero_codes(oracle):
    # AABB() is (-MAX, +MAX) (aabb.cu:25-34) and seeds the scene-box reduction
    # (build_bvh.cu:243), so every normalised centroid is 0 and every code is 0
    x0, x1, _ = random_mesh_soup(3)
    _, _, codes = oracle.bvh(x0, return_codes=True)
    assert (codes == 0).all()
    _, _, codes_m = oracle.bvh(x0, x1, return_codes=True)
    assert (codes_m == 0).all()
    _, _, codes32 = oracle.bvh(x0.astype(np.float32), return_codes=True)
    assert (codes32 == 0).all()
    # a bounded scene box gives real codes
    _, _, codes_s = oracle.bvh(x0, spatial=True, return_codes=True)
    assert len(np.unique(codes_s)) > 10


def _ulp(x):
    return math.ulp(x)


def test_cbrt_within_one_ulp(oracle):
    g = np.random.default_rng(5)
    xs = list(np.exp(g.uniform(-700, 700, 3000))) + [1e-310, 5e-324, 8.0, 27.0, 1.0, 0.001, 1e-16]
    for x in xs:
        y = oracle.cbrt(float(x))
        if x == 8.0:
            assert y == 2.0
        if x == 27.0:
            assert y == 3.0
        fx = Fraction(float(x))
        # correctly rounded c satisfies (c - ulp/2)^3 <= x <= (c + ulp/2)^3; accept 1 ulp
        u = Fraction(_ulp(y))
        lo = Fraction(y) - u
        hi = Fraction(y) + u
        assert lo ** 3 <= fx <= hi ** 3, x
        assert oracle.cbrt(-float(x)) == -y


def test_trig_within_two_ulp(oracle):
    g = np.random.default_rng(7)
    for x in g.uniform(-1.0, 1.0, 4000):
        a = oracle.acos(float(x))
        assert abs(a - math.acos(x)) <= 2 * _ulp(math.acos(x)), x
    for x in list(g.uniform(0.0, math.pi / 3, 4000)) + [0.0, 1e-300, 1.0471975511965976]:
        c, s = oracle.cos(float(x)), oracle.sin(float(x))
        assert abs(c - math.cos(x)) <= 2 * _ulp(math.cos(x)), x
        assert abs(s - math.sin(x)) <= 2 * max(_ulp(math.sin(x)), 5e-324), x
    assert oracle.acos(1.0) == 0.0
    assert abs(oracle.acos(-1.0) - math.pi) <= _ulp(math.pi)
    assert math.isnan(oracle.acos(1.5))


def test_certmul_matches_exact_products(oracle):
    # certifiedMul<1,1,2> gives an exact 2-term expansion of a double product
    # (multiplication.h:132-184); <2,1,2> rounds a 3-term exact product to 2 terms
    g = np.random.default_rng(11)
    for _ in range(3000):
        b = float(g.uniform(-1, 1) * 10.0 ** g.integers(-12, 3))
        r = oracle.certmul(b, b)
        assert Fraction(r[0]) + Fraction(r[1]) == Fraction(b) * Fraction(b)
        assert r[0] == b * b
        c = oracle.certmul(r, b)
        exact = Fraction(b) ** 3
        approx = Fraction(c[0]) + Fraction(c[1])
        if exact != 0:
            assert abs(approx - exact) <= abs(exact) * Fraction(1, 2 ** 100)
        # leading term within one ulp of the correctly rounded cube
        assert abs(c[0] - float(exact)) <= _ulp(float(exact)) if exact != 0 else c[0] == 0


# ----------------------------------------------------------------------------- cubic solver

def test_solve_cubic_branches(oracle):
    # linear (a == b == 0): the reference never stores the root
    assert (oracle.solve_cubic(0.0, 0.0, 1.0, -0.5) == -1).all()
    # quadratic (|a| < 1e-16): (t - 0.25)(t - 0.75) = t^2 - t + 0.1875
    r = oracle.solve_cubic(1e-18, 1.0, -1.0, 0.1875)
    assert sorted(r[:2]) == pytest.approx([0.25, 0.75], abs=1e-15) and r[2] == -1
    # three real roots: (t - 0.1)(t - 0.5)(t - 0.9)
    a, b, c, d = 1.0, -1.5, 0.59, -0.045
    r = oracle.solve_cubic(a, b, c, d)
    assert sorted(r) == pytest.approx([0.1, 0.5, 0.9], abs=1e-12)
    # one real root (h > 0): (t - 0.3)(t^2 + 1)
    r = oracle.solve_cubic(1.0, -0.3, 1.0, -0.3)
    assert r[0] == pytest.approx(0.3, abs=1e-14) and (r[1:] == -1).all()
    # roots outside [-eps, 1 + eps] are dropped: (t - 2)(t - 3)(t - 4)
    assert (oracle.solve_cubic(1.0, -9.0, 26.0, -24.0) == -1).all()
    # triple root (f == g == h == 0): (t - 0.5)^3 -> d / a = -0.125, root from float cbrt
    r = oracle.solve_cubic(1.0, -1.5, 0.75, -0.125)
    assert r[0] == pytest.approx(0.5, abs=1e-6)


def _tet(v, dv):
    return np.concatenate([np.asarray(v, float).ravel(), np.asarray(dv, float).ravel()])


def test_cubic_coeffs_vertex_face_analytic(oracle):
    # face z = 0 (points 0..2), vertex at z = 1 moving -2 per step: det linear in t with
    # root 0.5; the cubic's coefficients are those of det(v - v3 + t (dv - dv3))
    v = [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0.2, 0.2, 1.0]]
    dv = [[0, 0, 0], [0, 0, 0], [0, 0, 0], [0, 0, -2.0]]
    c = oracle.cubic_coeffs(_tet(v, dv))
    m = lambda t: np.array(v[:3]) - np.array(v[3]) + t * (np.array(dv[:3]) - np.array(dv[3]))
    for t in (0.0, 0.3, 1.0, -2.0):
        assert c[0] * t ** 3 + c[1] * t ** 2 + c[2] * t + c[3] == pytest.approx(np.linalg.det(m(t)), abs=1e-12)


# ----------------------------------------------------------------------------- CCD known answers

def _soup(*tris):
    return np.ascontiguousarray(np.array(tris, dtype=np.float64))


def test_ccd_vertex_face_time_of_impact(oracle):
    # face of triangle 0 stays in z = 0 but grows (v1, v2 move outward in the plane);
    # triangle 1's vertex 0 goes from z = 0.4 to z = -0.6: det(t) ~ (0.4 - t)(1 + t/2)^2,
    # a genuine cubic with the impact at t = 0.4 (inside the face)
    t0 = [[0, 0, 0], [1, 0, 0], [0, 1, 0]]
    t0n = [[0, 0, 0], [1.5, 0, 0], [0, 1.5, 0]]
    t1 = [[0.2, 0.2, 0.4], [2.0, 2.0, 0.4], [2.0, 3.0, 0.4]]
    t1n = [[0.2, 0.2, -0.6], [2.0, 2.0, 0.4], [2.0, 3.0, 0.4]]
    x0 = _soup(t0, t1)
    x1 = _soup(t0n, t1n)
    bb, tr = oracle.bvh(x0, x1)
    rows, times = oracle.ccd(bb, tr, x0, x1)
    vf = [t for r, t in zip(rows.tolist(), times.tolist()) if tuple(r) == (0, 1, 9)]
    assert len(vf) == 1 and abs(vf[0] - 0.4) < 1e-12


def test_ccd_rigid_translation_is_dropped(oracle):
    # a static face and a vertex translating through it make the coplanarity polynomial
    # linear (a == b == 0); the reference computes -d/c into a local and never stores it
    # (collisions_continuous.cu:532-536), so no row is reported
    t0 = [[0, 0, 0], [1, 0, 0], [0, 1, 0]]
    t1 = [[0.2, 0.2, 0.4], [2.0, 2.0, 0.4], [2.0, 3.0, 0.4]]
    t1n = [[0.2, 0.2, -0.6], [2.0, 2.0, -0.6], [2.0, 3.0, -0.6]]
    x0 = _soup(t0, t1)
    x1 = _soup(t0, t1n)
    bb, tr = oracle.bvh(x0, x1)
    rows, _ = oracle.ccd(bb, tr, x0, x1)
    assert len(rows) == 0
    # the sub-test itself is a candidate
    assert (0, 1, 9) in set(map(tuple, oracle.mincol_cand(bb, tr, x0, x1).tolist()))


def test_ccd_edge_edge_crossing(oracle):
    # edge (0,1) of triangle 0 along x at z = 0 (static); edge (0,1) of triangle 1 along y
    # at z = 0.2 moving down 0.4 while stretching -> crossing at t = 0.5 at both midpoints
    t0 = [[-1, 0, 0], [1, 0, 0], [0, -3, -5]]
    t1 = [[0, -1, 0.2], [0, 1, 0.2], [3, 0, 5]]
    t1n = [[0, -1.5, -0.2], [0, 1.5, -0.2], [3, 0, 5]]
    x0 = _soup(t0, t1)
    x1 = _soup(t0, t1n)
    bb, tr = oracle.bvh(x0, x1)
    rows, times = oracle.ccd(bb, tr, x0, x1)
    ee = [t for r, t in zip(rows.tolist(), times.tolist()) if tuple(r) == (0, 1, 0)]
    assert len(ee) == 1 and abs(ee[0] - 0.5) < 1e-12


def test_ccd_shared_vertex_rejected(oracle):
    # triangles sharing a vertex (exact coordinates) never produce sub-tests
    t0 = [[0, 0, 0], [1, 0, 0], [0, 1, 0]]
    t1 = [[0, 0, 0], [0.3, 0.3, 0.5], [0.3, -0.2, -0.5]]
    x0 = _soup(t0, t1)
    x1 = x0.copy()
    x1[1, 1:, 2] *= -1
    bb, tr = oracle.bvh(x0, x1)
    rows, _ = oracle.ccd(bb, tr, x0, x1)
    assert len(rows) == 0
    assert len(oracle.mincol_cand(bb, tr, x0, x1)) == 0


def test_root_filter_known_answers(oracle):
    """filterCollisions / is_inside (collisions_continuous.cu:615-684) on static tetrahedra
    (zero displacement, so the points at the root are the points themselves).  Edge-edge:
    the closest-point parameters s, p of the two lines must lie in [0, 1]; vertex-face: the
    barycentrics of the vertex's projection on the face's plane must lie in [0, 1].  A NaN
    parameter fails no comparison and passes."""
    dv = [[0, 0, 0]] * 4
    # edge-edge (k < 9): edge (p0, p1) against edge (p2, p3)
    crossing = [[0, 0, 0], [1, 0, 0], [0.5, -0.5, 0], [0.5, 0.5, 0]]
    assert oracle.ccd_filter(_tet(crossing, dv), 0, 0.5)
    beyond = [[0, 0, 0], [1, 0, 0], [1.5, -0.5, 0], [1.5, 0.5, 0]]          # s = 1.5
    assert not oracle.ccd_filter(_tet(beyond, dv), 0, 0.5)
    parallel = [[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0]]                # |da x db| = 0: NaN
    assert oracle.ccd_filter(_tet(parallel, dv), 4, 0.5)
    # vertex-face: face (p0, p1, p2) and vertex p3 for k = 9..11
    face = [[0, 0, 0], [1, 0, 0], [0, 1, 0]]
    assert oracle.ccd_filter(_tet(face + [[0.2, 0.2, 0.3]], dv), 9, 0.5)    # projection inside
    assert not oracle.ccd_filter(_tet(face + [[0.8, 0.8, 0.0]], dv), 10, 0.5)
    point = [[0.3, 0.3, 0.0]] * 3                                          # degenerate face: NaN
    assert oracle.ccd_filter(_tet(point + [[5.0, 5.0, 5.0]], dv), 11, 0.5)
    # k = 12..14: vertex p0 and face (p1, p2, p3)
    assert oracle.ccd_filter(_tet([[0.2, 0.2, -0.3]] + face, dv), 12, 0.5)
    assert not oracle.ccd_filter(_tet([[-0.1, 0.5, 0.0]] + face, dv), 13, 0.5)
    # roots below -1e-16 are rejected before any test
    assert not oracle.ccd_filter(_tet(crossing, dv), 0, -0.5)


def test_contact_kinematics_known_answers(oracle):
    """compute_coeficients_and_directions (collisions_impulses.cu:162-543): the normal of
    the tetrahedron's first two edges at the root, turned from side 0 to side 1 (by the
    points at the start), the normal velocity, and the mass pair mixed by the contact
    parameters.  Output: (normal xyz, normal velocity, mass 0, mass 1)."""
    q = [1.0, 2.0, 3.0, 4.0]
    face = [[0, 0, 0], [1, 0, 0], [0, 1, 0]]
    still = [[0, 0, 0]] * 3
    # vertex above the face falling onto it (k = 9): barycentrics (0.6, 0.2, 0.2) of the
    # face's points, face mass 3 * 0.2 + 1 * 0.6 + 2 * 0.2
    o = oracle.contact(_tet(face + [[0.2, 0.2, 0.1]], still + [[0, 0, -0.2]]), 9, 0.5, q)
    np.testing.assert_allclose(o, [0, 0, 1, -0.2, 1.6, 4.0], atol=1e-12)
    # vertex below the face rising onto it (k = 12: vertex first); the normal comes out
    # turned back towards the face's side and the masses swap sides
    o = oracle.contact(_tet([[0.2, 0.2, -0.1]] + face, [[0, 0, 0.2]] + still), 12, 0.5, q)
    np.testing.assert_allclose(o, [0, 0, 1, -0.2, 1.0, 4 * 0.2 + 2 * 0.6 + 3 * 0.2], atol=1e-12)
    # parallel edges (|da x db|^2 < 1e-15): s = t = 0.5, masses (q0 + q1) / 2, (q2 + q3) / 2
    ee = [[0, 0, 0], [1, 0, 0], [0, 0, 0.1], [1, 0, 0.1]]
    o = oracle.contact(_tet(ee, [[0, 0, 0], [0, 0, 0], [0, -0.1, 0], [0, -0.1, 0]]), 0, 0.0, q)
    np.testing.assert_allclose(o, [0, -1, 0, 0.1, 1.5, 3.5], atol=1e-12)


# ----------------------------------------------------------------------------- static SAT

def test_sat_known_configurations(oracle):
    a = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], dtype=np.float64)
    pierce = np.array([[0.2, 0.2, -1], [0.3, 0.2, 1], [0.2, 0.3, 1]], dtype=np.float64)
    above = pierce + [0, 0, 3.0]
    assert oracle.sat(a, pierce)
    assert not oracle.sat(a, above)
    assert oracle.sat(a, above, threshold=2.5)     # the threshold widens every interval
    # coplanar overlapping and coplanar disjoint
    assert oracle.sat(a, a + [0.1, 0.1, 0])
    assert not oracle.sat(a, a + [2.0, 0, 0])
    assert oracle.sat(a.astype(np.float32), pierce.astype(np.float32))


# ----------------------------------------------------------------------------- proximity

@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_proximity_parallel_triangles(oracle, dtype):
    """Triangle 1 lies h above triangle 0, parallel and inside its outline
    (proximity_static.cu:11-508).  Within the threshold, at distance h:
    * faces against vertices (k = 9, 10, 11): every vertex of triangle 1 projects inside
      triangle 0; triangle 0's vertices lie 0.2 outside triangle 1's box, so k = 12..14
      fail the sub-box test;
    * no edge pair (k = 3 * e0 + e1, edges 01, 02, 12): triangle 0's edge 12 (x + y = 1)
      passes over the lines of edges 01 and 02 of triangle 1 beyond their ends (t = 1.5,
      k = 6, 7); the two edges 12 are parallel (NaN s and t, the point-segment fallback)
      and sqrt(0.02 + h^2) = 0.15 apart, beyond the threshold (k = 8); the other edge
      pairs are 0.2 apart in x or y and fail the sub-box test."""
    h, th = 0.05, 0.1
    x = np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]],
                  [[0.2, 0.2, h], [0.6, 0.2, h], [0.2, 0.6, h]]], dtype=dtype)
    bb, tr = oracle.bvh(x)
    rows, dist = oracle.proximity(bb, tr, x, th)
    got = sorted(map(tuple, rows.tolist()))
    assert got == [(0, 1, k) for k in (9, 10, 11)]
    np.testing.assert_allclose(dist, h, rtol=1e-6)
    # below the height nothing is close enough; a threshold of 0.2 adds the parallel edges
    assert len(oracle.proximity(bb, tr, x, 0.04)[0]) == 0
    wide, wdist = oracle.proximity(bb, tr, x, 0.2)
    assert (0, 1, 8) in set(map(tuple, wide.tolist()))
    np.testing.assert_allclose(wdist[wide[:, 2] == 8], np.sqrt(0.02 + h * h), rtol=1e-6)


# ----------------------------------------------------------------------------- brute force

def _brute_pairs(bb, tr, th=0.0):
    n = (bb.shape[0] + 1) // 2
    lo, hi, ids = bb[n - 1:, :3], bb[n - 1:, 3:], tr[n - 1:, 3]
    out = set()
    for p in range(n):
        ok = np.all((lo[p] <= hi + th) & (hi[p] >= lo - th), axis=1)
        for q in np.nonzero(ok)[0]:
            if q > p:
                out.add((min(ids[p], ids[q]), max(ids[p], ids[q])))
    return out


@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_candidates_equal_brute_force(oracle, seed, dtype):
    x0, x1, _ = random_mesh_soup(seed, dtype=dtype)
    for motion in (False, True):
        bb, tr = oracle.bvh(x0, x1 if motion else None)
        for th in (0.0, 0.01):
            c = oracle.candidates(bb, tr, threshold=th)
            assert len(c) == len(set(map(tuple, c.tolist())))
            assert set(map(tuple, c.tolist())) == _brute_pairs(bb, tr, dtype(th))
    # the spatial (Morton) build gives the same candidate set
    bbs, trs = oracle.bvh(x0, x1, spatial=True)
    bbr, trr = oracle.bvh(x0, x1)
    assert set(map(tuple, oracle.candidates(bbs, trs).tolist())) == set(map(tuple, oracle.candidates(bbr, trr).tolist()))


def test_partial_mask_semantics(oracle):
    x0, x1, _ = random_mesh_soup(4)
    bb, tr = oracle.bvh(x0, x1)
    n = x0.shape[0]
    full = set(map(tuple, oracle.candidates(bb, tr).tolist()))
    allm = np.ones(n, dtype=np.uint8)
    c = oracle.candidates(bb, tr, mask=allm)
    # all triangles checked: each overlapping pair once (query id < other id)
    assert sorted(map(tuple, c.tolist())) == sorted(full)
    none = np.zeros(n, dtype=np.uint8)
    assert len(oracle.candidates(bb, tr, mask=none)) == 0
    g = np.random.default_rng(0)
    m = (g.random(n) < 0.3).astype(np.uint8)
    cm = oracle.candidates(bb, tr, mask=m)
    # a pair appears iff one of its triangles is checked; pairs with both checked once,
    # pairs with one checked once (identity leaf order: position == id)
    expect = sorted(p for p in full if m[p[0]] or m[p[1]])
    assert sorted(map(tuple, cm.tolist())) == expect


def test_ccd_multithreaded_equals_single(oracle):
    x0, x1, _ = random_mesh_soup(6, nx=12, ny=12)
    bb, tr = oracle.bvh(x0, x1)
    r1, t1 = oracle.ccd(bb, tr, x0, x1, nthreads=1)
    r4, t4 = oracle.ccd(bb, tr, x0, x1, nthreads=4)
    assert oracle.row_multiset(r1, t1) == oracle.row_multiset(r4, t4)
    assert len(r1) > 0


def test_impulses_from_rows_match_full(oracle):
    x0, x1, m = random_mesh_soup(8)
    bb, tr = oracle.bvh(x0, x1)
    rows, times = oracle.ccd(bb, tr, x0, x1)
    dv, dx, cnt, nc = oracle.impulses(bb, tr, x0, x1, m)
    dv2, dx2, cnt2 = oracle.impulses_from_rows(x0, x1, m, rows, times)
    assert nc == len(rows) > 0
    assert (cnt == cnt2).all()
    assert np.allclose(dv, dv2, rtol=1e-12, atol=1e-15)
    assert np.allclose(dx, dx2, rtol=1e-12, atol=1e-15)
    # every contact touches exactly four corners
    assert cnt.sum() == 4 * nc


@pytest.mark.parametrize("family", [0, 1, 2, 3])
def test_double_double_short_paths_match_the_bin_algorithm(oracle, family):
    """The short paths of certifiedMul<1,1,2> and of the leading term of certifiedMul<2,1,2>
    (TwoProd and a compensated sum away from ties) give the bin algorithm's bits: random
    significands, 1..30-bit significands (exact and tied products), neighbours of powers of
    two, and zeros / subnormals / huge / non-finite operands."""
    bad, fast = oracle.ddmul_check(4_000_000, 77 + family, family)
    assert bad == 0
    assert fast > (3_000_000 if family < 3 else 1_000_000)
