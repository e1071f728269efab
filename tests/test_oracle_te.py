"""Known-answer and brute-force pins of the oracle's triangle-edge helpers (no GPU needed).

find_triangle_edge_collisions / _candidates / _candidates2 (collisions_static.cu:345-942,
icontour.cu:11-281): intersecting candidate pairs, then six edge sub-tests per pair
(cid 0..2: edge (v0v1, v1v2, v2v0)[cid] of the first triangle against the second,
cid 3..5 the other way round).
"""
import numpy as np
import pytest

from conftest import random_mesh_soup

FACE = [(0.0, 0.0, 0.0), (1.0, 0.0, 0.0), (0.0, 1.0, 0.0)]


def _pair(dtype):
    # triangle 1 stands in the plane x = 0.25 and is crossed by edge v1-v2 of triangle 0 at
    # t = 0.75; its own edge v0-v1 pierces triangle 0 at t = 0.5
    b = [(0.25, 0.25, -1.0), (0.25, 0.25, 1.0), (0.25, 2.0, 0.0)]
    return np.array([FACE, b], dtype=dtype)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_edge_crossings_known_answer(oracle, dtype):
    tri = _pair(dtype)
    bb, tr = oracle.bvh(tri)
    rows, coefs = oracle.triangle_edge_collisions(bb, tr, tri)
    got = sorted((tuple(r), float(c)) for r, c in zip(rows.tolist(), coefs.tolist()))
    assert got == [((0, 1, 1, -1), 0.75), ((0, 1, 3, -1), 0.5)]
    assert coefs.dtype == dtype


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_shared_vertex_pair_known_answer(oracle, dtype):
    # the pair shares corner 0: it is left out of the crossings (no shared vertex allowed) and
    # kept by the candidate queries (one allowed); edge 0 of triangle 0 starts at the shared
    # corner (loop node), edges ending there are skipped, the rest pass the box test
    tri = np.array([FACE, [(0.0, 0.0, 0.0), (-1.0, 0.0, 0.5), (0.0, -1.0, 0.5)]], dtype=dtype)
    bb, tr = oracle.bvh(tri)
    rows, coefs = oracle.triangle_edge_collisions(bb, tr, tri)
    assert len(rows) == 0
    cand = oracle.triangle_edge_candidates(bb, tr, tri)
    assert sorted(map(tuple, cand.tolist())) == [(0, 1, 0, 0), (0, 1, 1, -1), (0, 1, 4, -1)]
    pairs, masks = oracle.triangle_edge_candidates2(bb, tr, tri)
    assert pairs.tolist() == [[0, 1]]
    assert masks.tolist() == [[(1 << 0) | (1 << 1) | (1 << 4), 1 << 0]]


def test_edge_neighbours_are_left_out(oracle):
    # two triangles sharing an edge (two vertices) are no candidates for any of the queries
    tri = np.array([FACE, [(1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (1.0, 1.0, 0.3)]], dtype=np.float64)
    bb, tr = oracle.bvh(tri)
    assert len(oracle.triangle_edge_collisions(bb, tr, tri)[0]) == 0
    assert len(oracle.triangle_edge_candidates(bb, tr, tri)) == 0
    assert len(oracle.triangle_edge_candidates2(bb, tr, tri)[0]) == 0


def _np_crossing(face, p0, p1):
    """Edge / triangle crossing in plain float64 (no fused products): (hit, t, margin)."""
    e1, e2 = face[1] - face[0], face[2] - face[0]
    n = np.cross(e1, e2)
    n = n / np.sqrt(n @ n)
    d = p1 - p0
    en = d @ n
    if en == 0:
        return False, 0.0, abs(en)
    t = (n @ face[0] - n @ p0) / en
    x = p0 + d * t
    ep = x - face[0]
    d00, d01, d11, d20, d21 = e1 @ e1, e1 @ e2, e2 @ e2, ep @ e1, ep @ e2
    den = d00 * d11 - d01 * d01
    v = (d11 * d20 - d01 * d21) / den
    w = (d00 * d21 - d01 * d20) / den
    u = 1.0 - v - w
    margin = min(abs(t), abs(t - 1), abs(u), abs(v), abs(w))
    return (0 <= t <= 1 and den >= 1e-15 and u >= 0 and v >= 0 and w >= 0), t, margin


def test_crossings_against_brute_force(oracle):
    """All pairs (O(F^2)) through the separating-axis test, a vertex-sharing check and a
    float64 restatement of the crossing; rows may differ only within 1e-9 of a boundary."""
    x, _, _ = random_mesh_soup(5, nx=9, ny=8)
    F = x.shape[0]
    bb, tr = oracle.bvh(x)
    rows, coefs = oracle.triangle_edge_collisions(bb, tr, x)
    got = {tuple(r): c for r, c in zip(rows.tolist(), coefs.tolist())}
    assert len(got) == len(rows) and len(rows) > 0
    expect, near = {}, set()
    for i in range(F):
        for j in range(i + 1, F):
            shared = sum(any((x[i, a] == x[j, b]).all() for b in range(3)) for a in range(3))
            if shared or not oracle.sat(x[i], x[j]):
                continue
            for cid in range(6):
                t1, face = (x[i], x[j]) if cid < 3 else (x[j], x[i])
                e = cid % 3
                hit, t, margin = _np_crossing(face, t1[e], t1[(e + 1) % 3])
                key = (i, j, cid, -1)
                if margin < 1e-9:
                    near.add(key)
                if hit:
                    expect[key] = t
    assert set(got) ^ set(expect) <= near
    for k in set(got) & set(expect):
        assert abs(got[k] - expect[k]) <= 1e-12 * max(1.0, abs(expect[k]))


def test_candidates2_lists_the_candidate_pairs(oracle):
    """candidates2 holds the pairs of candidates, and its masks match the candidate rows."""
    x, _, _ = random_mesh_soup(6, nx=10, ny=9)
    bb, tr = oracle.bvh(x)
    cand = oracle.triangle_edge_candidates(bb, tr, x)
    pairs, masks = oracle.triangle_edge_candidates2(bb, tr, x)
    assert len(pairs) > 0 and len(cand) > 0
    mx, my = {}, {}
    for i, j, cid, flag in cand.tolist():
        mx[(i, j)] = mx.get((i, j), 0) | (1 << cid)
        if flag == 0:
            my[(i, j)] = my.get((i, j), 0) | (1 << cid)
    for (i, j), (a, b) in zip(pairs.tolist(), masks.tolist()):
        assert a == mx.get((i, j), 0) and b == my.get((i, j), 0)
    assert set(mx) <= set(map(tuple, pairs.tolist()))
