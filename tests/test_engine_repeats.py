"""Repeated sub-tests in the resident engine's collision step: each tetrahedron that several
triangle pairs of a mesh share is solved once and its rows are written for every pair.

The meshes here hold every case the corner classes must get right, and each is compared
with the oracle, which solves every pair's sub-tests on its own: corners at one start
position that move apart (a cut), +0 and -0 at a shared vertex, coordinates that do not
come back from their displacement (x0 + (x1 - x0) != x1), edges of three triangles, a
vertex of more triangles than a class may hold, and triangles with two equal corners.  The
impulse loop, which solves every pair's sub-tests and tests the exact leaf boxes of the
engine's candidates, runs the same cases against the oracle's loop.
"""
from collections import Counter

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _fold(seed, nx=12, ny=10, noise=0.02, drop=0.05):
    """Indexed jittered fold: verts0, verts1 (V, 3), faces (F, 3)."""
    from cccollisions_b200 import workloads as W
    g = np.random.default_rng(seed)
    v, f = W.grid(nx, ny)
    v[:, 2] = g.normal(0, noise, v.shape[0])
    m = v[:, 0] > 0.5
    v[m, 0] = 1.0 - v[m, 0]
    v[m, 2] += 0.01
    v1 = v.copy()
    v1[:, 2] -= drop
    v1 += g.normal(0, noise, v.shape)
    return v, v1, f


def _cut(v0, v1, f, seed):
    """Some vertices split in two: the same start position, different end positions."""
    g = np.random.default_rng(seed)
    v0, v1, f = v0.copy(), v1.copy(), f.copy()
    for v in g.choice(v0.shape[0], size=max(1, v0.shape[0] // 6), replace=False):
        tris = np.nonzero((f == v).any(axis=1))[0]
        if len(tris) < 2:
            continue
        n = v0.shape[0]
        v0 = np.vstack([v0, v0[v]])
        v1 = np.vstack([v1, v1[v] + np.array([0.0, 0.0, 1e-3])])
        for t in tris[: len(tris) // 2]:
            f[t][f[t] == v] = n
    return v0, v1, f


def _fin(v0, v1, f, seed):
    """Triangles added on existing edges (three triangles an edge), plus a few with two
    equal corners."""
    g = np.random.default_rng(seed)
    v0, v1, f = v0.copy(), v1.copy(), [*f]
    for t in g.choice(len(f), size=max(1, len(f) // 8), replace=False):
        a, b = f[t][0], f[t][1]
        mid0 = 0.5 * (v0[a] + v0[b]) + np.array([0.0, 0.0, 0.02])
        mid1 = 0.5 * (v1[a] + v1[b]) + np.array([0.0, 0.0, -0.02])
        v0 = np.vstack([v0, mid0])
        v1 = np.vstack([v1, mid1])
        f.append(np.array([a, b, v0.shape[0] - 1]))
    for t in g.choice(len(f), size=3, replace=False):
        f.append(np.array([f[t][0], f[t][0], f[t][2]]))
    return v0, v1, np.array(f)


def _fan(v0, v1, f, k=20):
    """A vertex of k thin triangles just above the sheet, moving through it."""
    c = np.argmin(np.abs(v0[:, 0] - 0.25) + np.abs(v0[:, 1] - 0.5))
    p0 = v0[c] + np.array([0.0, 0.0, 0.004])
    p1 = v1[c] + np.array([0.0, 0.0, -0.004])
    ang = np.linspace(0, 2 * np.pi, k, endpoint=False)
    ring = np.stack([0.03 * np.cos(ang), 0.03 * np.sin(ang), np.zeros(k)], axis=1)
    n = v0.shape[0]
    v0 = np.vstack([v0, p0, p0 + ring])
    v1 = np.vstack([v1, p1, p1 + ring])
    tris = [[n, n + 1 + i, n + 1 + (i + 1) % k] for i in range(k)]
    return v0, v1, np.vstack([f, np.array(tris)])


def _soups(v0, v1, f, dtype):
    return v0[f].astype(dtype), v1[f].astype(dtype)


def _signed_zero(x0, seed):
    """-0 in place of +0 at some corners' start coordinates (still one vertex)."""
    g = np.random.default_rng(seed)
    x0 = x0.copy()
    z = np.argwhere(x0 == 0.0)
    pick = z[g.random(len(z)) < 0.5]
    x0[tuple(pick.T)] = -0.0
    return x0


def _cases(dtype):
    base = _fold(7)
    out = {"fold": _soups(*base, dtype)}
    out["cut"] = _soups(*_cut(*base, 1), dtype)
    out["fin"] = _soups(*_fin(*base, 2), dtype)
    out["fan"] = _soups(*_fan(*base), dtype)
    x0, x1 = _soups(*base, dtype)
    out["signed_zero"] = (_signed_zero(x0, 3), x1)
    # moving 3 along x: x0 + (x1 - x0) rounds away from x1 at many coordinates
    out["inexact"] = (x0, x1 + dtype(3.0))
    return out


def _ms(rows, times):
    return Counter(zip(map(tuple, np.asarray(rows).tolist()), np.asarray(times, dtype=np.float64).tolist()))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_shared_sub_tests_give_the_oracle_rows(cuda, oracle, dtype):
    from cccollisions_b200 import _native as N
    from cccollisions_b200.engine import Engine
    cases = _cases(dtype)
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    with N.math_library(N.LIB_PORTABLE):
        eng = Engine(tri_capacity=sum(a.shape[0] for a, _ in cases.values()) + 64,
                     mesh_capacity=len(cases) + 2, dtype=tdt, max_candidates_per_triangle=64,
                     max_collisions_per_triangle=64)
        sids = []
        for x0, x1 in cases.values():
            sid = eng.add_mesh(x0.shape[0])
            eng.upload_soup(sid, x0, x1)
            sids.append(sid)
        eng.set_active(sids)
        eng.build(sids)
        eng.ccd()
        st = eng.state(sids)
        cnt = eng.counters()
        assert st["status"] == 0
        for name, sid, (x0, x1), n in zip(cases, sids, cases.values(), st["rows"]):
            rows, times = eng.collisions(sid, int(n))
            bb, tr = oracle.bvh(x0, x1)
            er, et = oracle.ccd(bb, tr, x0, x1)
            assert len(er) > 0, name
            assert _ms(rows.cpu().numpy(), times.cpu().numpy()) == _ms(er, et), name
        # the repeats were shared: fewer sub-tests solved than there are
        assert 0 < cnt["solved"] < cnt["subtests"]
        eng.close()


def test_classes_stay_within_a_mesh(cuda, oracle):
    """Two copies of one mesh in one batch (every corner of one has a twin at the same
    position in the other): each copy gets the oracle's rows, and both work counters are
    exactly twice those of the mesh alone, so no class spans two meshes."""
    from cccollisions_b200 import _native as N
    from cccollisions_b200.engine import Engine
    x0, x1 = _soups(*_fold(11, 16, 14), np.float64)
    bb, tr = oracle.bvh(x0, x1)
    er, et = oracle.ccd(bb, tr, x0, x1)
    counts = []
    with N.math_library(N.LIB_PORTABLE):
        for copies in (1, 2):
            eng = Engine(tri_capacity=copies * x0.shape[0] + 64, mesh_capacity=4)
            sids = []
            for _ in range(copies):
                sid = eng.add_mesh(x0.shape[0])
                eng.upload_soup(sid, x0, x1)
                sids.append(sid)
            eng.set_active(sids)
            eng.build(sids)
            eng.ccd()
            st = eng.state(sids)
            assert st["status"] == 0
            for sid, n in zip(sids, st["rows"]):
                rows, times = eng.collisions(sid, int(n))
                assert _ms(rows.cpu().numpy(), times.cpu().numpy()) == _ms(er, et)
            counts.append(eng.counters())
            eng.close()
    one, two = counts
    assert 0 < one["solved"] < one["subtests"]
    assert two["subtests"] == 2 * one["subtests"] and two["solved"] == 2 * one["solved"]


def _loop_cases():
    from cccollisions_b200 import workloads as W
    v0, v1, vel, f, m = W.impulse_fold_mesh(21, 14, 12)
    out = [(v0, v1, vel, f, m)]
    a0, a1, af = _cut(v0, v1, f.astype(np.int64), 4)
    out.append((a0, a1, a1 - a0, af.astype(np.int32), np.ones((af.shape[0], 3))))
    b0, b1, bf = _fin(v0, v1, f.astype(np.int64), 5)
    out.append((b0, b1, b1 - b0, bf.astype(np.int32), np.ones((bf.shape[0], 3))))
    c0, c1, cf = _fan(v0, v1, f.astype(np.int64))
    out.append((c0, c1, c1 - c0, cf.astype(np.int32), np.ones((cf.shape[0], 3))))
    # a second vertex at a -0 start coordinate where another is at +0
    z = np.argwhere(v0[:, 0] == 0.0)[:, 0]
    d0, d1, df = v0.copy(), v1.copy(), f.astype(np.int64).copy()
    for v in z[::2]:
        tris = np.nonzero((df == v).any(axis=1))[0]
        if len(tris) < 2:
            continue
        n = d0.shape[0]
        d0 = np.vstack([d0, d0[v] * np.array([-1.0, 1.0, 1.0])])
        d1 = np.vstack([d1, d1[v]])
        for t in tris[:1]:
            df[t][df[t] == v] = n
    out.append((d0, d1, d1 - d0, df.astype(np.int32), np.ones((df.shape[0], 3))))
    return out


def test_edge_case_meshes_in_the_impulse_loop_match_oracle(cuda, oracle):
    from cccollisions_b200 import _native as N
    from cccollisions_b200.engine import Engine
    meshes = _loop_cases()
    with N.math_library(N.LIB_PORTABLE):
        F = sum(m[3].shape[0] for m in meshes)
        V = sum(m[0].shape[0] for m in meshes)
        eng = Engine(tri_capacity=F + 64, vert_capacity=V + 64, mesh_capacity=len(meshes) + 2,
                     max_candidates_per_triangle=64, max_collisions_per_triangle=64)
        sids = []
        for v0, v1, vel, faces, masses in meshes:
            sid = eng.add_mesh(faces.shape[0], v0.shape[0])
            eng.upload_mesh(sid, v0, v1, vel, faces, masses)
            sids.append(sid)
        eng.set_active(sids)
        eng.loop_prepare(sids)
        for _ in range(12):
            eng.loop_step(12)
            if (eng.state(sids)["flags"] & 1).all():
                break
        st = eng.state(sids)
        # (triangles with two equal corners give non-finite impulses, which the engine and
        # the oracle both leave out; the engine reports them with status bit 16)
        assert st["status"] & ~16 == 0
        for i, (sid, (v0, v1, vel, faces, masses)) in enumerate(zip(sids, meshes)):
            ev1, evel, it, conv, per = oracle.impulse_loop(v0, v1, vel, faces, masses, max_iter=12)
            assert int(st["iterations"][i]) == it, i
            view = eng.view(sid)
            assert np.array_equal(view["verts1"].cpu().numpy(), ev1), i
            assert np.array_equal(view["vel"].cpu().numpy(), evel), i
        eng.close()
