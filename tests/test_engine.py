"""The resident multi-mesh engine (include/ccc_engine.h) on the GPU.

Collision rows of every mesh in a batch of uneven meshes equal the oracle's (bit for bit in
the portable math mode) and the reference-format path's; a captured graph replays the
same step for a changed active set; the impulse loop matches the oracle's loop bit for bit
and gives each mesh the same result alone and in a mix.
"""
from collections import Counter

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _meshes(n, seed=0, dtype=np.float64):
    from cccollisions_b200 import workloads as W
    g = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nx, ny = int(g.integers(5, 16)), int(g.integers(5, 16))
        x0, x1, m = W.jittered_fold(100 + i, nx, ny, dtype=dtype)
        out.append((x0, x1, m))
    return out


def _engine(meshes, dtype=torch.float64, **kw):
    from cccollisions_b200.engine import Engine
    cap = sum(x0.shape[0] for x0, _, _ in meshes) + 64
    eng = Engine(tri_capacity=cap, mesh_capacity=max(8, len(meshes) + 2), dtype=dtype, **kw)
    sids = []
    for x0, x1, _ in meshes:
        sid = eng.add_mesh(x0.shape[0])
        eng.upload_soup(sid, x0, x1)
        sids.append(sid)
    return eng, sids


def _ms(rows, times):
    return Counter(zip(map(tuple, np.asarray(rows).tolist()), np.asarray(times, dtype=np.float64).tolist()))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_engine_rows_match_oracle(cuda, oracle, dtype):
    from cccollisions_b200 import _native as N
    meshes = _meshes(12, dtype=dtype)
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    with N.math_library(N.LIB_PORTABLE):
        eng, sids = _engine(meshes, tdt)
        eng.set_active(sids)
        eng.build(sids)
        eng.ccd()
        st = eng.state(sids)
        assert st["status"] == 0
        for sid, (x0, x1, _), n in zip(sids, meshes, st["rows"]):
            rows, times = eng.collisions(sid, int(n))
            bb, tr = oracle.bvh(x0, x1)
            er, et = oracle.ccd(bb, tr, x0, x1)
            assert _ms(rows.cpu().numpy(), times.cpu().numpy()) == _ms(er, et)
        eng.close()


def test_engine_rows_match_reference_format_path(cuda):
    import cccollisions_b200 as C
    meshes = _meshes(10, seed=3)
    eng, sids = _engine(meshes)
    eng.set_active(sids)
    eng.build(sids)
    eng.ccd()
    st = eng.state(sids)
    for sid, (x0, x1, _), n in zip(sids, meshes, st["rows"]):
        X0 = torch.from_numpy(x0[None]).cuda()
        X1 = torch.from_numpy(x1[None]).cuda()
        bb, tr = C.bvh_motion(X0, X1)
        rows, times = C.find_collisions_continuous(bb, tr, X0, X1)
        r = rows[0].cpu().numpy()
        k = int((r[:, 0] >= 0).sum())
        got_r, got_t = eng.collisions(sid, int(n))
        assert _ms(got_r.cpu().numpy(), got_t.cpu().numpy()) == _ms(r[:k], times[0, :k, 0].cpu().numpy())
    eng.close()


def test_graph_replay_follows_the_active_set(cuda):
    meshes = _meshes(9, seed=5)
    eng, sids = _engine(meshes)
    eng.set_active(sids)
    eng.build(sids)
    eng.ccd()
    direct = {}
    st = eng.state(sids)
    for sid, n in zip(sids, st["rows"]):
        r, t = eng.collisions(sid, int(n))
        direct[sid] = _ms(r.cpu().numpy(), t.cpu().numpy())
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        eng.capture(0)
        sub = sids[::2]
        eng.set_active(sub)
        eng.replay(0)
        st2 = eng.state(sub)
        for sid, n in zip(sub, st2["rows"]):
            r, t = eng.collisions(sid, int(n))
            assert _ms(r.cpu().numpy(), t.cpu().numpy()) == direct[sid]
        # meshes outside the active set were not touched by the replay
        assert all(st2["rows"][i] == st["rows"][sids.index(sid)] for i, sid in enumerate(sub))
    s.synchronize()
    eng.close()


@pytest.mark.parametrize("warp", [0, 1])
def test_every_schedule_gives_the_oracle_rows(cuda, oracle, warp):
    """Each candidate schedule of the autotuner, with the traversal run one query per thread
    (k_traverse_q) or 32 queries per warp (k_traverse_w), gives the oracle's rows bit for
    bit; the meshes are uneven, so warps straddle mesh boundaries."""
    from cccollisions_b200 import _native as N
    from cccollisions_b200.engine import Engine
    meshes = _meshes(11, seed=21)
    scheds = [i for i, s in enumerate(Engine.schedules()) if s["warp_traversal"] == warp]
    assert scheds
    with N.math_library(N.LIB_PORTABLE):
        eng, sids = _engine(meshes)
        eng.set_active(sids)
        eng.build(sids)
        expect = {}
        for sid, (x0, x1, _) in zip(sids, meshes):
            bb, tr = oracle.bvh(x0, x1)
            expect[sid] = _ms(*oracle.ccd(bb, tr, x0, x1))
        for i in scheds:
            eng.set_schedule(i)
            eng.ccd()
            st = eng.state(sids)
            assert st["status"] == 0
            for sid, n in zip(sids, st["rows"]):
                r, t = eng.collisions(sid, int(n))
                assert _ms(r.cpu().numpy(), t.cpu().numpy()) == expect[sid], (i, sid)
        eng.close()


def test_autotune_and_cached_choice(cuda):
    meshes = _meshes(6, seed=9)
    eng, sids = _engine(meshes)
    eng.set_active(sids)
    eng.build(sids)
    c1 = eng.autotune()
    c2 = eng.autotune()
    assert c1 == c2 and c1 >= 0
    eng.ccd()
    assert eng.state(sids)["status"] == 0
    eng.close()


def test_slots_are_reused_and_capacity_is_reported(cuda):
    from cccollisions_b200.engine import Engine
    eng = Engine(tri_capacity=1000, vert_capacity=100, mesh_capacity=3)
    a = eng.add_mesh(600)
    assert eng.try_add_mesh(600) is None             # no contiguous room
    b = eng.add_mesh(300, 50)
    assert eng.try_add_mesh(50, 60) is None          # vertices exhausted
    eng.remove_mesh(a)
    c = eng.add_mesh(500)
    assert c == a
    assert eng.free_slots()[0] == 100
    eng.close()


def _loop_meshes(n, seed=0):
    from cccollisions_b200 import workloads as W
    g = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nx, ny = int(g.integers(8, 20)), int(g.integers(8, 20))
        out.append(W.impulse_fold_mesh(200 + i, nx, ny))
    return out


def _loop_engine(meshes):
    from cccollisions_b200.engine import Engine
    F = sum(m[3].shape[0] for m in meshes)
    V = sum(m[0].shape[0] for m in meshes)
    eng = Engine(tri_capacity=F + 64, vert_capacity=V + 64, mesh_capacity=len(meshes) + 2)
    sids = []
    for v0, v1, vel, faces, masses in meshes:
        sid = eng.add_mesh(faces.shape[0], v0.shape[0])
        eng.upload_mesh(sid, v0, v1, vel, faces, masses)
        sids.append(sid)
    return eng, sids


def _run_loop(eng, sids, max_iter=50):
    eng.set_active(sids)
    eng.loop_prepare(sids)
    for _ in range(max_iter):
        eng.loop_step(max_iter)
        st = eng.state(sids)
        if (st["flags"] & 1).all():
            break
    return eng.state(sids)


def test_impulse_loop_matches_oracle_bit_for_bit(cuda, oracle):
    from cccollisions_b200 import _native as N
    meshes = _loop_meshes(5)
    with N.math_library(N.LIB_PORTABLE):
        eng, sids = _loop_engine(meshes)
        st = _run_loop(eng, sids, 20)
        assert st["status"] == 0
        for i, (sid, m) in enumerate(zip(sids, meshes)):
            v0, v1, vel, faces, masses = m
            ev1, evel, it, conv, per = oracle.impulse_loop(v0, v1, vel, faces, masses, max_iter=20)
            assert int(st["iterations"][i]) == it
            assert bool(st["flags"][i] & 2) == conv
            view = eng.view(sid)
            assert np.array_equal(view["verts1"].cpu().numpy(), ev1)
            assert np.array_equal(view["vel"].cpu().numpy(), evel)
        eng.close()


def test_impulse_loop_separates_folds_like_the_oracle(cuda, oracle):
    """Folds whose layers start apart and cross during the step: the loop ends because no pair
    collides any more, after the oracle's number of iterations and with its positions and
    velocities."""
    from cccollisions_b200 import _native as N
    from cccollisions_b200 import workloads as W
    meshes = [W.impulse_fold_mesh(300 + i, 14 + 3 * i, 12 + 2 * i, **W.SEPARATED_FOLD) for i in range(3)]
    with N.math_library(N.LIB_PORTABLE):
        eng, sids = _loop_engine(meshes)
        st = _run_loop(eng, sids)
        assert st["status"] == 0
        for i, (sid, m) in enumerate(zip(sids, meshes)):
            ev1, evel, it, conv, per = oracle.impulse_loop(*m, max_iter=50)
            assert conv and 1 <= it < 50
            assert int(st["iterations"][i]) == it and bool(st["flags"][i] & 2)
            view = eng.view(sid)
            assert np.array_equal(view["verts1"].cpu().numpy(), ev1)
            assert np.array_equal(view["vel"].cpu().numpy(), evel)
        eng.close()


def test_impulse_loop_same_alone_and_in_mix(cuda):
    meshes = _loop_meshes(6, seed=4)
    eng, sids = _loop_engine(meshes)
    _run_loop(eng, sids)
    mix = {sid: eng.view(sid)["verts1"].cpu().numpy().copy() for sid in sids}
    eng.close()
    for k in (0, 3):
        e1, s1 = _loop_engine([meshes[k]])
        _run_loop(e1, s1)
        assert np.array_equal(e1.view(s1[0])["verts1"].cpu().numpy(), mix[sids[k]])
        e1.close()


def test_impulse_loop_graph_replay(cuda):
    meshes = _loop_meshes(3, seed=8)
    eng, sids = _loop_engine(meshes)
    ref = _run_loop(eng, sids, 30)
    out_direct = {sid: eng.view(sid)["verts1"].cpu().numpy().copy() for sid in sids}
    eng.close()
    eng, sids = _loop_engine(meshes)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        eng.set_active(sids)
        eng.loop_prepare(sids)
        eng.capture(1, 30)
        for _ in range(30):
            eng.replay(1)
        st = eng.state(sids)
    assert (st["iterations"] == ref["iterations"]).all()
    for sid in sids:
        assert np.array_equal(eng.view(sid)["verts1"].cpu().numpy(), out_direct[sid])
    eng.close()


def test_engine_edge_cases_match_oracle(cuda, oracle):
    """A two-triangle mesh, a flat sheet in rigid translation far from everything and a
    static mesh (x1 = x0) — both without rows, every root being a dropped linear case — and
    a slot reused by a different mesh."""
    from cccollisions_b200 import _native as N
    from cccollisions_b200 import workloads as W
    two = W.jittered_fold(40, 2, 3)                      # 2 triangles
    far = W.jittered_fold(41, 6, 6, noise=0.0, fold=False)      # flat sheet, rigid translation
    far = (far[0] + 100.0, far[1] + 100.0, far[2])
    fold = W.jittered_fold(42, 9, 9)
    static = (fold[0], fold[0].copy(), fold[2])
    meshes = [two, far, fold, static]
    with N.math_library(N.LIB_PORTABLE):
        eng, sids = _engine(meshes + [W.jittered_fold(43, 12, 12)])
        # replace the last mesh by another of a different size in the freed slots
        eng.remove_mesh(sids[-1])
        other = W.jittered_fold(44, 10, 8)
        sid = eng.add_mesh(other[0].shape[0])
        eng.upload_soup(sid, other[0], other[1])
        meshes, sids = meshes + [other], sids[:-1] + [sid]
        eng.set_active(sids)
        eng.build(sids)
        eng.ccd()
        st = eng.state(sids)
        assert st["status"] == 0
        for sid, (x0, x1, _), n in zip(sids, meshes, st["rows"]):
            rows, times = eng.collisions(sid, int(n))
            bb, tr = oracle.bvh(x0, x1)
            er, et = oracle.ccd(bb, tr, x0, x1)
            assert _ms(rows.cpu().numpy(), times.cpu().numpy()) == _ms(er, et)
        assert st["rows"][1] == 0 and st["rows"][3] == 0
        eng.close()


def test_engine_rejects_misuse(cuda):
    from cccollisions_b200.engine import Engine
    eng = Engine(tri_capacity=256, mesh_capacity=4)
    with pytest.raises(RuntimeError):
        eng.add_mesh(1)                                  # a mesh needs two triangles
    a = eng.add_mesh(20)
    eng.set_active([a])
    with pytest.raises(RuntimeError):
        eng.ccd()                                        # no tree built yet
    with pytest.raises(RuntimeError):
        eng.set_active([a, a])                           # duplicate slot
    with pytest.raises(RuntimeError):
        eng.set_active([3])                              # unused slot
    with pytest.raises(RuntimeError):
        eng.loop_prepare([a])                            # collision-only mesh has no vertices
    eng.close()


def test_engine_full_size_meshes_match_reference_format_path(cuda):
    """Eight meshes of the batched workload at their real sizes (cloth of log-uniform
    1e3..1e5 triangles over a 20,480-triangle sphere): rows and times equal, as multisets,
    to the reference-format path's, in the default math mode."""
    import cccollisions_b200 as C
    from cccollisions_b200 import workloads as W
    meshes = [(x0, x1, None) for x0, x1 in W.batched(8, seed0=2000)]
    eng, sids = _engine(meshes, max_candidates_per_triangle=32)
    eng.set_active(sids)
    eng.build(sids)
    eng.ccd()
    st = eng.state(sids)
    assert st["status"] == 0
    for sid, (x0, x1, _), n in zip(sids, meshes, st["rows"]):
        X0 = torch.from_numpy(x0[None]).cuda()
        X1 = torch.from_numpy(x1[None]).cuda()
        bb, tr = C.bvh_motion(X0, X1)
        rows, times = C.find_collisions_continuous(bb, tr, X0, X1, 32, 16)
        r = rows[0].cpu().numpy()
        k = int((r[:, 0] >= 0).sum())
        got = eng.collisions(sid, int(n))
        assert _ms(got[0].cpu().numpy(), got[1].cpu().numpy()) == _ms(r[:k], times[0, :k, 0].cpu().numpy())
    eng.close()


def test_refit_across_block_ranges_matches_oracle(cuda, oracle):
    """Many small meshes beside larger ones, so that blocks of the block-local refit pass
    straddle mesh boundaries and hand climbs of every size to the second pass; after a
    change of positions (refit only, no rebuild) the rows equal the oracle's for the new
    positions."""
    from cccollisions_b200 import _native as N
    from cccollisions_b200 import workloads as W
    g = np.random.default_rng(9)
    meshes = []
    for i in range(40):
        nx, ny = (int(g.integers(2, 5)), int(g.integers(2, 5))) if i % 5 else (int(g.integers(12, 30)), 14)
        meshes.append(W.jittered_fold(400 + i, nx, ny))
    with N.math_library(N.LIB_PORTABLE):
        eng, sids = _engine(meshes, max_candidates_per_triangle=32)     # about 18 pairs a triangle
        eng.set_active(sids)
        eng.build(sids)
        moved = []
        for sid, (x0, x1, _) in zip(sids, meshes):
            x1b = x0 + 1.3 * (x1 - x0)
            eng.upload_soup(sid, x0, x1b)
            moved.append((x0, x1b))
        eng.ccd()
        st = eng.state(sids)
        assert st["status"] == 0
        for sid, (x0, x1), n in zip(sids, moved, st["rows"]):
            rows, times = eng.collisions(sid, int(n))
            bb, tr = oracle.bvh(x0, x1)
            er, et = oracle.ccd(bb, tr, x0, x1)
            assert _ms(rows.cpu().numpy(), times.cpu().numpy()) == _ms(er, et)
        eng.close()
