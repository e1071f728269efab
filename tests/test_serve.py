"""The served form (continuous batching over the resident engine) on the GPU."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _requests(n, seed=0, lo=8, hi=24, spacing=0.002):
    from cccollisions_b200 import workloads as W
    from cccollisions_b200.serve import Request
    g = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nx, ny = int(g.integers(lo, hi)), int(g.integers(lo, hi))
        v0, v1, vel, f, m = W.impulse_fold_mesh(300 + i, nx, ny)
        out.append(Request(v0, v1, vel, f, m, arrival=i * spacing, rid=i))
    return out


def test_results_are_the_same_alone_and_in_the_mix(cuda):
    from cccollisions_b200.serve import Server
    reqs = _requests(10)
    srv = Server(budget_bytes=256 << 20, mesh_capacity=64)
    stats = srv.run(reqs)
    assert stats["requests"] == 10 and stats["p99_ms"] >= stats["p50_ms"] > 0
    mix = [r.verts1_out.copy() for r in reqs]
    iters = [r.iterations for r in reqs]
    for k in (0, 4, 9):
        alone = _requests(10)[k]
        alone.arrival = 0.0
        srv.run([alone])
        assert alone.iterations == iters[k]
        assert np.array_equal(alone.verts1_out, mix[k])
    srv.close()


def test_results_match_the_oracle_loop(cuda, oracle):
    from cccollisions_b200 import _native as N
    from cccollisions_b200.serve import Server
    reqs = _requests(4, seed=2)
    with N.math_library(N.LIB_PORTABLE):
        srv = Server(budget_bytes=128 << 20, mesh_capacity=16, max_iter=20)
        srv.run(reqs, realtime=False)
        srv.close()
    for r in reqs:
        ev1, _, it, conv, _ = oracle.impulse_loop(r.verts0, r.verts1, r.vel, r.faces, r.masses, max_iter=20)
        assert r.iterations == it and r.converged == conv
        assert np.array_equal(r.verts1_out, ev1)


def test_admission_waits_for_memory(cuda):
    from cccollisions_b200.serve import Server, engine_capacity
    reqs = _requests(6, seed=5, lo=20, hi=22, spacing=0.0)
    biggest = max(r.F for r in reqs)
    # a block with room for about two requests at a time, beside the library's fixed
    # module-data array
    from cccollisions_b200 import _native as N
    fixed = N.lib().ccc_static_scratch_bytes()
    extra = 1 << 16
    while engine_capacity(fixed + extra, mesh_capacity=8, vert_ratio=1.0)[0] < 2 * biggest + 16:
        extra *= 2
    budget = fixed + extra
    srv = Server(budget_bytes=budget, mesh_capacity=8, vert_ratio=1.0)
    tc = engine_capacity(budget, mesh_capacity=8, vert_ratio=1.0)[0]
    assert tc < sum(r.F for r in reqs)               # not everything fits at once
    stats = srv.run(reqs, realtime=False)
    assert stats["requests"] == 6 and all(r.verts1_out is not None for r in reqs)
    admitted = sorted(r.admitted for r in reqs)
    assert admitted[-1] > admitted[0]                # later requests waited for slots
    srv.close()


def test_active_triangle_cap(cuda):
    """Under a backlog, the cap admits requests in waves: the first finish before the last
    are admitted, a request larger than the cap still runs alone, and results are those of
    the uncapped server."""
    from cccollisions_b200.serve import Server
    reqs = _requests(8, seed=7, lo=12, hi=16, spacing=0.0)
    srv = Server(budget_bytes=256 << 20, mesh_capacity=64, max_active_triangles=None)
    srv.run(reqs, realtime=False)
    free_out = [r.verts1_out.copy() for r in reqs]
    srv.close()
    capped = _requests(8, seed=7, lo=12, hi=16, spacing=0.0)
    cap = 2 * max(r.F for r in capped)
    srv = Server(budget_bytes=256 << 20, mesh_capacity=64, max_active_triangles=cap)
    srv.run(capped, realtime=False)
    assert min(r.finished for r in capped) <= max(r.admitted for r in capped)
    for a, b in zip(capped, free_out):
        assert np.array_equal(a.verts1_out, b)
    big = _requests(1, seed=8, lo=20, hi=21)[0]
    small_cap = Server(budget_bytes=256 << 20, mesh_capacity=64, max_active_triangles=big.F // 2)
    small_cap.run([big], realtime=False)
    assert big.verts1_out is not None
    small_cap.close()
    srv.close()
