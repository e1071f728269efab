"""The no-allocation continuous-collision entry point (ccc_find_collisions_continuous_static).

It exists for callers that cannot allocate device memory, such as a plugin running inside
a host framework that owns all of the GPU's memory through its own pool, or a real-time
step loop that forbids allocations; its scratch is a fixed device array inside the
library.  Checked through the C ABI against the workspace-taking entry point on the same
inputs, twice in a row (the array keeps the previous call's contents, so the second call
shows that everything that must start at zero is cleared).  This file is collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOI_RTOL = 1e-9


def _rows(rows, times):
    r = rows.cpu().numpy().reshape(-1, 3)
    t = times.cpu().numpy().reshape(-1)
    n = int((r[:, 0] >= 0).sum())
    assert (r[:n, 0] >= 0).all() and (r[n:] == -1).all()
    return sorted((tuple(a), float(b)) for a, b in zip(r[:n].tolist(), t[:n].tolist()))


def _same(a, b):
    assert [k for k, _ in a] == [k for k, _ in b]
    ta = np.array([t for _, t in a])
    tb = np.array([t for _, t in b])
    assert (np.abs(ta - tb) <= TOI_RTOL * np.maximum(np.abs(tb), 1e-12)).all()


def test_static_scratch_entry_point_matches_workspace_entry_point():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cccollisions_b200 import build
    build.build()
    from cccollisions_b200 import _native as N
    from cccollisions_b200 import workloads as W
    import cccollisions_b200 as C

    lib = N.lib()
    dev = torch.device("cuda:0")
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    maxc = maxcol = 16
    cases = [W.cloth_sphere(seed=3, nx=40, ny=40, level=3),
             W.cloth_sphere(seed=4, nx=40, ny=40, level=3, dtype=np.float32),
             tuple(a[None] for a in W.jittered_fold(77, 14, 12)[:2])]
    for x0, x1 in cases:
        B, F = x0.shape[0], x0.shape[1]
        dtype = 1 if x0.dtype == np.float64 else 0
        X0 = torch.from_numpy(x0).to(dev)
        X1 = torch.from_numpy(x1).to(dev)
        bb, tr = C.bvh_motion(X0, X1)
        # reference answer: the entry point that takes a caller workspace
        ws = torch.empty(lib.ccc_workspace_size(N.OP_CONTINUOUS, B, F, maxc), dtype=torch.uint8, device=dev)
        r0 = torch.full((B, F * maxcol, 3), -1, dtype=torch.int64, device=dev)
        t0 = torch.full((B, F * maxcol, 1), -1, dtype=X0.dtype, device=dev)
        assert lib.ccc_find_collisions_continuous(dtype, P(bb), P(tr), P(X0), P(X1), None, B, F, maxc, maxcol, P(r0),
                                                  P(t0), P(ws), ws.numel(), stream) == 0
        expect = _rows(r0, t0)
        assert len(expect) > 0
        for _ in range(2):
            r1 = torch.full_like(r0, -1)
            t1 = torch.full_like(t0, -1)
            rc = lib.ccc_find_collisions_continuous_static(dtype, P(bb), P(tr), P(X0), P(X1), None, B, F, maxc,
                                                           maxcol, P(r1), P(t1), stream)
            assert rc == 0
            torch.cuda.synchronize(dev)
            _same(_rows(r1, t1), expect)
            st = (ctypes.c_int32 * 3)()
            assert lib.ccc_static_scratch_read_status(1, st, stream) == 0
            assert st[0] == 0 and st[2] == len(expect)


def test_static_scratch_status_reports_candidate_overflow():
    """A caller of the no-allocation entry point reads its status word without a workspace
    pointer: one candidate per triangle is far too few for a folded cloth, so the
    candidate-overflow bit is set (the rows are then a truncated set, as the reference
    warns); a following call with room clears it again."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cccollisions_b200 import _native as N
    from cccollisions_b200 import workloads as W
    import cccollisions_b200 as C

    lib = N.lib()
    dev = torch.device("cuda:0")
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    x0, x1, _ = W.jittered_fold(78, 14, 12)
    X0 = torch.from_numpy(x0[None]).to(dev)
    X1 = torch.from_numpy(x1[None]).to(dev)
    bb, tr = C.bvh_motion(X0, X1)
    F = x0.shape[0]
    for maxc, overflow in ((1, True), (16, False)):
        rows = torch.full((1, F * 16, 3), -1, dtype=torch.int64, device=dev)
        times = torch.full((1, F * 16, 1), -1, dtype=torch.float64, device=dev)
        assert lib.ccc_find_collisions_continuous_static(1, P(bb), P(tr), P(X0), P(X1), None, 1, F, maxc, 16,
                                                         P(rows), P(times), stream) == 0
        st = (ctypes.c_int32 * 3)()
        assert lib.ccc_static_scratch_read_status(1, st, stream) == 0
        assert bool(st[0] & N.CCC_ST_CAND_OVERFLOW) == overflow
        assert st[1] > F if overflow else st[1] <= 16 * F
        ctr = (ctypes.c_int32 * 4)()
        assert lib.ccc_static_scratch_read_counters(ctr, stream) == 0
        assert ctr[0] == st[0] and ctr[1] == st[1]


def test_static_scratch_rejects_oversized_problems():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cccollisions_b200 import _native as N
    lib = N.lib()
    limit = lib.ccc_static_scratch_bytes()
    assert limit == 64 << 20
    F = 400_000
    assert lib.ccc_workspace_size(N.OP_CONTINUOUS, 1, F, 16) > limit
    # rejected before any pointer is touched
    rc = lib.ccc_find_collisions_continuous_static(1, None, None, None, None, None, 1, F, 16, 16, None, None, None)
    assert rc == N.CCC_ERR_TOO_LARGE
