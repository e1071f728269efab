"""The default (reference-math) mode against the reference extension at the measured
workloads' full sizes (tests/golden/full_*.npz, written by tests/golden/make_full_golden.py,
which ran the reference's own query calls on a B200 on reference-order trees).

Bars:
  * continuous-collision rows: equal multisets with bit-equal times, shown by equal digests
    (SHA-256 of the rows sorted with their times' IEEE bits) and, for the cloth-over-sphere
    step, row by row (a time within 1e-9 relative is the declared tolerance; every time is
    in fact bit-equal);
  * impulses: every corner counter equal; dv / dx within 1e-6 relative (plus 1e-12 of the
    largest magnitude) at 16,384 seeded contact corners; column sums within 1e-9 of the
    summed magnitudes (fp64 atomics add the contacts in any order).
The inputs are regenerated from their seeds and checked against the recorded input digests.
"""
import os
import sys

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
from make_full_golden import canonical_rows, input_digest, partial_mask, row_digest  # noqa: E402

TOI_RTOL = 1e-9
IMPULSE_RTOL = 1e-6


def _load(name):
    p = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(p):
        pytest.skip(f"missing fixture {name}")
    return np.load(p)


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _valid(rows, times):
    r = rows[0].cpu().numpy()
    n = int((r[:, 0] >= 0).sum())
    assert (r[n:] == -1).all()
    return r[:n], times[0, :n, 0].cpu().numpy().astype(np.float64)


@pytest.fixture
def reference_math(cuda):
    from cccollisions_b200 import _native as N
    with N.math_library(N.LIB_REFERENCE):
        yield


def test_cloth_sphere_rows_equal_reference(reference_math):
    """52,738 fp64 triangles, bvh_motion + find_collisions_continuous(16, 16) and the partial
    variant under a seeded 30 % mask."""
    import cccollisions_b200 as C
    from cccollisions_b200 import workloads as W
    d = _load("full_cloth_sphere")
    x0, x1 = W.cloth_sphere()
    assert input_digest(x0[0], x1[0]) == str(d["input_digest"])
    X0, X1 = _t(x0), _t(x1)
    bb, tr = C.bvh_motion(X0, X1)
    r, t = _valid(*C.find_collisions_continuous(bb, tr, X0, X1, 16, 16))
    got = canonical_rows(r, t)
    assert got.shape[0] == d["rows"].shape[0] == 79914
    assert (got[:, :3] == d["rows"]).all()
    gt = got[:, 3].view(np.float64)
    err = np.abs(gt - d["times"]) / np.maximum(np.abs(d["times"]), 1e-12)
    assert err.max() <= TOI_RTOL
    assert (got[:, 3] == d["times"].view(np.int64)).all()
    assert row_digest(r, t) == str(d["digest"])
    mask = partial_mask(x0.shape[1])
    pr, pt = _valid(*C.find_collisions_continuous_partial(bb, tr, X0, X1, _t(mask[None]), 16, 16))
    assert len(pr) == int(d["partial_rows"])
    assert row_digest(pr, pt) == str(d["partial_digest"])


def test_impulse_fold_matches_reference(reference_math):
    """130,050 fp64 triangles folded through themselves, compute_impulses(32, 16)."""
    import cccollisions_b200 as C
    from cccollisions_b200 import workloads as W
    d = _load("full_impulse_fold")
    x0, x1, m = W.impulse_fold()
    assert input_digest(x0[0], x1[0], m[0]) == str(d["input_digest"])
    X0, X1 = _t(x0), _t(x1)
    bb, tr = C.bvh_motion(X0, X1)
    dv, dx, cnt = C.compute_impulses(bb, tr, X0, X1, _t(m), 32, 16)
    cnt = cnt[0].cpu().numpy()
    assert cnt.sum() > 1_000_000
    assert (cnt == d["cnt"]).all()
    idx = d["corners"]
    for got, key in ((dv, "dv"), (dx, "dx")):
        g = got[0].cpu().numpy().reshape(-1, 3)
        want = d[key]
        scale = np.abs(want).max()
        assert (np.abs(g[idx] - want) <= IMPULSE_RTOL * np.abs(want) + 1e-12 * scale).all()
        assert (g[cnt.reshape(-1) == 0] == 0).all()
        assert (np.abs(g.sum(axis=0) - d[key + "_sum"]) <= 1e-9 * d[key + "_abs_sum"]).all()


def _batched_meshes(d):
    from cccollisions_b200 import workloads as W
    meshes = W.batched()
    assert [a.shape[0] for a, _ in meshes] == d["F"].tolist()
    for (a, b), dig in zip(meshes, d["input_digests"]):
        assert input_digest(a, b) == str(dig)
    return meshes


def test_batched_engine_rows_equal_reference(reference_math):
    """The batched step (64 meshes, 2.62 M triangles, resident engine) against the reference's
    find_collisions_continuous per mesh: per-mesh row counts and digests."""
    from cccollisions_b200.engine import Engine
    d = _load("full_batched")
    meshes = _batched_meshes(d)
    Fs = d["F"].tolist()
    eng = Engine(tri_capacity=sum(Fs) + 64, mesh_capacity=len(Fs), max_candidates_per_triangle=32,
                 max_collisions_per_triangle=16)
    try:
        sids = [eng.add_mesh(f) for f in Fs]
        for sid, (a, b) in zip(sids, meshes):
            eng.upload_soup(sid, a, b)
        eng.set_active(sids)
        eng.build(sids)
        eng.ccd()
        st = eng.state(sids)
        assert st["status"] == 0
        assert st["rows"].tolist() == d["rows"].tolist()
        bad = []
        for i, sid in enumerate(sids):
            r, t = [x.cpu().numpy() for x in eng.collisions(sid, int(st["rows"][i]))]
            if row_digest(r, t) != str(d["digests"][i]):
                bad.append(i)
        assert not bad, bad
    finally:
        eng.close()


def test_batched_reference_format_rows_equal_reference(reference_math):
    """The plain per-mesh path (bvh_motion + find_collisions_continuous through the
    reference-format API) on the same 64 meshes: per-mesh digests."""
    import cccollisions_b200 as C
    d = _load("full_batched")
    meshes = _batched_meshes(d)
    bad = []
    for i, (a, b) in enumerate(meshes):
        A, B = _t(a[None]), _t(b[None])
        bb, tr = C.bvh_motion(A, B)
        r, t = _valid(*C.find_collisions_continuous(bb, tr, A, B, int(d["maxc"][i]), 16))
        if len(r) != int(d["rows"][i]) or row_digest(r, t) != str(d["digests"][i]):
            bad.append(i)
    assert not bad, bad
