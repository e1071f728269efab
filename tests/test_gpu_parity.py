"""Parity of the sm_100a path (through the C ABI) with the CPU oracle.

Bars (stated per result):
  * BVH tensors: bit-exact (same topology, same boxes, same ids).
  * Collision / proximity / candidate rows: equal as multisets (the reference's row order
    is nondeterministic), -1 padding after the valid rows.
  * Times of impact: bit-exact (both sides evaluate the same IEEE expressions with the
    same elementary functions); the declared tolerance is 1e-9 relative.
  * Impulses dv, dx: within 1e-6 relative (floating-point atomics sum in any order);
    counters exact.
"""
import numpy as np
import pytest
import torch

from conftest import random_mesh_soup

pytestmark = pytest.mark.gpu

TOI_RTOL = 1e-9


@pytest.fixture(autouse=True)
def portable_math(cuda):
    """The oracle shares the library's portable elementary functions, so bit-exact parity
    is checked in that mode (the default mode calls CUDA's, as the reference does, and is
    checked against the reference's own outputs in test_gpu_reference.py)."""
    from cccollisions_b200 import _native as N
    with N.math_library(N.LIB_PORTABLE):
        yield
IMPULSE_RTOL = 1e-6


def _t(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _valid_prefix(rows):
    """rows (R, k) int64 numpy: valid rows must be a prefix, the rest all -1."""
    valid = rows[:, 0] >= 0
    n = int(valid.sum())
    assert valid[:n].all(), "valid rows are not packed at the front"
    assert (rows[n:] == -1).all()
    return n


def _rows_multiset(rows, times=None):
    if times is None:
        return sorted(map(tuple, rows.tolist()))
    return sorted((tuple(r), float(t)) for r, t in zip(rows.tolist(), np.asarray(times).ravel().tolist()))


def _assert_same_rows_times(got_rows, got_times, exp_rows, exp_times):
    g = _rows_multiset(got_rows, got_times)
    e = _rows_multiset(exp_rows, exp_times)
    gk = [r for r, _ in g]
    ek = [r for r, _ in e]
    assert len(gk) == len(ek), f"row counts differ: gpu {len(gk)} oracle {len(ek)}"
    assert gk == ek, "row multisets differ"
    gt = np.array([t for _, t in g])
    et = np.array([t for _, t in e])
    err = np.abs(gt - et) / np.maximum(np.abs(et), 1e-12)
    assert err.max(initial=0) <= TOI_RTOL, f"TOI rel err {err.max()}"
    assert (gt == et).all(), f"TOI not bit-exact: max rel err {err.max()}"


def _impulse_close(a, b):
    """dv / dx agreement: 1e-6 relative for float64.  Contacts are summed per corner with
    atomics in any order, so in float32 the bound is float32 summation error: 1e-5
    relative plus 1e-6 of the largest magnitude."""
    single = np.asarray(b).dtype == np.float32
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.abs(b).max(initial=0.0)
    if single:
        tol = 1e-5 * np.abs(b) + 1e-6 * max(scale, 1e-30)
    else:
        tol = IMPULSE_RTOL * np.abs(b) + 1e-12 * max(scale, 1e-30)
    bad = ~(np.abs(a - b) <= tol)
    both_nan = np.isnan(a) & np.isnan(b)
    bad &= ~both_nan
    return not bad.any(), float(np.nanmax(np.abs(a - b), initial=0.0))


# ------------------------------------------------------------------------------ BVH

@pytest.mark.parametrize("seed,dtype,motion", [(0, np.float32, False), (1, np.float64, False),
                                               (2, np.float64, True), (3, np.float32, True)])
def test_bvh_bit_exact(cuda, oracle, seed, dtype, motion):
    import cccollisions_b200 as C
    x0, x1, _ = random_mesh_soup(seed, nx=11, ny=9, dtype=dtype)
    if motion:
        bb, tr = C.bvh_motion(_t(x0[None], cuda), _t(x1[None], cuda))
        ebb, etr = oracle.bvh(x0, x1)
    else:
        bb, tr = C.bvh(_t(x0[None], cuda))
        ebb, etr = oracle.bvh(x0)
    assert bb.dtype == torch.float64 if dtype == np.float64 else torch.float32
    assert tr.dtype == torch.int64
    assert (tr[0].cpu().numpy() == etr).all()
    assert (bb[0].cpu().numpy() == ebb).all()


def test_bvh_full_size_cloth_sphere(cuda, oracle):
    import cccollisions_b200 as C
    from cccollisions_b200 import workloads as W
    x0, x1 = W.cloth_sphere()
    bb, tr = C.bvh_motion(_t(x0, cuda), _t(x1, cuda))
    ebb, etr = oracle.bvh(x0[0], x1[0])
    assert (tr[0].cpu().numpy() == etr).all()
    assert (bb[0].cpu().numpy() == ebb).all()


def test_bvh_two_triangles_and_batch(cuda, oracle):
    import cccollisions_b200 as C
    x0, _, _ = random_mesh_soup(9, nx=3, ny=2)        # F = 4
    x = np.stack([x0[:2], x0[2:]])                     # B = 2, F = 2
    bb, tr = C.bvh(_t(x, cuda))
    for b in range(2):
        ebb, etr = oracle.bvh(x[b])
        assert (tr[b].cpu().numpy() == etr).all()
        assert (bb[b].cpu().numpy() == ebb).all()


# ------------------------------------------------------------------------------ static

@pytest.mark.parametrize("threshold", [0.0, 0.01])
def test_find_collisions_static_fold(cuda, oracle, threshold):
    import cccollisions_b200 as C
    from cccollisions_b200 import workloads as W
    x = W.static_fold()
    bb, tr = C.bvh(_t(x, cuda))
    out = C.find_collisions(bb, tr, _t(x, cuda), threshold=threshold, max_collisions=16)
    assert out.shape == (1, x.shape[1] * 16, 2) and out.dtype == torch.int64
    rows = out[0].cpu().numpy()
    n = _valid_prefix(rows)
    exp = oracle.find_collisions(bb[0].cpu().numpy(), tr[0].cpu().numpy(), x[0], threshold=threshold)
    assert n == len(exp) > 0
    assert _rows_multiset(rows[:n]) == _rows_multiset(exp)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_find_collisions_batch_random(cuda, oracle, dtype):
    import cccollisions_b200 as C
    xs = np.stack([random_mesh_soup(s, nx=10, ny=10, dtype=dtype)[0] for s in (11, 12, 13)])
    bb, tr = C.bvh(_t(xs, cuda))
    F, mc = xs.shape[1], 32
    for b in range(3):    # stay within the candidate capacity (the reference wraps around beyond it)
        assert len(oracle.candidates(bb[b].cpu().numpy(), tr[b].cpu().numpy(), threshold=0.005)) <= F * mc
    out = C.find_collisions(bb, tr, _t(xs, cuda), 0.005, mc).cpu().numpy()
    for b in range(3):
        n = _valid_prefix(out[b])
        exp = oracle.find_collisions(bb[b].cpu().numpy(), tr[b].cpu().numpy(), xs[b], threshold=0.005)
        assert _rows_multiset(out[b][:n]) == _rows_multiset(exp)


# ------------------------------------------------------------------------------ continuous

@pytest.mark.parametrize("seed,dtype", [(20, np.float64), (21, np.float64), (22, np.float32)])
def test_ccd_random(cuda, oracle, seed, dtype):
    import cccollisions_b200 as C
    x0, x1, _ = random_mesh_soup(seed, nx=14, ny=12, dtype=dtype)
    bb, tr = C.bvh_motion(_t(x0[None], cuda), _t(x1[None], cuda))
    rows, times = C.find_collisions_continuous(bb, tr, _t(x0[None], cuda), _t(x1[None], cuda))
    r = rows[0].cpu().numpy()
    t = times[0].cpu().numpy()
    n = _valid_prefix(r)
    assert (t[n:] == -1).all()
    er, et = oracle.ccd(bb[0].cpu().numpy(), tr[0].cpu().numpy(), x0, x1)
    assert len(er) > 0
    _assert_same_rows_times(r[:n], t[:n, 0], er, et)


def test_ccd_cloth_sphere_full_size(cuda, oracle):
    import cccollisions_b200 as C
    from cccollisions_b200 import workloads as W
    x0, x1 = W.cloth_sphere()
    X0, X1 = _t(x0, cuda), _t(x1, cuda)
    bb, tr = C.bvh_motion(X0, X1)
    rows, times = C.find_collisions_continuous(bb, tr, X0, X1, 16, 16)
    r = rows[0].cpu().numpy()
    t = times[0].cpu().numpy()
    n = _valid_prefix(r)
    er, et = oracle.ccd(bb[0].cpu().numpy(), tr[0].cpu().numpy(), x0[0], x1[0], nthreads=0)
    _assert_same_rows_times(r[:n], t[:n, 0], er, et)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_ccd_rigid_pieces(cuda, oracle, dtype):
    """Triangles that stand still or translate rigidly (all six vertices of a pair with the
    same displacement) beside deforming ones: the pairs inside a rigid piece give nothing,
    the pairs across pieces give the oracle's rows."""
    import cccollisions_b200 as C
    x0, x1, _ = random_mesh_soup(24, nx=16, ny=14, dtype=dtype)
    F = x0.shape[0]
    x1 = x1.copy()
    x1[: F // 3] = x0[: F // 3]                                   # static piece
    x1[F // 3: 2 * F // 3] = x0[F // 3: 2 * F // 3] + dtype(0.125)  # translating piece
    bb, tr = C.bvh_motion(_t(x0[None], cuda), _t(x1[None], cuda))
    # room for every candidate and row (the pieces overlap after the fold: up to 24 rows a triangle)
    rows, times = C.find_collisions_continuous(bb, tr, _t(x0[None], cuda), _t(x1[None], cuda), 128, 64)
    r = rows[0].cpu().numpy()
    n = _valid_prefix(r)
    er, et = oracle.ccd(bb[0].cpu().numpy(), tr[0].cpu().numpy(), x0, x1)
    assert len(er) > 0
    _assert_same_rows_times(r[:n], times[0].cpu().numpy()[:n, 0], er, et)
    # the box-only candidate rows still list the rigid pairs' sub-tests
    mrows = C.find_mincol_cand(bb, tr, _t(x0[None], cuda), _t(x1[None], cuda), 128)
    mr = mrows[0].cpu().numpy()
    nm = _valid_prefix(mr)
    emr = oracle.mincol_cand(bb[0].cpu().numpy(), tr[0].cpu().numpy(), x0, x1)
    assert _rows_multiset(mr[:nm]) == _rows_multiset(emr)


def test_ccd_partial(cuda, oracle):
    import cccollisions_b200 as C
    x0, x1, _ = random_mesh_soup(23, nx=14, ny=12)
    g = np.random.default_rng(1)
    mask = g.random(x0.shape[0]) < 0.4
    bb, tr = C.bvh_motion(_t(x0[None], cuda), _t(x1[None], cuda))
    m = torch.from_numpy(mask[None]).to(cuda)
    rows, times = C.find_collisions_continuous_partial(bb, tr, _t(x0[None], cuda), _t(x1[None], cuda), m)
    r = rows[0].cpu().numpy()
    n = _valid_prefix(r)
    er, et = oracle.ccd(bb[0].cpu().numpy(), tr[0].cpu().numpy(), x0, x1, mask=mask.astype(np.uint8))
    _assert_same_rows_times(r[:n], times[0].cpu().numpy()[:n, 0], er, et)


def test_mincol_cand(cuda, oracle):
    import cccollisions_b200 as C
    x0, x1, _ = random_mesh_soup(24, nx=10, ny=10)
    bb, tr = C.bvh_motion(_t(x0[None], cuda), _t(x1[None], cuda))
    out = C.find_mincol_cand(bb, tr, _t(x0[None], cuda), _t(x1[None], cuda), 16)
    assert out.shape == (1, x0.shape[0] * 16 * 15, 3)
    r = out[0].cpu().numpy()
    n = _valid_prefix(r)
    exp = oracle.mincol_cand(bb[0].cpu().numpy(), tr[0].cpu().numpy(), x0, x1)
    assert _rows_multiset(r[:n]) == _rows_multiset(exp)


# ------------------------------------------------------------------------------ impulses

@pytest.mark.parametrize("seed,dtype", [(30, np.float64), (31, np.float32)])
def test_compute_impulses_random(cuda, oracle, seed, dtype):
    import cccollisions_b200 as C
    x0, x1, m = random_mesh_soup(seed, nx=14, ny=12, dtype=dtype)
    X0, X1, Mt = _t(x0[None], cuda), _t(x1[None], cuda), _t(m[None], cuda)
    bb, tr = C.bvh_motion(X0, X1)
    dv, dx, cnt = C.compute_impulses(bb, tr, X0, X1, Mt)
    assert dv.shape == (1, x0.shape[0], 3, 3) and cnt.dtype == torch.int32
    edv, edx, ecnt, nc = oracle.impulses(bb[0].cpu().numpy(), tr[0].cpu().numpy(), x0, x1, m)
    assert nc > 0
    assert (cnt[0].cpu().numpy() == ecnt).all()
    ok, err = _impulse_close(dv[0].cpu().numpy(), edv)
    assert ok, err
    ok, err = _impulse_close(dx[0].cpu().numpy(), edx)
    assert ok, err


def test_compute_impulses_partial(cuda, oracle):
    import cccollisions_b200 as C
    x0, x1, m = random_mesh_soup(32, nx=14, ny=12)
    mask = np.random.default_rng(2).random(x0.shape[0]) < 0.5
    X0, X1, Mt = _t(x0[None], cuda), _t(x1[None], cuda), _t(m[None], cuda)
    bb, tr = C.bvh_motion(X0, X1)
    dv, dx, cnt = C.compute_impulses_partial(bb, tr, X0, X1, Mt, torch.from_numpy(mask[None]).to(cuda))
    edv, edx, ecnt, _ = oracle.impulses(bb[0].cpu().numpy(), tr[0].cpu().numpy(), x0, x1, m,
                                        mask=mask.astype(np.uint8))
    assert (cnt[0].cpu().numpy() == ecnt).all()
    assert _impulse_close(dv[0].cpu().numpy(), edv)[0]
    assert _impulse_close(dx[0].cpu().numpy(), edx)[0]


def test_compute_impulses_from_collisions(cuda, oracle):
    import cccollisions_b200 as C
    x0, x1, m = random_mesh_soup(33, nx=14, ny=12)
    X0, X1, Mt = _t(x0[None], cuda), _t(x1[None], cuda), _t(m[None], cuda)
    bb, tr = C.bvh_motion(X0, X1)
    rows, times = C.find_collisions_continuous(bb, tr, X0, X1)
    # includes the -1 padding rows, which are skipped
    dv, dx, cnt = C.compute_impulses_from_collisions(rows, times, X0, X1, Mt)
    r = rows[0].cpu().numpy()
    n = _valid_prefix(r)
    edv, edx, ecnt = oracle.impulses_from_rows(x0, x1, m, r[:n], times[0].cpu().numpy()[:n, 0])
    assert (cnt[0].cpu().numpy() == ecnt).all()
    assert _impulse_close(dv[0].cpu().numpy(), edv)[0]
    assert _impulse_close(dx[0].cpu().numpy(), edx)[0]


def test_compute_impulses_fold_full_size(cuda, oracle):
    import cccollisions_b200 as C
    from cccollisions_b200 import workloads as W
    x0, x1, m = W.impulse_fold()
    X0, X1, Mt = _t(x0, cuda), _t(x1, cuda), _t(m, cuda)
    bb, tr = C.bvh_motion(X0, X1)
    # 21.3 candidates per triangle: the reference's default of 16 would wrap around
    dv, dx, cnt = C.compute_impulses(bb, tr, X0, X1, Mt, 32, 16)
    edv, edx, ecnt, nc = oracle.impulses(bb[0].cpu().numpy(), tr[0].cpu().numpy(), x0[0], x1[0], m[0], nthreads=0)
    assert nc > 1000
    assert (cnt[0].cpu().numpy() == ecnt).all()
    assert _impulse_close(dv[0].cpu().numpy(), edv)[0]
    assert _impulse_close(dx[0].cpu().numpy(), edx)[0]


# ------------------------------------------------------------------------------ proximity

@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_find_proximity(cuda, oracle, dtype):
    import cccollisions_b200 as C
    x0, _, _ = random_mesh_soup(40, nx=12, ny=12, dtype=dtype)
    X = _t(x0[None], cuda)
    bb, tr = C.bvh(X)
    (rows,) = C.find_proximity(bb, tr, X, 0.02)
    r = rows[0].cpu().numpy()
    n = _valid_prefix(r)
    er, _ = oracle.proximity(bb[0].cpu().numpy(), tr[0].cpu().numpy(), x0, 0.02)
    assert len(er) > 0
    assert _rows_multiset(r[:n]) == _rows_multiset(er)


# ------------------------------------------------------------------------------ interchange / errors

def test_foreign_spatial_tree_gives_same_pairs(cuda, oracle):
    # the traversal accepts any valid (bboxes, tree): a Morton-ordered tree from the
    # oracle's spatial build yields the same collision set
    import cccollisions_b200 as C
    x0, x1, _ = random_mesh_soup(50, nx=14, ny=12)
    sbb, str_ = oracle.bvh(x0, x1, spatial=True)
    X0, X1 = _t(x0[None], cuda), _t(x1[None], cuda)
    rows, times = C.find_collisions_continuous(_t(sbb[None], cuda), _t(str_[None], cuda), X0, X1)
    r = rows[0].cpu().numpy()
    n = _valid_prefix(r)
    bb, tr = oracle.bvh(x0, x1)
    er, et = oracle.ccd(bb, tr, x0, x1)
    _assert_same_rows_times(r[:n], times[0].cpu().numpy()[:n, 0], er, et)


def test_candidate_overflow_warns_and_truncates(cuda, oracle):
    import cccollisions_b200 as C
    from cccollisions_b200 import api
    x0, x1, _ = random_mesh_soup(51, nx=14, ny=12)
    X0, X1 = _t(x0[None], cuda), _t(x1[None], cuda)
    bb, tr = C.bvh_motion(X0, X1)
    with pytest.warns(RuntimeWarning, match="exceeds maximal allowed number"):
        rows, _ = C.find_collisions_continuous(bb, tr, X0, X1, 1, 16)
    _valid_prefix(rows[0].cpu().numpy())
    api.STRICT = True
    try:
        with pytest.raises(RuntimeError, match="exceeds maximal allowed number"):
            C.find_collisions_continuous(bb, tr, X0, X1, 1, 16)
    finally:
        api.STRICT = False
    # output capacity overflow keeps exactly F * max_collisions rows
    with pytest.warns(RuntimeWarning):
        rows, times = C.find_collisions_continuous(bb, tr, X0, X1, 16, 1)
    r = rows[0].cpu().numpy()
    er, _ = oracle.ccd(bb[0].cpu().numpy(), tr[0].cpu().numpy(), x0, x1)
    if len(er) > x0.shape[0]:
        assert _valid_prefix(r) == x0.shape[0]


def test_input_checks(cuda):
    import cccollisions_b200 as C
    x0, _, _ = random_mesh_soup(52)
    X = _t(x0[None], cuda)
    bb, tr = C.bvh(X)
    with pytest.raises(RuntimeError, match="contiguous"):
        C.find_collisions(bb.transpose(1, 2), tr, X)
    with pytest.raises(RuntimeError, match="CUDA"):
        C.find_collisions(bb, tr, X.cpu())


def test_empty_result(cuda, oracle):
    import cccollisions_b200 as C
    # two far-apart triangles: no candidate, all rows -1, impulses zero
    x0 = np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]], [[5, 5, 5], [6, 5, 5], [5, 6, 5]]], dtype=np.float64)
    x1 = x0 + 0.1
    X0, X1 = _t(x0[None], cuda), _t(x1[None], cuda)
    bb, tr = C.bvh_motion(X0, X1)
    rows, times = C.find_collisions_continuous(bb, tr, X0, X1)
    assert (rows == -1).all() and (times == -1).all()
    dv, dx, cnt = C.compute_impulses(bb, tr, X0, X1, torch.ones((1, 2, 3), dtype=torch.float64, device=cuda))
    assert (dv == 0).all() and (cnt == 0).all()
