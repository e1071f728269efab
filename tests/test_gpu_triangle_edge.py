"""Parity of the triangle-edge queries on sm_100a (through the C ABI) with the CPU oracle.

find_triangle_edge_collisions / _candidates / _candidates2 (collisions_static.cu:345-942,
icontour.cu:11-281).  Bars: rows equal as multisets (the reference's order is
nondeterministic), -1 padding after the valid rows; edge coefficients bit-exact (the same
IEEE expressions on both sides, portable elementary functions).
"""
import numpy as np
import pytest
import torch

from conftest import random_mesh_soup

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def portable_math(cuda):
    from cccollisions_b200 import _native as N
    with N.math_library(N.LIB_PORTABLE):
        yield


def _t(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _valid(rows):
    n = int((rows[:, 0] >= 0).sum())
    assert (rows[:n, 0] >= 0).all() and (rows[n:] == -1).all(), "valid rows are not packed at the front"
    return n


def _check_mesh(C, oracle, x, dev, mc):
    X = _t(x[None], dev)
    bb, tr = C.bvh(X)
    b, t = bb[0].cpu().numpy(), tr[0].cpu().numpy()
    rows, coefs = C.find_triangle_edge_collisions(bb, tr, X, 0.0, mc)
    assert rows.shape == (1, x.shape[0] * mc, 4) and coefs.shape == (1, x.shape[0] * mc, 1)
    assert coefs.dtype == bb.dtype
    r = rows[0].cpu().numpy()
    n = _valid(r)
    c = coefs[0, :, 0].cpu().numpy()
    assert (c[n:] == -1).all()
    er, ec = oracle.triangle_edge_collisions(b, t, x)
    assert sorted(zip(map(tuple, r[:n].tolist()), c[:n].tolist())) == sorted(zip(map(tuple, er.tolist()),
                                                                                  ec.tolist()))
    cand = C.find_triangle_edge_candidates(bb, tr, X, 0.0, mc)[0].cpu().numpy()
    n = _valid(cand)
    ecand = oracle.triangle_edge_candidates(b, t, x)
    assert sorted(map(tuple, cand[:n].tolist())) == sorted(map(tuple, ecand.tolist()))
    pairs, masks = C.find_triangle_edge_candidates2(bb, tr, X, 0.0, mc)
    assert masks.dtype == torch.int32
    p = pairs[0].cpu().numpy()
    m = masks[0].cpu().numpy()
    n = _valid(p)
    assert (m[n:] == 0).all()
    ep, em = oracle.triangle_edge_candidates2(b, t, x)
    got = sorted(zip(map(tuple, p[:n].tolist()), map(tuple, m[:n].tolist())))
    assert got == sorted(zip(map(tuple, ep.tolist()), map(tuple, em.tolist())))
    return len(er), len(ecand), len(ep)


@pytest.mark.parametrize("seed,dtype", [(60, np.float64), (61, np.float32)])
def test_triangle_edge_random_fold(cuda, oracle, seed, dtype):
    import cccollisions_b200 as C
    x, _, _ = random_mesh_soup(seed, nx=14, ny=12, dtype=dtype)
    nx, nc, np_ = _check_mesh(C, oracle, x, cuda, 32)
    assert nx > 0 and nc > 0 and np_ > 0


def test_triangle_edge_static_fold_full_size(cuda, oracle):
    # the folded 64 x 64 sheet (7,938 triangles, fp32): about 14 candidate rows a triangle
    import cccollisions_b200 as C
    from cccollisions_b200 import workloads as W
    x = W.static_fold()[0]
    nx, nc, np_ = _check_mesh(C, oracle, x, cuda, 32)
    assert nx > 1000 and nc > 50000


def test_triangle_edge_known_answer(cuda, oracle):
    import cccollisions_b200 as C
    x = np.array([[(0.0, 0.0, 0.0), (1.0, 0.0, 0.0), (0.0, 1.0, 0.0)],
                  [(0.25, 0.25, -1.0), (0.25, 0.25, 1.0), (0.25, 2.0, 0.0)]])
    X = _t(x[None], cuda)
    bb, tr = C.bvh(X)
    rows, coefs = C.find_triangle_edge_collisions(bb, tr, X)
    r = rows[0].cpu().numpy()
    n = _valid(r)
    got = sorted(zip(map(tuple, r[:n].tolist()), coefs[0, :n, 0].cpu().tolist()))
    assert got == [((0, 1, 1, -1), 0.75), ((0, 1, 3, -1), 0.5)]


def test_triangle_edge_batch_slices(cuda, oracle):
    """Each batch item's rows land in its own slice, with mesh-local triangle ids."""
    import cccollisions_b200 as C
    xs = [random_mesh_soup(62 + k, nx=10, ny=9)[0] for k in range(3)]
    X = _t(np.stack(xs), cuda)
    bb, tr = C.bvh(X)
    rows, coefs = C.find_triangle_edge_collisions(bb, tr, X, 0.0, 32)
    cand = C.find_triangle_edge_candidates(bb, tr, X, 0.0, 32)
    for k, x in enumerate(xs):
        b, t = bb[k].cpu().numpy(), tr[k].cpu().numpy()
        r = rows[k].cpu().numpy()
        n = _valid(r)
        er, ec = oracle.triangle_edge_collisions(b, t, x)
        assert sorted(zip(map(tuple, r[:n].tolist()), coefs[k, :n, 0].cpu().tolist())) == \
            sorted(zip(map(tuple, er.tolist()), ec.tolist()))
        c = cand[k].cpu().numpy()
        assert sorted(map(tuple, c[:_valid(c)].tolist())) == \
            sorted(map(tuple, oracle.triangle_edge_candidates(b, t, x).tolist()))


def test_triangle_edge_capacity_and_empty(cuda, oracle):
    import cccollisions_b200 as C
    x, _, _ = random_mesh_soup(64, nx=12, ny=12)
    X = _t(x[None], cuda)
    bb, tr = C.bvh(X)
    ecand = oracle.triangle_edge_candidates(bb[0].cpu().numpy(), tr[0].cpu().numpy(), x)
    assert len(ecand) > x.shape[0]
    # two rows per triangle of room: the capacity is filled with oracle rows and the overflow
    # is reported as a warning (the reference writes past its tensor in this case)
    with pytest.warns(RuntimeWarning, match="exceeds maximal allowed number"):
        cand = C.find_triangle_edge_candidates(bb, tr, X, 0.0, 2)
    c = cand[0].cpu().numpy()
    assert _valid(c) == 2 * x.shape[0]
    assert set(map(tuple, c.tolist())) <= set(map(tuple, ecand.tolist()))
    # two far-apart triangles: nothing
    far = np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]], [[5, 5, 5], [6, 5, 5], [5, 6, 5]]], dtype=np.float64)
    F = _t(far[None], cuda)
    bb, tr = C.bvh(F)
    rows, coefs = C.find_triangle_edge_collisions(bb, tr, F)
    assert (rows == -1).all() and (coefs == -1).all()
    pairs, masks = C.find_triangle_edge_candidates2(bb, tr, F)
    assert (pairs == -1).all() and (masks == 0).all()
