"""Device arithmetic of the cubic solver vs the CPU oracle (bit for bit), and the library's
own elementary functions vs CUDA's (error bounds)."""
import ctypes
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _run(op, inp):
    from cccollisions_b200 import _native as N
    x = torch.from_numpy(np.ascontiguousarray(inp, dtype=np.float64).reshape(-1, 4)).cuda()
    out = torch.empty((x.shape[0], 3), dtype=torch.float64, device="cuda")
    rc = N.lib().ccc_debug_math(op, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()), x.shape[0],
                                ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _col(v):
    a = np.zeros((len(v), 4))
    a[:, 0] = v
    return a


def _bits_equal(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return (a.view(np.int64) == b.view(np.int64)) | (np.isnan(a) & np.isnan(b))


def test_elementary_functions_match_oracle(cuda, oracle):
    g = np.random.default_rng(3)
    xs = np.concatenate([np.exp(g.uniform(-700, 700, 2000)), -np.exp(g.uniform(-50, 50, 500)), [0.0, 1e-310]])
    got = _run(0, _col(xs))[:, 0]
    exp = np.array([oracle.cbrt(x) for x in xs])
    assert _bits_equal(got, exp).all(), xs[~_bits_equal(got, exp)][:5]
    us = g.uniform(-1, 1, 3000)
    assert _bits_equal(_run(1, _col(us))[:, 0], [oracle.acos(x) for x in us]).all()
    ts = g.uniform(0, math.pi / 3, 3000)
    assert _bits_equal(_run(2, _col(ts))[:, 0], [oracle.cos(x) for x in ts]).all()
    assert _bits_equal(_run(3, _col(ts))[:, 0], [oracle.sin(x) for x in ts]).all()


def test_elementary_functions_vs_cuda(cuda):
    g = np.random.default_rng(4)
    xs = np.exp(g.uniform(-300, 300, 2000))
    ours = _run(0, _col(xs))[:, 0]
    theirs = _run(6, _col(xs))[:, 0]
    assert (np.abs(ours - theirs) <= 2 * np.spacing(np.abs(theirs))).all()
    us = g.uniform(-1, 1, 2000)
    assert (np.abs(_run(1, _col(us))[:, 0] - _run(7, _col(us))[:, 0]) <= 4 * np.spacing(np.pi)).all()
    ts = g.uniform(0, math.pi / 3, 2000)
    for a, b in ((2, 8), (3, 9)):
        o, c = _run(a, _col(ts))[:, 0], _run(b, _col(ts))[:, 0]
        assert (np.abs(o - c) <= 3 * np.spacing(np.maximum(np.abs(c), 1e-300))).all()


def test_certified_product_matches_oracle(cuda, oracle):
    g = np.random.default_rng(5)
    rows = []
    exp = []
    for _ in range(2000):
        b = float(g.uniform(-1, 1) * 10.0 ** g.integers(-12, 3))
        r = oracle.certmul(b, b)
        rows.append([b, 0.0, 1, b])
        exp.append(r)
        rows.append([r[0], r[1], 2, b])
        exp.append(oracle.certmul(r, b))
    got = _run(4, np.array(rows))[:, :2]
    assert _bits_equal(got, np.array(exp)).all()


def test_solve_cubic_matches_oracle(cuda, oracle):
    g = np.random.default_rng(6)
    cases = []
    for _ in range(3000):
        r = np.sort(g.uniform(-0.5, 1.5, 3))
        s = 10.0 ** g.uniform(-12, 0)
        a = s
        b = -s * r.sum()
        c = s * (r[0] * r[1] + r[1] * r[2] + r[0] * r[2])
        d = -s * r.prod()
        cases.append([a, b, c, d])
    for _ in range(1000):
        cases.append(list(g.normal(0, 1, 4) * 10.0 ** g.uniform(-10, 0)))
    cases += [[1e-18, 1.0, -1.0, 0.1875], [0.0, 0.0, 1.0, -0.5], [1.0, -1.5, 0.75, -0.125]]
    cases = np.array(cases)
    got = _run(5, cases)
    exp = np.array([oracle.solve_cubic(*c) for c in cases])
    bad = ~_bits_equal(got, exp).all(axis=1)
    assert not bad.any(), (cases[bad][:3], got[bad][:3], exp[bad][:3])
