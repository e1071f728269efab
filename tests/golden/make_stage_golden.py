"""Record the reference's continuous-collision arithmetic stage by stage on a GPU.

    python oracle/build_ref.py                         # here: builds oracle/_ref/libref_probe.so
    python tests/golden/make_stage_golden.py [--out DIR]   # on a CUDA machine

oracle/ref_probe.cu exposes four of the reference's own kernels (cubic coefficients,
Cardano solve, root filter, contact kinematics), compiled with the reference's build flags.
This script feeds them the tetrahedra of sampled (i, j, type) sub-tests from the golden
soups (tests/golden/soup_*.npz) and from the cloth-over-sphere workload, and writes
``stages_<name>.npz``: the sampled items plus each stage's outputs.  Sub-tests are sampled,
not exhaustive, to keep fixtures small.  All kernels are straight-line code on valid
inputs.
"""
from __future__ import annotations

import argparse
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

EA, EB = [0, 0, 1], [1, 2, 2]


def tet_points(k):
    if k < 9:
        e0, e1 = k // 3, k % 3
        return [(0, EA[e0]), (0, EB[e0]), (1, EA[e1]), (1, EB[e1])]
    if k < 12:
        return [(0, 0), (0, 1), (0, 2), (1, k - 9)]
    return [(0, k - 12), (1, 0), (1, 1), (1, 2)]


def tets_of(x0, x1, items):
    """MovingTetrahedron rows (v0..v3, dv0..dv3) of (i, j, k) items, dv = x1 - x0."""
    out = np.zeros((len(items), 24))
    for n, (i, j, k) in enumerate(items):
        for p, (s, c) in enumerate(tet_points(int(k))):
            t = j if s else i
            out[n, 3 * p:3 * p + 3] = x0[t, c]
            out[n, 12 + 3 * p:12 + 3 * p + 3] = x1[t, c] - x0[t, c]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "golden_out"))
    ap.add_argument("--per-source", type=int, default=4000)
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    import torch
    from cccollisions_b200 import workloads as W
    from oracle import oracle as O
    O.build()
    L = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_probe.so"))
    dev = torch.device("cuda:0")
    P = lambda t: ctypes.c_void_p(t.data_ptr())

    sources = {}
    for name in ("soup_20_float64", "soup_21_float64", "soup_23_float64"):
        d = np.load(os.path.join(HERE, name + ".npz"))
        sources[name] = (d["x0"], d["x1"])
    x0, x1 = W.cloth_sphere()
    sources["cloth_sphere"] = (x0[0], x1[0])
    g = np.random.default_rng(0)
    for name, (x0, x1) in sources.items():
        bb, tr = O.bvh(x0, x1)
        mc = O.mincol_cand(bb, tr, x0, x1)
        sel = np.sort(g.choice(len(mc), min(args.per_source, len(mc)), replace=False))
        items = mc[sel]
        tets = tets_of(x0, x1, items)
        n = len(items)
        T = torch.from_numpy(tets).to(dev)
        C = torch.zeros((n, 4), dtype=torch.float64, device=dev)
        S = torch.zeros((n, 3), dtype=torch.int64, device=dev)
        assert L.ref_cubic_coeffs(P(T), P(C), P(S), n) == 0
        R = torch.full((n, 3), -1.0, dtype=torch.float64, device=dev)
        assert L.ref_solve_cubic(P(C), P(R), n) == 0
        roots = R.cpu().numpy()
        # one filter / contact row per root in [0, 1] (flatten_cubic_roots order)
        fi = [(a, s) for a in range(n) for s in range(3) if 0 <= roots[a, s] <= 1]
        idx = np.array([a for a, _ in fi], dtype=np.int64)
        fr = np.array([roots[a, s] for a, s in fi])
        m = len(fi)
        out = {"items": items.astype(np.int32), "coefs": C.cpu().numpy(), "roots": roots,
               "flt_item": idx.astype(np.int32), "flt_root": fr}
        if m:
            Tf = torch.from_numpy(tets[idx]).to(dev)
            tids = torch.from_numpy(items[idx].astype(np.int64)).to(dev)
            Rf = torch.from_numpy(fr).to(dev)
            V = torch.zeros(m, dtype=torch.bool, device=dev)
            assert L.ref_filter(P(Tf), P(tids), P(Rf), P(V), m) == 0
            mq = g.uniform(0.5, 2.0, (m, 4))
            MQ = torch.from_numpy(mq).to(dev)
            co = torch.full((m, 3), -1.0, dtype=torch.float64, device=dev)
            nr = torch.full((m, 3), -1.0, dtype=torch.float64, device=dev)
            vn = torch.zeros(m, dtype=torch.float64, device=dev)
            ve = torch.zeros(m, dtype=torch.float64, device=dev)
            mp = torch.zeros((m, 2), dtype=torch.float64, device=dev)
            assert L.ref_contact(P(Tf), P(tids), P(Rf), P(MQ), P(co), P(nr), P(vn), P(ve), P(mp), m) == 0
            out.update(flt_valid=V.cpu().numpy(), ct_mass_quads=mq, ct_coefficients=co.cpu().numpy(),
                       ct_normals=nr.cpu().numpy(), ct_vn=vn.cpu().numpy(), ct_mass_pairs=mp.cpu().numpy())
        if name == "cloth_sphere":
            out["tets"] = tets
        np.savez_compressed(os.path.join(args.out, f"stages_{name}.npz"), **out)
        print(name, "items", n, "roots in [0,1]", m)


if __name__ == "__main__":
    main()
