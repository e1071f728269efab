"""Generate triangle-edge golden fixtures by running the reference extension on a GPU.

    python oracle/build_ref.py                       # here, where the reference sources are
    python tests/golden/make_te_golden.py [--out DIR]   # on a machine with a CUDA GPU

Runs the reference's find_triangle_edge_collisions / _candidates / _candidates2 (compiled
by oracle/build_ref.py into oracle/_ref/cccollisions.so) on seeded meshes and writes one
compressed .npz per case: the inputs, the oracle-built tree (bboxes, tree) and the
reference's valid rows.

Safety, checked on the CPU with the oracle before each call: F >= 2, tree depth far below
the reference's 64-entry traversal stack, candidates within F * max_collisions (no wrap of
the candidate buffer), and 6 x (intersecting pairs) within F * max_collisions rows, because
the reference copies six rows per intersecting pair into its output tensor
(collisions_static.cu:758-763, 910-915) and would write past its end otherwise.  The
reference's own bvh() is not run (see make_golden.py); the trees come from the oracle.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from make_golden import load_reference, tree_depth, valid  # noqa: E402

MC = 32


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "golden_out"))
    ap.add_argument("--extra-seeds", type=int, nargs="*", default=[],
                    help="further jittered folds (fp32 and fp64) to record, beside the fixed cases")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)

    import torch
    from cccollisions_b200 import workloads as W
    from oracle import oracle as O
    O.build()
    R = load_reference()
    dev = torch.device("cuda:0")
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    cases = {
        "te_fold_60_float64": W.jittered_fold(60, 14, 12, dtype=np.float64)[0],
        "te_fold_61_float32": W.jittered_fold(61, 14, 12, dtype=np.float32)[0],
        "te_fold_70_float32": W.jittered_fold(70, 14, 12, dtype=np.float32)[0],
        "te_fold_75_float32": W.jittered_fold(75, 14, 12, dtype=np.float32)[0],
        "te_fold_75_float64": W.jittered_fold(75, 14, 12, dtype=np.float64)[0],
        "te_static_fold": W.static_fold()[0],
    }
    for seed in args.extra_seeds:
        for dt in (np.float32, np.float64):
            cases[f"te_fold_{seed}_{np.dtype(dt).name}"] = W.jittered_fold(seed, 14, 12, dtype=dt)[0]
    for name, x in cases.items():
        F = x.shape[0]
        assert F >= 2
        bb, tr = O.bvh(x)
        assert tree_depth(tr) <= 48
        assert len(O.candidates(bb, tr)) <= MC * F
        nv0 = len(O.find_collisions(bb, tr, x))
        nv1 = len(O.triangle_edge_candidates2(bb, tr, x)[0])
        assert 6 * max(nv0, nv1) <= MC * F, (name, nv0, nv1)
        Bb, Tr, X = T(bb[None]), T(tr[None]), T(x[None])
        rows, coefs = R.find_triangle_edge_collisions(Bb, Tr, X, 0.0, MC)
        r = rows[0].cpu().numpy()
        n = int((r[:, 0] >= 0).sum())
        out = {"x": x, "bboxes": bb, "tree": tr, "te_rows": r[:n], "te_coefs": coefs[0, :n, 0].cpu().numpy()}
        out["cand_rows"] = valid(R.find_triangle_edge_candidates(Bb, Tr, X, 0.0, MC)[0].cpu().numpy())
        pairs, masks = R.find_triangle_edge_candidates2(Bb, Tr, X, 0.0, MC)
        p = pairs[0].cpu().numpy()
        n2 = int((p[:, 0] >= 0).sum())
        out["cand2_pairs"], out["cand2_masks"] = p[:n2], masks[0, :n2].cpu().numpy()
        torch.cuda.synchronize()
        np.savez_compressed(os.path.join(args.out, name + ".npz"), **out)
        print(name, F, "crossings", n, "candidate rows", len(out["cand_rows"]), "pairs", n2, flush=True)


if __name__ == "__main__":
    main()
