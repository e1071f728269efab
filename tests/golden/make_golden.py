"""Generate golden fixtures by running the reference extension itself on a GPU.

    python oracle/build_ref.py            # here, where the reference sources are
    python tests/golden/make_golden.py [--out DIR]   # on a machine with a CUDA GPU

Loads the reference extension compiled by oracle/build_ref.py (oracle/_ref/cccollisions.so),
runs its query and impulse functions on seeded inputs, and writes one compressed .npz per
case (inputs + reference outputs) plus ``report.json`` comparing the reference with the
CPU oracle on full-size workloads.

Safety: every call is checked on the CPU first (oracle counts against the output
capacities, F >= 2, tree depth far below the 64-entry traversal stack), and only valid
rows are passed to compute_impulses_from_collisions (the reference reads out of bounds on
-1 rows).  The reference's own bvh()/bvh_motion() are NOT run: their split search
(build_bvh.cu:117-123) leaves its loop only through signed 32-bit overflow followed by an
integer division by zero, which a current compiler may turn into an endless loop on the
GPU.  The trees fed to the reference are built by the oracle in the reference's order.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def load_reference():
    """The reference extension built by oracle/build_ref.py, loaded from its file (this
    repository's own ``cccollisions`` package has the same module name)."""
    import importlib.util

    import torch  # noqa: F401  (loads libtorch for the extension)
    spec = importlib.util.spec_from_file_location("cccollisions", os.path.join(ROOT, "oracle", "_ref",
                                                                                "cccollisions.so"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def tree_depth(tr):
    n = (tr.shape[0] + 1) // 2
    depth = 0
    st = [(0, 1)]
    while st:
        k, d = st.pop()
        depth = max(depth, d)
        if k < n - 1:
            st.append((int(tr[k, 1]), d + 1))
            st.append((int(tr[k, 2]), d + 1))
    return depth


def valid(rows):
    return rows[rows[:, 0] >= 0]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "golden_out"))
    ap.add_argument("--full", action="store_true", help="also compare full-size workloads (report only)")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)

    import torch
    from cccollisions_b200 import workloads as W
    from oracle import oracle as O
    O.build()
    R = load_reference()
    dev = torch.device("cuda:0")
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    report = {"cases": {}}

    def safe_tree(x0, x1=None):
        bb, tr = O.bvh(x0, x1)
        assert x0.shape[0] >= 2
        assert tree_depth(tr) <= 48
        return bb, tr

    # ---------------------------------------------------------------- small random soups
    for seed, dtype in ((20, np.float64), (21, np.float64), (22, np.float32), (23, np.float64)):
        x0, x1, m = W.jittered_fold(seed, 14, 12, dtype=dtype)
        F = x0.shape[0]
        bb, tr = safe_tree(x0, x1)
        mask = np.random.default_rng(seed).random(F) < 0.4
        cand = O.candidates(bb, tr)
        assert len(cand) <= 16 * F
        bbs, trs = safe_tree(x0)
        out = {"x0": x0, "x1": x1, "masses": m, "mask": mask}
        Bb, Tr, X0, X1, M = T(bb[None]), T(tr[None]), T(x0[None]), T(x1[None]), T(m[None])
        rows, times = R.find_collisions_continuous(Bb, Tr, X0, X1, 16, 16)
        r = rows[0].cpu().numpy()
        n = int((r[:, 0] >= 0).sum())
        out["ccd_rows"], out["ccd_times"] = r[:n], times[0, :n, 0].cpu().numpy()
        rows, times = R.find_collisions_continuous_partial(Bb, Tr, X0, X1, T(mask[None]), 16, 16)
        r = rows[0].cpu().numpy()
        n2 = int((r[:, 0] >= 0).sum())
        out["ccdp_rows"], out["ccdp_times"] = r[:n2], times[0, :n2, 0].cpu().numpy()
        mc = R.find_mincol_cand(Bb, Tr, X0, X1, 16)
        out["mincol_rows"] = valid(mc[0].cpu().numpy())
        dv, dx, cnt = R.compute_impulses(Bb, Tr, X0, X1, M, 16, 16)
        out["imp_dv"], out["imp_dx"], out["imp_cnt"] = dv[0].cpu().numpy(), dx[0].cpu().numpy(), cnt[0].cpu().numpy()
        dv, dx, cnt = R.compute_impulses_partial(Bb, Tr, X0, X1, M, T(mask[None]), 16, 16)
        out["impp_dv"], out["impp_dx"], out["impp_cnt"] = dv[0].cpu().numpy(), dx[0].cpu().numpy(), cnt[0].cpu().numpy()
        if n > 0:
            dv, dx, cnt = R.compute_impulses_from_collisions(T(out["ccd_rows"][None]), T(out["ccd_times"][None, :, None]),
                                                             X0, X1, M)
            out["impr_dv"], out["impr_dx"], out["impr_cnt"] = (dv[0].cpu().numpy(), dx[0].cpu().numpy(),
                                                               cnt[0].cpu().numpy())
        Bs, Ts = T(bbs[None]), T(trs[None])
        for th in (0.0, 0.005):
            c = R.find_collisions(Bs, Ts, X0, th, 16)
            out[f"static_{th}"] = valid(c[0].cpu().numpy())
        pr, _ = O.proximity(bbs, trs, x0, 0.02)
        assert len(pr) <= 16 * F
        (p,) = R.find_proximity(Bs, Ts, X0, 0.02, 16)
        out["prox_rows"] = valid(p[0].cpu().numpy())
        torch.cuda.synchronize()
        name = f"soup_{seed}_{np.dtype(dtype).name}"
        np.savez_compressed(os.path.join(args.out, name + ".npz"), **out)
        report["cases"][name] = {"F": F, "ccd_rows": n, "ccd_partial_rows": n2, "mincol": len(out["mincol_rows"]),
                                 "static": len(out["static_0.0"]), "prox": len(out["prox_rows"]),
                                 "contacts": int(out["imp_cnt"].sum() // 4)}

    # ---------------------------------------------------------------- small cloth over sphere
    x0, x1 = W.cloth_sphere(seed=7, nx=24, ny=24, level=2)
    x0, x1 = x0[0], x1[0]
    F = x0.shape[0]
    m = np.ones((F, 3))
    bb, tr = safe_tree(x0, x1)
    assert len(O.candidates(bb, tr)) <= 16 * F
    Bb, Tr, X0, X1, M = T(bb[None]), T(tr[None]), T(x0[None]), T(x1[None]), T(m[None])
    rows, times = R.find_collisions_continuous(Bb, Tr, X0, X1, 16, 16)
    r = rows[0].cpu().numpy()
    n = int((r[:, 0] >= 0).sum())
    dv, dx, cnt = R.compute_impulses(Bb, Tr, X0, X1, M, 16, 16)
    np.savez_compressed(os.path.join(args.out, "cloth_sphere_small.npz"), x0=x0, x1=x1, masses=m, ccd_rows=r[:n],
                        ccd_times=times[0, :n, 0].cpu().numpy(), imp_dv=dv[0].cpu().numpy(),
                        imp_dx=dx[0].cpu().numpy(), imp_cnt=cnt[0].cpu().numpy())
    report["cases"]["cloth_sphere_small"] = {"F": F, "ccd_rows": n}

    # ---------------------------------------------------------------- static fold (fp32)
    x = W.static_fold()[0]
    F = x.shape[0]
    bb, tr = safe_tree(x)
    Bb, Tr, X = T(bb[None]), T(tr[None]), T(x[None])
    out = {"x": x}
    for th in (0.0, 0.005):
        assert len(O.candidates(bb, tr, threshold=th)) <= 16 * F
        c = R.find_collisions(Bb, Tr, X, th, 16)
        out[f"static_{th}"] = valid(c[0].cpu().numpy())
    pr, _ = O.proximity(bb, tr, x, 0.002)
    if len(pr) <= 16 * F:
        (p,) = R.find_proximity(Bb, Tr, X, 0.002, 16)
        out["prox_rows"] = valid(p[0].cpu().numpy())
    np.savez_compressed(os.path.join(args.out, "static_fold.npz"), **out)
    report["cases"]["static_fold"] = {"F": F, "static": len(out["static_0.0"])}

    # ---------------------------------------------------------------- full-size comparisons
    if args.full:
        full = {}
        x0, x1 = W.cloth_sphere()
        x0, x1 = x0[0], x1[0]
        F = x0.shape[0]
        bb, tr = safe_tree(x0, x1)
        assert len(O.candidates(bb, tr, nthreads=0)) <= 16 * F
        Bb, Tr, X0, X1 = T(bb[None]), T(tr[None]), T(x0[None]), T(x1[None])
        t0 = time.perf_counter()
        rows, times = R.find_collisions_continuous(Bb, Tr, X0, X1, 16, 16)
        torch.cuda.synchronize()
        tref = time.perf_counter() - t0
        r = rows[0].cpu().numpy()
        n = int((r[:, 0] >= 0).sum())
        rr, rt = r[:n], times[0, :n, 0].cpu().numpy()
        er, et = O.ccd(bb, tr, x0, x1, nthreads=0)
        full["cloth_sphere"] = compare_rows(rr, rt, er, et)
        full["cloth_sphere"]["reference_seconds_first_call"] = tref
        np.savez_compressed(os.path.join(args.out, "cloth_sphere_full_reference.npz"), rows=rr, times=rt)
        report["full"] = full
    json.dump(report, open(os.path.join(args.out, "report.json"), "w"), indent=1, default=float)
    print(json.dumps(report, default=float)[:2000])


def compare_rows(rr, rt, er, et):
    from collections import Counter
    ref = Counter((tuple(a), ) for a in rr.tolist())
    orc = Counter((tuple(a), ) for a in er.tolist())
    only_ref = ref - orc
    only_orc = orc - ref
    res = {"reference_rows": int(len(rr)), "oracle_rows": int(len(er)), "only_reference": int(sum(only_ref.values())),
           "only_oracle": int(sum(only_orc.values()))}
    # time differences of rows present once on both sides
    dr = {tuple(a): t for a, t in zip(rr.tolist(), rt.tolist())}
    de = {tuple(a): t for a, t in zip(er.tolist(), et.tolist())}
    common = [k for k in dr if k in de]
    if common:
        d = np.array([abs(dr[k] - de[k]) / max(abs(de[k]), 1e-12) for k in common])
        res["toi_max_rel_diff_common"] = float(d.max())
        res["toi_bit_equal_fraction"] = float(np.mean([dr[k] == de[k] for k in common]))
    res["examples_only_reference"] = [list(k[0]) for k in list(only_ref)[:10]]
    res["examples_only_oracle"] = [list(k[0]) for k in list(only_orc)[:10]]
    return res


if __name__ == "__main__":
    main()
