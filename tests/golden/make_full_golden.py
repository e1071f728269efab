"""Full-size golden fixtures from the reference extension itself, on a GPU.

    python oracle/build_ref.py --src <reference checkout>     # where the reference sources are
    python tests/golden/make_full_golden.py [--out DIR]        # on a machine with a CUDA GPU

Runs the reference's query calls (oracle/_ref/cccollisions.so) at the measured workloads' full
sizes and records what a test needs to pin the default (reference-math) mode there:

* ``full_cloth_sphere.npz`` — the cloth-over-sphere CCD step (52,738 fp64 triangles):
  every row and time of ``find_collisions_continuous(.., 16, 16)``, plus the digest and row
  count of ``find_collisions_continuous_partial`` under a seeded 30 % mask;
* ``full_impulse_fold.npz`` — one ``compute_impulses(.., 32, 16)`` call on the folded
  256x256 cloth (130,050 fp64 triangles, 21.3 candidates per triangle, so 32 candidates
  per triangle leave no wrap-around): every corner counter, dv / dx at 16,384 seeded
  contact corners, and the column sums of dv and dx;
* ``full_batched.npz`` — the 64 batched cloth+sphere meshes (2.62 M triangles): per mesh
  the row count and the digest of ``find_collisions_continuous`` with 16 or 32 candidates
  per triangle (whichever holds every candidate pair);
* ``full_report.json`` — the same calls through this library's default mode (reference-
  format API and, for the batched meshes, the resident engine) compared with the
  reference: rows only on one side, times bit-equal, dv / dx error.

A digest is the SHA-256 of the rows sorted with their times (int64 i, j, k and the time's
IEEE bits): equal digests mean equal row multisets with bit-equal times.

Trees fed to the reference come from the CPU oracle in the reference's order (its own
bvh() is not run: see make_golden.py).  Every call is checked on the CPU first: F >= 2,
tree depth far below the 64-entry stack, candidate pairs within the capacity.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

MASK_SEED = 5          # the partial call's mask: rng(MASK_SEED).random(F) < 0.3
SAMPLE_SEED = 6        # the corners whose dv / dx are stored
SAMPLE = 16384


def input_digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def canonical_rows(rows, times):
    """(N, 3) rows and (N,) times sorted by (i, j, k, time bits): int64 (N, 4)."""
    r = np.asarray(rows, dtype=np.int64).reshape(-1, 3)
    tb = np.asarray(times, dtype=np.float64).reshape(-1).view(np.int64)
    o = np.lexsort((tb, r[:, 2], r[:, 1], r[:, 0]))
    return np.concatenate([r[o], tb[o, None]], axis=1)


def row_digest(rows, times) -> str:
    return hashlib.sha256(np.ascontiguousarray(canonical_rows(rows, times)).tobytes()).hexdigest()


def partial_mask(F):
    return np.random.default_rng(MASK_SEED).random(F) < 0.3


def sample_corners(cnt):
    nz = np.flatnonzero(np.asarray(cnt).reshape(-1) > 0)
    g = np.random.default_rng(SAMPLE_SEED)
    k = min(SAMPLE, nz.size)
    return np.sort(g.choice(nz, size=k, replace=False))


def compare(ref_rows, ref_times, got_rows, got_times):
    from collections import Counter
    a = Counter(map(tuple, canonical_rows(ref_rows, ref_times)[:, :3].tolist()))
    b = Counter(map(tuple, canonical_rows(got_rows, got_times)[:, :3].tolist()))
    res = {"reference_rows": int(len(ref_rows)), "rows": int(len(got_rows)),
           "only_reference": int(sum((a - b).values())), "only_here": int(sum((b - a).values())),
           "digest_equal": row_digest(ref_rows, ref_times) == row_digest(got_rows, got_times)}
    ex = list((a - b).elements())[:5] + list((b - a).elements())[:5]
    if ex:
        res["examples"] = [list(map(int, e)) for e in ex]
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "golden_out"))
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)

    import torch

    import cccollisions_b200 as C
    from cccollisions_b200 import _native as N, workloads as W
    from cccollisions_b200.engine import Engine
    from make_golden import load_reference, tree_depth
    from oracle import oracle as O
    O.build()
    R = load_reference()
    dev = torch.device("cuda:0")
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    assert N.lib().ccc_get_math_library() == N.LIB_REFERENCE
    report = {}

    def tree(x0, x1):
        bb, tr = O.bvh(x0, x1)
        assert x0.shape[0] >= 2 and tree_depth(tr) <= 48
        return bb, tr

    def valid(rows, times):
        r = rows[0].cpu().numpy()
        n = int((r[:, 0] >= 0).sum())
        assert (r[n:] == -1).all()
        return r[:n], times[0, :n, 0].cpu().numpy().astype(np.float64)

    # ------------------------------------------------------------ cloth over sphere
    x0, x1 = W.cloth_sphere()
    x0, x1 = x0[0], x1[0]
    F = x0.shape[0]
    bb, tr = tree(x0, x1)
    assert len(O.candidates(bb, tr, nthreads=0)) <= 16 * F
    Bb, Tr, X0, X1 = T(bb[None]), T(tr[None]), T(x0[None]), T(x1[None])
    rr, rt = valid(*R.find_collisions_continuous(Bb, Tr, X0, X1, 16, 16))
    mask = partial_mask(F)
    pr, pt = valid(*R.find_collisions_continuous_partial(Bb, Tr, X0, X1, T(mask[None]), 16, 16))
    torch.cuda.synchronize()
    can = canonical_rows(rr, rt)
    np.savez_compressed(os.path.join(args.out, "full_cloth_sphere.npz"), input_digest=input_digest(x0, x1),
                        rows=can[:, :3].astype(np.int32), times=can[:, 3].view(np.float64),
                        digest=row_digest(rr, rt), partial_rows=len(pr), partial_digest=row_digest(pr, pt))
    gr, gt = valid(*C.find_collisions_continuous(Bb, Tr, X0, X1, 16, 16))
    gpr, gpt = valid(*C.find_collisions_continuous_partial(Bb, Tr, X0, X1, T(mask[None]), 16, 16))
    report["cloth_sphere"] = {"F": F, "ccd": compare(rr, rt, gr, gt), "ccd_partial": compare(pr, pt, gpr, gpt)}
    print(json.dumps(report["cloth_sphere"]), flush=True)

    # ------------------------------------------------------------ folded cloth impulses
    x0, x1, m = W.impulse_fold()
    x0, x1, m = x0[0], x1[0], m[0]
    F = x0.shape[0]
    bb, tr = tree(x0, x1)
    assert len(O.candidates(bb, tr, nthreads=0)) <= 32 * F
    Bb, Tr, X0, X1, M = T(bb[None]), T(tr[None]), T(x0[None]), T(x1[None]), T(m[None])
    dv, dx, cnt = R.compute_impulses(Bb, Tr, X0, X1, M, 32, 16)
    dv, dx, cnt = dv[0].cpu().numpy(), dx[0].cpu().numpy(), cnt[0].cpu().numpy()
    assert int(cnt.sum()) // 4 <= 16 * F
    idx = sample_corners(cnt)
    dvf, dxf = dv.reshape(-1, 3), dx.reshape(-1, 3)
    np.savez_compressed(os.path.join(args.out, "full_impulse_fold.npz"), input_digest=input_digest(x0, x1, m),
                        cnt=cnt.astype(np.int32), corners=idx.astype(np.int32), dv=dvf[idx], dx=dxf[idx],
                        dv_sum=dvf.sum(axis=0), dx_sum=dxf.sum(axis=0), dv_abs_sum=np.abs(dvf).sum(axis=0),
                        dx_abs_sum=np.abs(dxf).sum(axis=0))
    gdv, gdx, gcnt = C.compute_impulses(Bb, Tr, X0, X1, M, 32, 16)
    gdv, gdx, gcnt = gdv[0].cpu().numpy(), gdx[0].cpu().numpy(), gcnt[0].cpu().numpy()
    scale = lambda a: max(float(np.abs(a).max()), 1e-300)
    report["impulse_fold"] = {"F": F, "contacts": int(cnt.sum()) // 4, "corners_with_contacts": int((cnt > 0).sum()),
                              "counters_equal": bool((gcnt == cnt).all()),
                              "counters_differing": int((gcnt != cnt).sum()),
                              "dv_max_abs_err_over_max": float(np.abs(gdv - dv).max() / scale(dv)),
                              "dx_max_abs_err_over_max": float(np.abs(gdx - dx).max() / scale(dx))}
    print(json.dumps(report["impulse_fold"]), flush=True)

    # ------------------------------------------------------------ the 64 batched meshes
    meshes = W.batched()
    Fs = [a.shape[0] for a, _ in meshes]
    counts, digests, maxcs, ins = [], [], [], []
    ref_sets, tref = [], 0.0
    for a, b in meshes:
        f = a.shape[0]
        bb, tr = tree(a, b)
        nc = len(O.candidates(bb, tr, nthreads=0))
        maxc = 16 if nc <= 16 * f else 32
        assert nc <= maxc * f
        Bb, Tr, A, Bx = T(bb[None]), T(tr[None]), T(a[None]), T(b[None])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r, t = valid(*R.find_collisions_continuous(Bb, Tr, A, Bx, maxc, 16))
        tref += time.perf_counter() - t0
        assert len(r) < 16 * f
        counts.append(len(r))
        digests.append(row_digest(r, t))
        maxcs.append(maxc)
        ins.append(input_digest(a, b))
        ref_sets.append((r, t))
    np.savez_compressed(os.path.join(args.out, "full_batched.npz"), F=np.array(Fs), rows=np.array(counts),
                        digests=np.array(digests), maxc=np.array(maxcs), input_digests=np.array(ins))
    # this library: the resident engine (the batched step) and the reference-format API
    eng = Engine(tri_capacity=sum(Fs) + 64, mesh_capacity=len(meshes), max_candidates_per_triangle=32,
                 max_collisions_per_triangle=16, device=dev)
    sids = [eng.add_mesh(f) for f in Fs]
    for sid, (a, b) in zip(sids, meshes):
        eng.upload_soup(sid, a, b)
    eng.set_active(sids)
    eng.build(sids)
    eng.ccd()
    st = eng.state(sids)
    eng_cmp, api_cmp = [], []
    for i, (sid, (a, b)) in enumerate(zip(sids, meshes)):
        er, et = [x.cpu().numpy() for x in eng.collisions(sid, int(st["rows"][i]))]
        eng_cmp.append(compare(*ref_sets[i], er, et))
        A, Bx = T(a[None]), T(b[None])
        bb, tr = C.bvh_motion(A, Bx)
        api_cmp.append(compare(*ref_sets[i], *valid(*C.find_collisions_continuous(bb, tr, A, Bx, 32, 16))))
    eng.close()
    report["batched"] = {"meshes": len(meshes), "triangles": int(sum(Fs)), "reference_rows": int(sum(counts)),
                         "reference_seconds_all_meshes_first_pass": tref,
                         "engine_digests_equal": sum(c["digest_equal"] for c in eng_cmp),
                         "api_digests_equal": sum(c["digest_equal"] for c in api_cmp),
                         "engine_rows_only_reference": sum(c["only_reference"] for c in eng_cmp),
                         "engine_rows_only_here": sum(c["only_here"] for c in eng_cmp),
                         "api_rows_only_reference": sum(c["only_reference"] for c in api_cmp),
                         "api_rows_only_here": sum(c["only_here"] for c in api_cmp),
                         "differing_meshes": [dict(mesh=i, **c) for i, c in enumerate(api_cmp) if not c["digest_equal"]]}
    print(json.dumps(report["batched"])[:3000], flush=True)
    json.dump(report, open(os.path.join(args.out, "full_report.json"), "w"), indent=1, default=float)


if __name__ == "__main__":
    main()
