"""Benchmark of the collision-handling step on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Metric: triangle-steps per second (one triangle carried through one full collision step of
its mesh: tree refit, traversal, continuous narrow phase), batched and served against the
plain per-mesh path, with exact pair sets and p50 / p99 latency.

* ``value`` — batched form: 64 cloth-over-sphere meshes of log-uniform size (1e3..1e5 cloth
  triangles plus a level-5 icosphere each, fp64, about 2.6 M triangles) resident in one
  engine block; one step = one CUDA-graph replay of refit + traversal + continuous narrow
  phase over all meshes (trees built once beforehand); CUDA events around every step, L2
  flushed (256 MiB write) between steps outside the events (inputs are larger than L2 too).
* ``plain`` — the same 64 meshes through the reference-format API one mesh at a time
  (bvh_motion + find_collisions_continuous, as the reference's caller does); its rows and
  times are compared with the batched form's as multisets (``pair_sets_equal``).
* ``served`` — a Poisson stream of impulse-loop requests (rate 2,000/s, meshes of
  log-uniform 2e3..2e5 triangles as in the impulse workload) under a 40 GB engine budget:
  throughput (request triangles over the makespan) and p50 / p99 latency (arrival to result
  on the host).
* ``e2e`` — the batched step through the public engine API from pinned host buffers
  (``engine.StepPipeline``): every step's H2D of both soups of every mesh, the graph replay,
  the rows packed on the device and one D2H copy of every row and time, with each step's
  copies overlapping the neighbouring steps' kernels.
* ``roofline`` — the dominant kernel (CUDA-event timing of the same step run ungraphed)
  against MEASURED_PEAKS.json; ``refit_roofline`` / ``build_roofline`` the tree kernels;
  ``fp64`` the narrow phase's arithmetic rate.
* ``cpu_baseline`` — the oracle (C++ restatement of the reference pipeline, OpenMP) on a
  bounded sample of the batched meshes on the host cores.

Multi-GPU: meshes are independent and the step has no exchange, so N ranks run N replicas
("replicas only"); value is the total over ranks divided by the slowest rank.
``--impl reference`` times the CPU implementation of the path (the oracle) on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from collections import Counter

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "triangle-steps/sec batched+served vs plain (exact pair sets); p50/p99 latency"
UNIT = "triangle-steps/s"
MAXC, MAXCOL = 32, 16            # no candidate overflow on any of the 64 meshes
FP64_PEAK_NOMINAL_GFLOPS = 37000.0   # B200 FP64 datasheet figure (not measured here)
FLOPS_PER_SUBTEST = 252          # coefficients 162 + Cardano and filter 90 (transcendentals as 1)
# DRAM bytes (read + write) of one k_ccd_narrow launch per candidate pair, from ncu's
# dram__bytes_read.sum + dram__bytes_write.sum on the 16-mesh batched step (74.6 MB + 4.8 MB
# for 3,091,227 pairs); the 64-mesh launch is too large for a full capture, so its traffic
# is this figure times its own pair count.
NARROW_DRAM_BYTES_PER_PAIR = (74.574848e6 + 4.76416e6) / 3091227


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--meshes", type=int, default=64)
    ap.add_argument("--served-requests", type=int, default=160)
    ap.add_argument("--served-plain-sample", type=int, default=12)
    ap.add_argument("--served-budget-gb", type=int, default=40,
                    help="device-memory budget of the served engine (the workload's is 40 GB)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    return ap.parse_args()


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while active."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if not self.path or not os.path.exists(self.path):
            return out
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if sm:
            out.update(sm_mhz=statistics.median(sm), sm_max_mhz=max(mx), reasons=sorted(reasons), samples=len(sm))
        return out


def batched_meshes(n):
    from cccollisions_b200 import workloads as W
    return W.batched(n)


def cpu_sample(meshes, seconds):
    """Oracle (C++ restatement of the reference pipeline, all host threads) over the meshes
    in order until `seconds` have passed: (triangle-steps/s, threads, description)."""
    from oracle import oracle as O
    O.build()
    nthreads = O.num_threads()
    tris, done = 0, 0
    t0 = time.perf_counter()
    for x0, x1 in meshes:
        bb, tr = O.bvh(x0, x1)
        O.ccd(bb, tr, x0, x1, nthreads=nthreads)
        tris += x0.shape[0]
        done += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    return tris / dt, nthreads, f"first {done} of the {len(meshes)} batched meshes ({tris} triangles: bvh_motion + " \
                                f"continuous collisions per mesh), {dt:.1f} s"


def refit_bytes(F):
    """Algorithmic bytes of one refit of a motion tree over F fp64 triangles (fp32 boxes)."""
    return F * 2 * 72 + (2 * F - 1) * 24 + 2 * (F - 1) * 24 + (F - 1) * 8


def build_bytes(F):
    """Algorithmic bytes of one motion-tree build (positions, keys, 4 radix passes, topology,
    boxes)."""
    return F * 2 * 72 + F * 8 + 4 * F * 16 + (F - 1) * 12 + (2 * F - 1) * 24 + 2 * (F - 1) * 24


def _ms(rows, times):
    return Counter(zip(map(tuple, np.asarray(rows).tolist()), np.asarray(times, dtype=np.float64).tolist()))


def run_ours(args, rank, world, dev):
    import torch

    import cccollisions_b200 as C
    from cccollisions_b200 import _native as N, api
    from cccollisions_b200.engine import Engine, StepPipeline
    from cccollisions_b200.multi import reduce_max

    meshes = batched_meshes(args.meshes)
    Fs = [x0.shape[0] for x0, _ in meshes]
    total = sum(Fs)
    warm = max(args.warmup, 3)
    stream = torch.cuda.Stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    ev = lambda: torch.cuda.Event(enable_timing=True)

    # ---------------- batched form: resident engine, graph replay
    eng = Engine(tri_capacity=total + 64, mesh_capacity=len(meshes), max_candidates_per_triangle=MAXC,
                 max_collisions_per_triangle=MAXCOL, device=dev)
    sids = [eng.add_mesh(f) for f in Fs]
    for sid, (x0, x1) in zip(sids, meshes):
        eng.upload_soup(sid, x0, x1)
    with torch.cuda.stream(stream):
        eng.set_active(sids)
        eng.build(sids)
        a, b = ev(), ev()
        a.record(stream)
        eng.build(sids)
        b.record(stream)
        stream.synchronize()
        build_ms = a.elapsed_time(b)
        shape = eng.autotune()
        eng.capture(N.ENGINE_OP_CCD, stream=stream)
        for _ in range(warm):
            eng.replay(N.ENGINE_OP_CCD)
        stream.synchronize()
        cnt = eng.counters()
        st = eng.state(sids)
        if world > 1:
            torch.distributed.barrier()
        steps = []
        launches0 = N.kernel_launches()
        with ClockSampler(dev.index if dev.index is not None else 0) as clk:
            for i in range(args.steps):
                flush.fill_(i & 0xFF)
                a, b = ev(), ev()
                a.record(stream)
                eng.replay(N.ENGINE_OP_CCD)
                b.record(stream)
                steps.append((a, b))
            stream.synchronize()
        launches = N.kernel_launches() - launches0
        step_ms = [x.elapsed_time(y) for x, y in steps]
        # per-kernel times of the same step, ungraphed
        N.timing_begin()
        for _ in range(3):
            eng.ccd()
        kern = N.timing_end()
        stream.synchronize()
    total_ms = reduce_max(sum(step_ms), dev)          # the slowest replica
    ms_per_step = total_ms / args.steps
    value = world * total * args.steps / (total_ms / 1e3)
    batched_rows = {sid: _ms(*[x.cpu().numpy() for x in eng.collisions(sid, int(n))]) for sid, n in
                    zip(sids, st["rows"])}

    # ---------------- e2e through the engine API from pinned host memory: StepPipeline streams
    # the steps, so step k's soups go up and step k-1's rows come down while step k runs;
    # every step's copies are inside the timed region
    nrow = [int(n) for n in st["rows"]]
    hx = [(torch.from_numpy(x0).pin_memory(), torch.from_numpy(x1).pin_memory()) for x0, x1 in meshes]
    pipe = StepPipeline(eng, sids)
    houts = [pipe.host_outputs(), pipe.host_outputs()]
    pipe.run([hx] * warm, [houts[k % 2] for k in range(warm)])
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    e2e_totals = pipe.run([hx] * args.steps, [houts[k % 2] for k in range(args.steps)])
    torch.cuda.synchronize(dev)
    e2e_ms = reduce_max((time.perf_counter() - t0) * 1e3 / args.steps, dev)
    # the streamed rows of the last step, split by mesh, are the batched step's rows
    rows_h, times_h, meta_h = [o.numpy() for o in houts[(args.steps - 1) % 2]]
    M = len(sids)
    e2e_equal = all(_ms(rows_h[meta_h[m]:meta_h[m + 1]], times_h[meta_h[m]:meta_h[m + 1]]) ==
                    batched_rows[int(meta_h[M + 1 + m])] for m in range(M))
    e2e_equal &= all(t == sum(nrow) for t in e2e_totals)
    h2d = sum(x0.nbytes + x1.nbytes for x0, x1 in meshes)
    d2h = sum(n * 32 for n in nrow) + 4 * (2 * len(sids) + 2)

    # ---------------- plain per-mesh path through the reference-format API
    X = [(torch.from_numpy(x0).to(dev), torch.from_numpy(x1).to(dev)) for x0, x1 in meshes]
    api.CHECK_STATUS = True
    plain_out = None

    def plain():
        out = []
        for X0, X1 in X:
            bb, tr = C.bvh_motion(X0[None], X1[None])
            out.append(C.find_collisions_continuous(bb, tr, X0[None], X1[None], MAXC, MAXCOL))
        return out

    torch.cuda.synchronize(dev)
    for _ in range(warm):
        plain_out = plain()
    torch.cuda.synchronize(dev)
    pms = []
    for i in range(args.steps):
        flush.fill_(i & 0xFF)
        torch.cuda.synchronize(dev)
        a, b = ev(), ev()
        a.record()
        plain_out = plain()
        b.record()
        torch.cuda.synchronize(dev)
        pms.append(a.elapsed_time(b))
    plain_ms = statistics.mean(pms)
    equal = True
    for sid, (rows, times) in zip(sids, plain_out):
        r = rows[0].cpu().numpy()
        k = int((r[:, 0] >= 0).sum())
        equal &= _ms(r[:k], times[0, :k, 0].cpu().numpy()) == batched_rows[sid]

    # ---------------- rooflines
    peak, peak_kind = load_peaks()
    dname, (dms, dcount) = max(kern.items(), key=lambda kv: kv[1][0])
    per_launch = dms / dcount
    narrow_bytes = cnt["candidates"] * (8 + 2 * 2 * 72) + int(sum(nrow)) * 32
    achieved = narrow_bytes / (per_launch / 1e3) / 1e9 if dname == "k_ccd_narrow" else None
    # the refit is two passes (block-local, then the climbs that leave a block)
    r1 = kern.get("k_engine_refit", (float("nan"), 1))
    r2 = kern.get("k_engine_refit_front", (0.0, 1))
    refit_ms = r1[0] / r1[1] + r2[0] / r2[1]
    rb = sum(refit_bytes(f) for f in Fs)
    bb_ = sum(build_bytes(f) for f in Fs)
    fp64_gflops = cnt["subtests"] * FLOPS_PER_SUBTEST / (kern["k_ccd_narrow"][0] / kern["k_ccd_narrow"][1] / 1e3) / 1e9
    eng.close()

    result = None
    if rank == 0:
        clocks = clk.summary()
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": warm,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded cloth grids + icospheres)",
            "config": {"workload": f"batched: {len(meshes)} cloth+icosphere meshes, log-uniform 1e3..1e5 cloth "
                                   f"triangles + 20,480 sphere triangles each, one CUDA-graph replay per step",
                       "triangles": total, "meshes": len(meshes), "max_candidates_per_triangle": MAXC,
                       "max_collisions_per_triangle": MAXCOL, "positions": "fp64", "tree_boxes": "fp32",
                       "l2": "flushed between steps (256 MiB write); inputs (377 MB) larger than L2",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "autotuned_shape": shape, "candidates": cnt["candidates"], "subtests": cnt["subtests"],
                       "roots_in_unit_interval": cnt["roots"], "collision_rows": int(sum(nrow)),
                       "status": cnt["status"]},
            "plain": {"value": world * total / (plain_ms / 1e3), "unit": UNIT, "ms_per_step": plain_ms,
                      "path": "per mesh: bvh_motion + find_collisions_continuous (reference-format API)"},
            "batched_over_plain": plain_ms / ms_per_step,
            "pair_sets_equal": bool(equal),
            "e2e": {"value": world * total / (e2e_ms / 1e3), "unit": UNIT, "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "path": "engine.StepPipeline: per step, H2D of both soups of every mesh from page-locked "
                            "memory, graph replay, device packing of the rows, D2H of rows + times; copies of "
                            "step k overlap the kernels of steps k-1 / k+1",
                    "rows_equal_batched": bool(e2e_equal)},
            "roofline": {"kernel": dname, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                         "traffic": (NARROW_DRAM_BYTES_PER_PAIR * cnt["candidates"]) if dname == "k_ccd_narrow"
                         else None,
                         "traffic_source": "ncu DRAM bytes per candidate pair of the 16-mesh capture, times this "
                                           "launch's pairs",
                         "alg_bytes_per_launch": narrow_bytes, "launch_ms": per_launch,
                         "note": "the narrow phase is FP64-latency bound; see fp64"},
            "fp64": {"kernel": "k_ccd_narrow", "achieved_gflops": fp64_gflops,
                     "peak_gflops": FP64_PEAK_NOMINAL_GFLOPS, "peak_source": "nominal (B200 datasheet)",
                     "frac": fp64_gflops / FP64_PEAK_NOMINAL_GFLOPS, "flops_per_subtest": FLOPS_PER_SUBTEST},
            "refit_roofline": {"kernel": "k_engine_refit + k_engine_refit_front", "bound": "hbm", "alg_bytes": rb, "launch_ms": refit_ms,
                               "achieved": rb / (refit_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                               "frac": rb / (refit_ms / 1e3) / 1e9 / peak},
            "build_roofline": {"kernels": "bounds, Morton, radix sort, Karras, refit", "bound": "hbm",
                               "alg_bytes": bb_, "ms": build_ms, "achieved": bb_ / (build_ms / 1e3) / 1e9,
                               "peak": peak, "unit": "GB/s", "frac": bb_ / (build_ms / 1e3) / 1e9 / peak},
            "kernel_ms_per_step": {k: v[0] / v[1] for k, v in kern.items()},
            "kernel_share": {k: round(v[0] / sum(x[0] for x in kern.values()), 4) for k, v in kern.items()},
            "gpu_launches": int(launches),
            "clocks": {"sm_mhz": clocks["sm_mhz"], "sm_max_mhz": clocks["sm_max_mhz"], "reasons": clocks["reasons"]},
        }
    return result, meshes


def plain_loop(r, dev, max_iter=50):
    """One impulse-loop request through the reference-format API, as a caller of the reference
    writes it: per iteration bvh_motion + compute_impulses on the soups, then each vertex moves
    by the average correction of its corners (torch index_add).  Returns iterations."""
    import torch

    import cccollisions_b200 as C
    faces = torch.from_numpy(r.faces.astype(np.int64)).to(dev)
    v0 = torch.from_numpy(r.verts0).to(dev)
    v1 = torch.from_numpy(r.verts1).to(dev).clone()
    vel = torch.from_numpy(r.vel).to(dev).clone()
    m = torch.from_numpy(r.masses).to(dev)[None].contiguous()
    x0 = v0[faces][None].contiguous()
    idx = faces.reshape(-1)
    V = v0.shape[0]
    for it in range(max_iter):
        x1 = v1[faces][None].contiguous()
        bb, tr = C.bvh_motion(x0, x1)
        dv, dx, cnt = C.compute_impulses(bb, tr, x0, x1, m, MAXC, MAXCOL)
        c = cnt[0].reshape(-1).to(v1.dtype)
        if float(c.sum()) == 0:
            return it
        sc = torch.zeros(V, dtype=v1.dtype, device=dev).index_add_(0, idx, c)
        sdx = torch.zeros((V, 3), dtype=v1.dtype, device=dev).index_add_(0, idx, dx[0].reshape(-1, 3))
        sdv = torch.zeros((V, 3), dtype=v1.dtype, device=dev).index_add_(0, idx, dv[0].reshape(-1, 3))
        w = torch.where(sc > 0, 1.0 / sc.clamp(min=1), torch.zeros_like(sc))[:, None]
        v1 += sdx * w
        vel += sdv * w
    return max_iter


def run_served(args, dev):
    import torch

    from cccollisions_b200 import workloads as W
    from cccollisions_b200.serve import Request, Server, requests_from_stream
    reqs = requests_from_stream(W.served_stream(num_requests=args.served_requests, rate=2000.0))
    srv = Server(budget_bytes=args.served_budget_gb << 30, device=dev)
    for r in reqs:
        srv._pin(r)
    st = srv.run(reqs)
    srv.close()
    # the same sample of requests (every k-th by arrival, so all sizes are represented) through
    # the engine (all admitted at once) and through the plain per-request path
    k = max(1, len(reqs) // max(1, args.served_plain_sample))
    sample = reqs[::k][:max(1, args.served_plain_sample)]
    copies = [Request(r.verts0, r.verts1, r.vel, r.faces, r.masses, rid=r.rid) for r in sample]
    srv = Server(budget_bytes=args.served_budget_gb << 30, device=dev)
    for r in copies:
        srv._pin(r)
    same = srv.run(copies, realtime=False)
    srv.close()
    plain_loop(sample[0], dev, 2)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    its = [plain_loop(r, dev) for r in sample]
    torch.cuda.synchronize(dev)
    dt = time.perf_counter() - t0
    ptris = sum(r.F for r in sample)
    return {"value": st["throughput"], "unit": UNIT, "requests": st["requests"], "rate_per_s": 2000.0,
            "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"], "makespan_s": st["makespan_s"],
            "request_triangles": st["triangles"], "ticks": st["ticks"], "mean_iterations": st["mean_iterations"],
            "converged_fraction": st["converged"], "budget_gb": args.served_budget_gb,
            "policy": f"FIFO admission, at most {srv.max_active_triangles} active triangles (a request alone is "
                      "always admitted)",
            "request": "impulse loop (max 50 iterations) on an impulse-workload mesh of log-uniform 2e3..2e5 "
                       "triangles, fp64",
            "same_set": {"requests": len(sample), "triangles": ptris,
                         "engine": {"value": same["throughput"], "seconds": same["makespan_s"],
                                    "mean_iterations": same["mean_iterations"]},
                         "plain": {"value": ptris / dt, "seconds": dt, "mean_iterations": float(np.mean(its)),
                                   "path": "per request, one after another: bvh_motion + compute_impulses per "
                                           "iteration, per-vertex averaging with torch"}}}


def run_reference(args):
    meshes = batched_meshes(args.meshes)
    per = max(1.0, args.cpu_seconds / max(args.steps + args.warmup, 1))
    vals = []
    desc, threads = "", 0
    for i in range(args.warmup + args.steps):
        v, threads, desc = cpu_sample(meshes, per)
        if i >= args.warmup:
            vals.append(v)
    v = statistics.median(vals)
    return {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sum(x0.shape[0] for x0, _ in meshes) / v * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded cloth grids + icospheres)",
            "config": {"workload": f"batched: {len(meshes)} cloth+icosphere meshes (CPU sample per step)",
                       "triangles": sum(x0.shape[0] for x0, _ in meshes)},
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"per step: {desc}"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)))
        return
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    try:
        res, meshes = run_ours(args, rank, world, dev)
        if world > 1:
            torch.distributed.barrier()
        if rank == 0:
            if world == 1 and args.served_requests > 0:
                res["served"] = run_served(args, dev)
                ss = res["served"]["same_set"]
                res["served_over_plain"] = ss["engine"]["value"] / ss["plain"]["value"]
            if world == 1:
                v, threads, desc = cpu_sample(meshes, args.cpu_seconds)
                res["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc}
            print(json.dumps(res))
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
