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
* ``query`` / ``reference_gpu`` — find_collisions_continuous alone per mesh on the same
  prebuilt reference-order trees: this library's, and the reference extension's own CUDA
  path (compiled unmodified from its sources into oracle/_ref; a baseline leg, like
  ``cpu_baseline``), whose rows are compared with the batched form's.  The reference's
  bvh_motion is not run: its split search can loop without end on a GPU.
* ``served`` — a Poisson stream of impulse-loop requests (rate 2,000/s, meshes of
  log-uniform 2e3..2e5 triangles as in the impulse workload) under a 40 GB engine budget:
  throughput (request triangles over the makespan) and p50 / p99 latency (arrival to result
  on the host).  ``served_separated``: the same stream of folds whose layers start apart
  (``workloads.SEPARATED_FOLD``), where the loop runs until no pair collides.
* ``e2e`` — the batched step through the public engine API from pinned host buffers
  (``engine.StepPipeline``): every step's H2D of both soups of every mesh, the graph replay,
  the rows packed on the device and one D2H copy of every row and time, with each step's
  copies overlapping the neighbouring steps' kernels.
* ``roofline`` — the dominant kernel (CUDA-event timing of the same step run ungraphed)
  against MEASURED_PEAKS.json; ``refit_roofline`` / ``build_roofline`` the tree kernels;
  ``fp64`` the narrow kernel's arithmetic rate over the sub-tests it solves, and
  ``narrow_phase`` the staging and narrow kernels together over every sub-test (a repeated
  sub-test is solved once for all the pairs that have it).
* ``cpu_baseline`` — the oracle (C++ restatement of the reference pipeline, OpenMP) on a
  bounded sample of the batched meshes on the host cores.

Multi-GPU: meshes are independent and the step has no exchange, so N ranks run N replicas
("replicas only"); value is the total over ranks divided by the slowest rank.
``--impl reference`` times the CPU implementation of the path (the oracle) on rank 0 only,
whole steps over every mesh of the same workload.
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
# DRAM bytes (read + write) of one k_ccd_narrow launch per sub-test solved, from ncu's
# dram__bytes_read.sum + dram__bytes_write.sum on the 32-mesh batched step; the 64-mesh
# launch is too large for a full capture, so its traffic is this figure times its own count.
NARROW_DRAM_BYTES_PER_SOLVED = (239520768 + 57656064) / 11536974
# the kernels of the narrow phase: staging (masks, solver choice), then the solves
NARROW_PHASE = ("k_ccd_stage_mask", "k_ccd_stage_pending", "k_ccd_narrow")


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
    """nvidia-smi clocks and throttle reasons sampled every 20 ms while active; entering
    waits (up to 3 s) for the first sample, so that sampling covers the timed region that
    follows."""

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
                 "-lms", "20"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        t0 = time.perf_counter()
        while self.proc is not None and time.perf_counter() - t0 < 3.0 and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.01)
        self.start_lines = self._lines()
        return self

    def _lines(self):
        try:
            with open(self.path) as f:
                return sum(1 for _ in f)
        except OSError:
            return 0

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
        # the samples taken after the timed region began (the first ones came before it)
        lines = open(self.path).read().splitlines()
        if len(lines) > getattr(self, "start_lines", 0):
            lines = lines[getattr(self, "start_lines", 0):]
        for line in lines:
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


def workload_config(meshes, world):
    """The workload, identical on both arms (no results in it)."""
    return {"workload": f"batched CCD: {len(meshes)} cloth+icosphere meshes (1e3..1e5 cloth tris + 20,480 sphere "
                        f"tris each)",
            "triangles": int(sum(x0.shape[0] for x0, _ in meshes)), "meshes": len(meshes),
            "max_candidates_per_triangle": MAXC, "max_collisions_per_triangle": MAXCOL, "positions": "fp64",
            "step": "refit + traversal + continuous narrow phase of every mesh",
            "l2": "flushed between steps (256 MiB write); inputs 377 MB > L2",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


def load_reference_extension():
    """The reference's own CUDA extension, compiled from its sources (unmodified) by
    oracle/build_ref.py into oracle/_ref/cccollisions.so, or None where it was not built.
    Used only by the reference-GPU baseline leg."""
    import importlib.util
    so = os.path.join(ROOT, "oracle", "_ref", "cccollisions.so")
    if not os.path.exists(so):
        return None
    spec = importlib.util.spec_from_file_location("cccollisions", so)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


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

    # ---------------- plain per-mesh path through the reference-format API, timed first (the
    # per-call host work makes it sensitive to what ran before it in the process)
    X = [(torch.from_numpy(x0).to(dev), torch.from_numpy(x1).to(dev)) for x0, x1 in meshes]
    api.CHECK_STATUS = True
    api.STRICT = True              # a candidate or row overflow would raise: no truncated sets
    plain_out = None

    def plain():
        out = []
        for X0, X1 in X:
            bb, tr = C.bvh_motion(X0[None], X1[None])
            out.append(C.find_collisions_continuous(bb, tr, X0[None], X1[None], MAXC, MAXCOL))
        return out

    def timed(fn, n):
        ms, res = [], None
        for i in range(n):
            # the previous step's outputs (about 1.3 GB of rows and times) are released before
            # the next step, as a caller's would be; kept alive, they slowed the step by 4-9 ms
            res = None
            flush.fill_(i & 0xFF)
            torch.cuda.synchronize(dev)
            a, b = ev(), ev()
            a.record()
            res = fn()
            b.record()
            torch.cuda.synchronize(dev)
            ms.append(a.elapsed_time(b))
        return statistics.mean(ms), res

    torch.cuda.synchronize(dev)
    for _ in range(warm):
        plain()
    plain_ms, plain_out = timed(plain, args.steps)
    api.STRICT = False

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

    def rows_of(out):
        res = []
        for rows, times in out:
            r = rows[0].cpu().numpy()
            k = int((r[:, 0] >= 0).sum())
            res.append(_ms(r[:k], times[0, :k, 0].cpu().numpy()))
        return res

    equal = all(a == batched_rows[sid] for sid, a in zip(sids, rows_of(plain_out)))

    # ---------------- query-only legs on the same reference-order trees: this library's
    # find_collisions_continuous and the reference extension's own (its bvh_motion is not
    # run: its split search can loop without end on a GPU)
    api.STRICT = True
    trees = [C.bvh_motion(X0[None], X1[None]) for X0, X1 in X]

    def query():
        return [C.find_collisions_continuous(bb, tr, X0[None], X1[None], MAXC, MAXCOL) for (bb, tr), (X0, X1) in
                zip(trees, X)]

    query()
    query_ms, _ = timed(query, args.steps)
    api.STRICT = False
    ref_gpu = None
    R = load_reference_extension()
    if R is None:
        ref_gpu = {"unavailable": "the reference extension (oracle/_ref/cccollisions.so) is not built"}
    else:
        def ref_query():
            return [R.find_collisions_continuous(bb, tr, X0[None], X1[None], MAXC, MAXCOL) for (bb, tr), (X0, X1)
                    in zip(trees, X)]

        ref_steps = max(1, min(args.steps, 5))
        ref_query()
        ref_ms, ref_out = timed(ref_query, ref_steps)
        ref_equal = all(a == batched_rows[sid] for sid, a in zip(sids, rows_of(ref_out)))
        ref_gpu = {"value": world * total / (ref_ms / 1e3), "ms_per_step": ref_ms, "steps": ref_steps,
                   "rows_equal_batched": bool(ref_equal),
                   "path": "reference extension: find_collisions_continuous per mesh on prebuilt trees"}

    # ---------------- rooflines
    peak, peak_kind = load_peaks()
    dname, (dms, dcount) = max(kern.items(), key=lambda kv: kv[1][0])
    per_launch = dms / dcount
    # k_ccd_narrow reads a 16-byte record per pair with work and gathers both triangles at
    # both ends of the step (2 x 2 x 72 bytes); it writes 32 bytes per row
    narrow_bytes = cnt["live_pairs"] * (16 + 2 * 2 * 72) + int(sum(nrow)) * 32
    achieved = narrow_bytes / (per_launch / 1e3) / 1e9 if dname == "k_ccd_narrow" else None
    # the refit is two passes (block-local, then the climbs that leave a block)
    r1 = kern.get("k_engine_refit", (float("nan"), 1))
    r2 = kern.get("k_engine_refit_front", (0.0, 1))
    refit_ms = r1[0] / r1[1] + r2[0] / r2[1]
    rb = sum(refit_bytes(f) for f in Fs)
    bb_ = sum(build_bytes(f) for f in Fs)
    narrow_ms = kern["k_ccd_narrow"][0] / kern["k_ccd_narrow"][1]
    fp64_gflops = cnt["solved"] * FLOPS_PER_SUBTEST / (narrow_ms / 1e3) / 1e9
    phase_ms = sum(kern[k][0] / kern[k][1] for k in NARROW_PHASE if k in kern)
    phase_gflops = cnt["subtests"] * FLOPS_PER_SUBTEST / (phase_ms / 1e3) / 1e9
    eng.close()

    result = None
    if rank == 0:
        clocks = clk.summary()
        r3 = lambda x: float(f"{x:.4g}")
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": warm,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded cloth grids + icospheres)",
            "gpu_launches": int(launches),
            "config": workload_config(meshes, world),
            "roofline": {"kernel": dname, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                         "traffic": (NARROW_DRAM_BYTES_PER_SOLVED * cnt["solved"]) if dname == "k_ccd_narrow"
                         else None,
                         "alg_bytes_per_launch": narrow_bytes, "launch_ms": per_launch},
            "clocks": {"sm_mhz": clocks["sm_mhz"], "sm_max_mhz": clocks["sm_max_mhz"], "reasons": clocks["reasons"],
                       "samples": clocks["samples"]},
            "e2e": {"value": world * total / (e2e_ms / 1e3), "unit": UNIT, "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "path": "engine.StepPipeline from pinned host memory, rows + times back",
                    "rows_equal_batched": bool(e2e_equal)},
            "work": {"autotuned_shape": shape, "candidates": cnt["candidates"], "subtests": cnt["subtests"],
                     "subtests_solved": cnt["solved"], "pairs_with_work": cnt["live_pairs"],
                     "roots_in_unit_interval": cnt["roots"], "collision_rows": int(sum(nrow)), "status": cnt["status"],
                     "tree_boxes": "fp32"},
            "kernel_ms_per_step": {k: r3(v[0] / v[1]) for k, v in kern.items()},
            "fp64": {"kernel": "k_ccd_narrow", "units": "sub-tests solved", "achieved_gflops": r3(fp64_gflops),
                     "peak_gflops": FP64_PEAK_NOMINAL_GFLOPS, "peak_source": "nominal (B200 datasheet)",
                     "frac": r3(fp64_gflops / FP64_PEAK_NOMINAL_GFLOPS)},
            "narrow_phase": {"kernels": list(NARROW_PHASE), "ms": r3(phase_ms), "units": "every sub-test",
                             "effective_gflops": r3(phase_gflops),
                             "frac": r3(phase_gflops / FP64_PEAK_NOMINAL_GFLOPS)},
            "refit_roofline": {"alg_bytes": rb, "ms": r3(refit_ms), "achieved": r3(rb / (refit_ms / 1e3) / 1e9),
                               "peak": peak, "unit": "GB/s", "frac": r3(rb / (refit_ms / 1e3) / 1e9 / peak)},
            "build_roofline": {"alg_bytes": bb_, "ms": r3(build_ms), "achieved": r3(bb_ / (build_ms / 1e3) / 1e9),
                               "peak": peak, "unit": "GB/s", "frac": r3(bb_ / (build_ms / 1e3) / 1e9 / peak)},
            "plain": {"value": world * total / (plain_ms / 1e3), "ms_per_step": plain_ms,
                      "path": "per mesh: bvh_motion + find_collisions_continuous"},
            "query": {"value": world * total / (query_ms / 1e3), "ms_per_step": query_ms,
                      "path": "per mesh: find_collisions_continuous on prebuilt trees"},
            "reference_gpu": ref_gpu,
            "pair_sets_equal": bool(equal),
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


def run_served(args, dev, fold=None):
    """The served stream through the request server, and a sample of it through the engine
    and the plain per-request loop; fold: the fold's shape (workloads.impulse_fold_mesh)."""
    import torch

    from cccollisions_b200 import workloads as W
    from cccollisions_b200.serve import Request, Server, requests_from_stream
    reqs = requests_from_stream(W.served_stream(num_requests=args.served_requests, rate=2000.0), fold=fold)
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
    r3 = lambda x: float(f"{x:.4g}")
    return {"value": r3(st["throughput"]), "unit": UNIT, "requests": st["requests"], "rate_per_s": 2000.0,
            "p50_ms": r3(st["p50_ms"]), "p99_ms": r3(st["p99_ms"]), "mean_ms": r3(st["mean_ms"]),
            "makespan_s": r3(st["makespan_s"]), "request_triangles": st["triangles"], "ticks": st["ticks"],
            "mean_iterations": st["mean_iterations"], "converged_fraction": st["converged"],
            "contacts_first_iteration": st["contacts_first_iteration"],
            "contacts_last_iteration": st["contacts_last_iteration"],
            "contacts_all_iterations": st["contacts_all_iterations"], "budget_gb": args.served_budget_gb,
            "max_active_triangles": srv.max_active_triangles,
            "same_set": {"requests": len(sample), "triangles": ptris,
                         "engine": {"value": r3(same["throughput"]), "seconds": r3(same["makespan_s"])},
                         "plain": {"value": r3(ptris / dt), "seconds": r3(dt), "mean_iterations": float(np.mean(its))}}}


def run_reference(args):
    """The CPU implementation of the path (the oracle: C++ restatement of the reference's
    bvh_motion + find_collisions_continuous, all host threads), whole steps over every mesh
    of the same workload: W untimed steps, then K timed ones (wall clock)."""
    from oracle import oracle as O
    O.build()
    meshes = batched_meshes(args.meshes)
    nthreads = O.num_threads()
    total = sum(x0.shape[0] for x0, _ in meshes)

    def step():
        for x0, x1 in meshes:
            bb, tr = O.bvh(x0, x1)
            O.ccd(bb, tr, x0, x1, nthreads=nthreads)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    ms = (time.perf_counter() - t0) * 1e3 / args.steps
    v = total / (ms / 1e3)
    return {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded cloth grids + icospheres)",
            "config": workload_config(meshes, args.gpus), "impl": "reference",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port",
                             "sample": f"every step: all {len(meshes)} meshes ({total} triangles), bvh_motion + "
                                       f"continuous collisions per mesh"},
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
            if world == 1:
                v, threads, desc = cpu_sample(meshes, args.cpu_seconds)
                res["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc}
            if world == 1 and args.served_requests > 0:
                res["served"] = run_served(args, dev)
                ss = res["served"]["same_set"]
                res["served_over_plain"] = ss["engine"]["value"] / ss["plain"]["value"]
                # the same stream of folds whose layers start apart, where the loop runs until
                # no pair collides
                from cccollisions_b200 import workloads as W
                res["served_separated"] = {"fold": W.SEPARATED_FOLD, **run_served(args, dev, W.SEPARATED_FOLD)}
            # the headline ratios last, so that any tail of the line holds them
            res["batched_over_plain"] = res["plain"]["ms_per_step"] / res["ms_per_step"]
            rg = res["reference_gpu"]
            if rg and "ms_per_step" in rg:
                res["batched_over_reference_gpu"] = rg["ms_per_step"] / res["ms_per_step"]
                res["query_over_reference_gpu"] = rg["ms_per_step"] / res["query"]["ms_per_step"]
            print(json.dumps(res))
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
