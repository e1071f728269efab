"""Benchmark of the collision-handling step on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload W]

Workload (default ``cloth_sphere``): the plain continuous-collision step of the reference's
API on a 128x128 cloth (32,258 triangles) falling onto a level-5 icosphere (20,480
triangles), fp64, as one 52,738-triangle soup: ``bvh_motion`` + ``find_collisions_continuous``
(max 16 candidates / 16 collisions per triangle).  Metric: triangle-steps per second (one
triangle carried through one full step).

* ``value``: inputs resident in HBM, outputs and scratch preallocated, C ABI calls on one
  stream, CUDA events around every step, L2 flushed (256 MiB write) between steps outside
  the timed events.
* ``e2e``: the public drop-in API from pinned host buffers: H2D copy of both triangle
  soups, bvh_motion, find_collisions_continuous (which reads back its status word), a
  count of valid rows and a D2H copy of those rows and times.
* ``roofline``: the kernel with the largest share of the timed region, its algorithmic
  bytes per launch over its CUDA-event duration, against MEASURED_PEAKS.json.
* ``cpu_baseline``: the same step on the host cores with the C++ oracle (OpenMP).

Multi-GPU: the step does not shard (one mesh, no exchange), so N ranks run N independent
replicas ("replicas only"); value is the total over ranks divided by the slowest rank.
``--impl reference`` times the CPU implementation (the oracle restatement of the
reference's algorithm) on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "triangle-steps/sec"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cloth_sphere", choices=["cloth_sphere"])
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


def cpu_baseline(x0, x1, seconds):
    """Oracle (C++ restatement of the reference pipeline) on the host cores."""
    from oracle import oracle as O
    O.build()
    nthreads = O.num_threads()
    F = x0.shape[1]
    reps = 0
    t0 = time.perf_counter()
    while True:
        bb, tr = O.bvh(x0[0], x1[0])
        O.ccd(bb, tr, x0[0], x1[0], nthreads=nthreads)
        reps += 1
        if time.perf_counter() - t0 >= seconds or reps >= 200:
            break
    dt = time.perf_counter() - t0
    return {"value": reps * F / dt, "unit": METRIC, "cores": nthreads, "kind": "port",
            "sample": f"{reps} full steps of the {F}-triangle cloth_sphere workload (bvh_motion + continuous "
                      f"collisions), {dt:.1f} s"}


def alg_bytes(kernel, F, cand, rows):
    """Algorithmic bytes of one launch (fp64, motion) for the kernels of this step."""
    tri = 72  # one fp64 triangle (9 doubles)
    if kernel == "k_leaf_rows":          # read x0, x1; write leaf box (48 B) + 3 tree fields (24 B)
        return F * (2 * tri + 48 + 24)
    if kernel == "k_karras_identity":    # write left/right/id of F-1 internal rows + 2F-2 parent fields
        return (F - 1) * 24 + (2 * F - 2) * 8
    if kernel == "k_refit":              # read parent links + 2 child boxes, write one box per internal node
        return (F - 1) * (2 * 48 + 48 + 24) + F * 8
    if kernel == "k_import_nodes":       # read internal tree rows + child boxes/ids, write 64 B node
        return (F - 1) * (32 + 2 * 48 + 64) + F * 8
    if kernel == "k_import_rightmost":   # parent links, node refs, rightmost writes
        return F * 8 + (F - 1) * (8 + 16 + 4 + 4)
    if kernel == "k_traverse":           # query box + id per leaf, every node once, candidate pairs out
        return F * (48 + 8) + (F - 1) * 64 + cand * 8
    if kernel == "k_ccd_narrow":         # candidate pair in, two moving triangles (x0, x1), rows + times out
        return cand * (8 + 2 * 2 * tri) + rows * (24 + 8)
    if kernel == "k_uniform_offsets":
        return 8
    return 0


def run_ours(args, rank, world, dev):
    import ctypes
    import torch

    from cccollisions_b200 import _native as N
    from cccollisions_b200 import api, workloads as W

    lib = N.lib()
    x0, x1 = W.cloth_sphere()
    B, F = x0.shape[0], x0.shape[1]
    maxc = maxcol = 16
    X0 = torch.from_numpy(x0).to(dev)
    X1 = torch.from_numpy(x1).to(dev)
    bboxes = torch.empty((B, 2 * F - 1, 6), dtype=torch.float64, device=dev)
    tree = torch.empty((B, 2 * F - 1, 4), dtype=torch.int64, device=dev)
    rows = torch.empty((B, F * maxcol, 3), dtype=torch.int64, device=dev)
    times = torch.empty((B, F * maxcol, 1), dtype=torch.float64, device=dev)
    ws_b = torch.empty(lib.ccc_workspace_size(N.OP_BVH, B, F, 0), dtype=torch.uint8, device=dev)
    ws_c = torch.empty(lib.ccc_workspace_size(N.OP_CONTINUOUS, B, F, maxc), dtype=torch.uint8, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(stream.cuda_stream)
    P = lambda t: ctypes.c_void_p(t.data_ptr())

    def step():
        rows.fill_(-1)
        times.fill_(-1)
        rc = lib.ccc_bvh(1, P(X0), P(X1), B, F, P(bboxes), P(tree), P(ws_b), ws_b.numel(), sp)
        assert rc == 0
        rc = lib.ccc_find_collisions_continuous(1, P(bboxes), P(tree), P(X0), P(X1), None, B, F, maxc, maxcol,
                                                P(rows), P(times), P(ws_c), ws_c.numel(), sp)
        assert rc == 0

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize(dev)
    st = (ctypes.c_int32 * 3)()
    lib.ccc_read_status(P(ws_c), 1, st, sp)
    status, cand, nrows = int(st[0]), int(st[1]), int(st[2])

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    launches0 = N.kernel_launches()
    N.timing_begin()
    with ClockSampler(dev.index if dev.index is not None else 0) as clk:
        for i in range(args.steps):
            flush.fill_(i & 0xFF)            # evict L2 between steps (outside the events)
            ev[i][0].record(stream)
            step()
            ev[i][1].record(stream)
        torch.cuda.synchronize(dev)
    kern = N.timing_end()
    launches = N.kernel_launches() - launches0
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
        torch.distributed.barrier()
    ms_per_step = total_ms / args.steps
    value = world * F * args.steps / (total_ms / 1e3)

    # ---- roofline of the dominant kernel
    peak, peak_kind = load_peaks()
    dom = max(kern.items(), key=lambda kv: kv[1][0])
    dname, (dms, dcount) = dom
    per_launch_ms = dms / dcount
    abytes = alg_bytes(dname, F, cand, nrows)
    achieved = abytes / (per_launch_ms / 1e3) / 1e9
    share = {k: round(v[0] / max(total_ms, 1e-9), 4) for k, v in kern.items()}

    # ---- end to end through the public API from pinned host memory
    hx0 = torch.from_numpy(x0).pin_memory()
    hx1 = torch.from_numpy(x1).pin_memory()
    api.CHECK_STATUS = True
    e2e_ev = []
    d2h = 0
    for i in range(max(args.warmup, 3) + args.steps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        flush.fill_(i & 0xFF)
        a.record(stream)
        dX0 = hx0.to(dev, non_blocking=True)
        dX1 = hx1.to(dev, non_blocking=True)
        import cccollisions_b200 as C
        bb, tr = C.bvh_motion(dX0, dX1)
        r, t = C.find_collisions_continuous(bb, tr, dX0, dX1, maxc, maxcol)
        n = int((r[0, :, 0] >= 0).sum().item())
        hr = r[0, :n].cpu()
        ht = t[0, :n].cpu()
        b.record(stream)
        torch.cuda.synchronize(dev)
        if i >= max(args.warmup, 3):
            e2e_ev.append(a.elapsed_time(b))
            d2h = 8 + hr.numel() * 8 + ht.numel() * 8
    e2e_ms = sum(e2e_ev) / len(e2e_ev)
    if world > 1:
        t_ = torch.tensor([e2e_ms], device=dev)
        torch.distributed.all_reduce(t_, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t_.item())
    e2e_value = world * F / (e2e_ms / 1e3)

    result = None
    if rank == 0:
        clocks = clk.summary()
        result = {
            "metric": METRIC, "value": value, "unit": "triangle-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded cloth + icosphere)",
            "config": {"workload": "cloth_sphere: plain CCD step, bvh_motion + find_collisions_continuous",
                       "triangles": F, "batch": B, "max_candidates_per_triangle": maxc,
                       "max_collisions_per_triangle": maxcol, "l2": "flushed between steps (256 MiB write)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "candidates": cand, "collision_rows": nrows, "status": status},
            "e2e": {"value": e2e_value, "unit": "triangle-steps/s", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": int(x0.nbytes + x1.nbytes), "d2h_bytes_per_step": int(d2h)},
            "roofline": {"kernel": dname, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind, "traffic": None,
                         "alg_bytes_per_launch": abytes, "launch_ms": per_launch_ms},
            "kernel_share": share,
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in kern.items()},
            "gpu_launches": int(launches),
            "clocks": {"sm_mhz": clocks["sm_mhz"], "sm_max_mhz": clocks["sm_max_mhz"], "reasons": clocks["reasons"]},
        }
        if world == 1:
            result["cpu_baseline"] = cpu_baseline(x0, x1, args.cpu_seconds)
    return result


def run_reference(args):
    from cccollisions_b200 import workloads as W
    x0, x1 = W.cloth_sphere()
    F = x0.shape[1]
    per = max(2.0, args.cpu_seconds / max(args.steps, 1))
    vals = []
    base = None
    for i in range(max(args.warmup, 0) + args.steps):
        base = cpu_baseline(x0, x1, per)
        if i >= args.warmup:
            vals.append(base["value"])
    v = statistics.median(vals)
    ms = F / v * 1e3
    base["value"] = v
    return {"metric": METRIC, "value": v, "unit": "triangle-steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded cloth + icosphere)",
            "config": {"workload": "cloth_sphere: plain CCD step, bvh_motion + find_collisions_continuous",
                       "triangles": F},
            "impl": "reference", "cpu_baseline": base,
            "e2e": {"value": v, "unit": "triangle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


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
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=dev)
    try:
        res = run_ours(args, rank, world, dev)
        if rank == 0:
            print(json.dumps(res))
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
