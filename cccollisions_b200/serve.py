"""Served form: a continuous-batching request loop over the resident engine.

Requests are impulse solves (the engine's impulse loop: collision check with impulses,
per-vertex corrections, repeated until a check finds no contact or ``max_iter``
iterations) on meshes given as vertices + faces.  The server owns one engine sized to a
device-memory budget and works in ticks:

1. one loop iteration for every active request (one CUDA graph replay);
2. while the GPU runs it, requests that have arrived are admitted in arrival order as long
   as their slots fit in the block and the active triangles stay within
   ``max_active_triangles`` (a request that does not fit waits, and so do the ones behind
   it; a request alone is always admitted), and their inputs are copied to the device on a
   second stream;
3. the tick's per-mesh flags are read back; finished requests copy their vertices back to
   the host, release their slots and report their latency (arrival to result on the host);
4. admitted requests get their trees and join the active set before the next tick.

Requests that arrive while others are on the GPU therefore join at the next iteration
boundary and share its launches.  The active-triangle cap trades nothing in throughput once
the active set fills the GPU (a few hundred thousand triangles) and bounds the time of a
tick, so under a backlog the early requests finish early instead of all requests finishing
together at the end of the backlog.  Each mesh is processed independently and the loop's
impulse sums are order independent, so a request's result is bit for bit the same alone
and in any mix.
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native as N
from .engine import Engine


@dataclass
class Request:
    verts0: np.ndarray
    verts1: np.ndarray
    vel: np.ndarray
    faces: np.ndarray
    masses: np.ndarray
    arrival: float = 0.0                 # seconds after the start of the run
    rid: int = 0
    # results
    admitted: float = float("nan")
    finished: float = float("nan")
    iterations: int = -1
    converged: bool = False
    verts1_out: np.ndarray | None = None
    contacts: list = field(default_factory=list)     # contacts found by each loop iteration
    _sid: int = field(default=-1, repr=False)
    _pinned: tuple = field(default=(), repr=False)
    _result: object = field(default=None, repr=False)    # pinned host buffer for verts1

    @property
    def F(self) -> int:
        return int(self.faces.shape[0])

    @property
    def V(self) -> int:
        return int(self.verts0.shape[0])

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def engine_capacity(budget_bytes: int, dtype=torch.float64, mesh_capacity: int = 4096,
                    vert_ratio: float = 0.75, maxc: int = 16) -> tuple[int, int]:
    """Largest (triangle, vertex) capacity whose engine block fits the budget, with
    vert_ratio vertices per triangle (a grid mesh has about 0.5).  The budget also holds the
    library's fixed module-data array (ccc_static_scratch_bytes, resident on every device
    where the library is loaded), so the block gets what is left after it."""
    code = 0 if dtype == torch.float32 else 1
    lo, hi = 2, 1 << 27
    L = N.lib()
    budget_bytes = int(budget_bytes) - int(L.ccc_static_scratch_bytes())
    while lo < hi:
        mid = (lo + hi + 1) // 2
        b = L.ccc_engine_bytes(code, mid, int(mid * vert_ratio) + 16, mesh_capacity, maxc, 1)
        if 0 < b <= budget_bytes:
            lo = mid
        else:
            hi = mid - 1
    return lo, int(lo * vert_ratio) + 16


class Server:
    def __init__(self, budget_bytes: int = 40 << 30, dtype=torch.float64, max_iter: int = 50,
                 mesh_capacity: int = 4096, maxc: int = 16, device=None, vert_ratio: float = 0.75,
                 max_active_triangles: int | None = 1 << 20):
        self.dtype = dtype
        self.max_iter = int(max_iter)
        self.max_active_triangles = max_active_triangles
        tc, vc = engine_capacity(budget_bytes, dtype, mesh_capacity, vert_ratio, maxc)
        self.engine = Engine(tri_capacity=tc, vert_capacity=vc, mesh_capacity=mesh_capacity,
                             max_candidates_per_triangle=maxc, max_collisions_per_triangle=1, dtype=dtype,
                             device=device)
        self.device = self.engine.device
        self.compute = torch.cuda.Stream(self.device)
        self.copy = torch.cuda.Stream(self.device)
        with torch.cuda.stream(self.compute):
            self.engine.set_active([])
            self.engine.capture(N.ENGINE_OP_LOOP_STEP, self.max_iter, self.compute)
        self.ticks = 0

    def close(self):
        self.engine.close()

    def _pin(self, r: Request):
        np_dt = np.float32 if self.dtype == torch.float32 else np.float64
        t = lambda a, dt=np_dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).pin_memory()
        r._pinned = (t(r.verts0), t(r.verts1), t(r.vel), t(r.faces, np.int32), t(r.masses))
        # page-locking memory is slow, so the result buffer is set up with the inputs
        r._result = torch.empty((r.V, 3), dtype=self.dtype).pin_memory()

    def run(self, requests: list[Request], realtime: bool = True) -> dict:
        """Serve the requests (arrival times in seconds from now when realtime, else all at
        once); returns throughput and latency statistics.  Results are stored on each request."""
        if not requests:
            raise ValueError("no requests to serve")
        for r in requests:
            if not r._pinned:
                self._pin(r)
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        active: dict[int, Request] = {}
        eng = self.engine
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0
        joining: list[tuple[Request, torch.cuda.Event]] = []
        cap = self.max_active_triangles
        load = [0]                       # triangles of the active and joining requests

        def admit():
            while pending and (not realtime or pending[0].arrival <= now()):
                r = pending[0]
                if cap is not None and load[0] > 0 and load[0] + r.F > cap:
                    break
                sid = eng.try_add_mesh(r.F, r.V)
                if sid is None:
                    break
                pending.popleft()
                load[0] += r.F
                r._sid = sid
                r.admitted = now()
                with torch.cuda.stream(self.copy):
                    eng.upload_mesh(sid, *r._pinned, non_blocking=True)
                    ev = torch.cuda.Event()
                    ev.record(self.copy)
                joining.append((r, ev))

        with torch.cuda.stream(self.compute):
            while pending or active or joining:
                if active:
                    eng.replay(N.ENGINE_OP_LOOP_STEP)
                    self.ticks += 1
                admit()
                done = []
                if active:
                    sids = list(active)
                    st = eng.state(sids)
                    if st["status"] & ~N.CCC_ST_NONFINITE:
                        raise RuntimeError(f"engine status {st['status']:#x}")
                    for sid, c in zip(sids, st["contacts"]):
                        active[sid].contacts.append(int(c))
                    done = [(sid, int(it), bool(fl & N.CCC_MESH_CONVERGED))
                            for sid, it, fl in zip(sids, st["iterations"], st["flags"]) if fl & N.CCC_MESH_DONE]
                    if done:
                        outs = []
                        for sid, it, conv in done:
                            r = active.pop(sid)
                            r.iterations, r.converged = it, conv
                            host = r._result
                            host.copy_(eng.view(sid)["verts1"], non_blocking=True)
                            outs.append((r, host))
                        self.compute.synchronize()
                        t = now()
                        for r, host in outs:
                            r.verts1_out = host.numpy().copy()
                            r.finished = t
                            eng.remove_mesh(r._sid)
                            load[0] -= r.F
                changed = bool(done)
                if joining:
                    ids = []
                    for r, ev in joining:
                        self.compute.wait_event(ev)
                        ids.append(r._sid)
                    eng.loop_prepare(ids)
                    for r, _ in joining:
                        active[r._sid] = r
                    joining = []
                    changed = True
                if changed:
                    eng.set_active(list(active))
                if not active and pending:
                    wait = pending[0].arrival - now() if realtime else 0.0
                    if wait > 0:
                        time.sleep(wait)
                    elif eng.free_slots()[0] < pending[0].F or eng.free_slots()[1] < pending[0].V:
                        raise RuntimeError(f"request {pending[0].rid} ({pending[0].F} triangles) does not fit the "
                                           "engine block")
        lat = np.array([r.latency for r in requests])
        first = min(r.arrival for r in requests)
        last = max(r.finished for r in requests)
        tris = sum(r.F for r in requests)
        return {"requests": len(requests), "triangles": tris, "makespan_s": last - first,
                "throughput": tris / (last - first), "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3), "mean_ms": float(lat.mean() * 1e3),
                "ticks": self.ticks, "mean_iterations": float(np.mean([r.iterations for r in requests])),
                "converged": float(np.mean([r.converged for r in requests])),
                "contacts_first_iteration": int(sum(r.contacts[0] for r in requests if r.contacts)),
                "contacts_last_iteration": int(sum(r.contacts[-1] for r in requests if r.contacts)),
                "contacts_all_iterations": int(sum(sum(r.contacts) for r in requests))}


def requests_from_stream(stream, dtype=np.float64, fold=None) -> list[Request]:
    """Requests of workloads.served_stream entries (arrival, seed, nx, ny); fold: keyword
    arguments of workloads.impulse_fold_mesh (such as workloads.SEPARATED_FOLD)."""
    from . import workloads as W
    out = []
    for i, (t, seed, nx, ny) in enumerate(stream):
        v0, v1, vel, faces, masses = W.impulse_fold_mesh(seed, nx, ny, dtype=dtype, **(fold or {}))
        out.append(Request(v0, v1, vel, faces, masses, arrival=t, rid=i))
    return out
