"""Resident multi-mesh engine (``include/ccc_engine.h``) for PyTorch callers.

The reference extension processes one batch of equal-size meshes per call and rebuilds its
trees on every call.  ``Engine`` keeps meshes of uneven size resident in one device block
and runs each step over all active meshes at once:

    eng = Engine(tri_capacity=2_000_000, mesh_capacity=64)
    sids = [eng.add_mesh(x0.shape[0]) for x0, _ in meshes]
    for sid, (x0, x1) in zip(sids, meshes):
        eng.upload_soup(sid, x0, x1)                 # (F, 3, 3) host or device tensors
    eng.set_active(sids)
    eng.build(sids)                                  # LBVH topology, once
    eng.ccd()                                        # refit + traversal + narrow phase
    rows, times = eng.collisions(sids[0])            # (n, 3) int64 rows, (n,) times

``capture``/``replay`` turn a step into one CUDA graph launch that follows the active set;
``loop_prepare``/``loop_step`` run the impulse loop on meshes given as vertices + faces.
The block is an ordinary torch allocation, and every per-mesh array is a tensor view of it.

``StepPipeline`` streams collision steps from page-locked host inputs to page-locked host
outputs, overlapping each step's copies with the kernels of its neighbours.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np
import torch

from . import _native as N


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _ids(sids: Sequence[int]):
    a = np.ascontiguousarray(np.asarray(list(sids), dtype=np.int32))
    return a, a.ctypes.data_as(ctypes.c_void_p), len(a)


class Engine:
    def __init__(self, tri_capacity: int, vert_capacity: int = 0, mesh_capacity: int = 64,
                 max_candidates_per_triangle: int = 16, max_collisions_per_triangle: int = 16,
                 dtype: torch.dtype = torch.float64, device=None):
        if dtype not in (torch.float32, torch.float64):
            raise RuntimeError(f"unsupported floating type {dtype} (float32 or float64)")
        dev = torch.device(device if device is not None else "cuda")
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.dtype = dtype
        self.code = 0 if dtype == torch.float32 else 1
        self.maxc = int(max_candidates_per_triangle)
        self.maxcol = int(max_collisions_per_triangle)
        L = N.lib()
        nbytes = L.ccc_engine_bytes(self.code, tri_capacity, vert_capacity, mesh_capacity, self.maxc, self.maxcol)
        if nbytes < 0:
            raise RuntimeError("invalid engine capacities")
        self.nbytes = int(nbytes)
        self.block = torch.empty(self.nbytes, dtype=torch.uint8, device=self.device)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            N.check(L.ccc_engine_create(self.code, tri_capacity, vert_capacity, mesh_capacity, self.maxc, self.maxcol,
                                        ctypes.c_void_p(self.block.data_ptr()), self.nbytes, _stream(self.device),
                                        ctypes.byref(h)), "ccc_engine_create")
        self.handle = h
        self._views = {}

    # ---- lifetime ----
    def close(self):
        if self.handle:
            torch.cuda.current_stream(self.device).synchronize()
            N.lib().ccc_engine_destroy(self.handle)
            self.handle = None
            self.block = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- slots ----
    def add_mesh(self, F: int, V: int = 0) -> int:
        sid = ctypes.c_int32(-1)
        N.check(N.lib().ccc_engine_add_mesh(self.handle, int(F), int(V), ctypes.byref(sid)), "ccc_engine_add_mesh")
        return int(sid.value)

    def try_add_mesh(self, F: int, V: int = 0):
        """Slot id, or None when the block has no room for the mesh."""
        sid = ctypes.c_int32(-1)
        rc = N.lib().ccc_engine_add_mesh(self.handle, int(F), int(V), ctypes.byref(sid))
        return int(sid.value) if rc == N.CCC_OK else None

    def remove_mesh(self, sid: int):
        self._views.pop(sid, None)
        N.check(N.lib().ccc_engine_remove_mesh(self.handle, int(sid)), "ccc_engine_remove_mesh")

    def free_slots(self):
        t, v = ctypes.c_int64(), ctypes.c_int64()
        N.check(N.lib().ccc_engine_free_slots(self.handle, ctypes.byref(t), ctypes.byref(v)), "ccc_engine_free_slots")
        return int(t.value), int(v.value)

    def view(self, sid: int) -> dict:
        """Tensor views of a mesh's resident arrays (aliasing the engine block)."""
        if sid in self._views:
            return self._views[sid]
        mv = N.MeshView()
        N.check(N.lib().ccc_engine_mesh_view(self.handle, int(sid), ctypes.byref(mv)), "ccc_engine_mesh_view")
        base = self.block.data_ptr()
        F, V = int(mv.F), int(mv.V)
        esz = 4 if self.code == 0 else 8

        def sub(ptr, count, dtype, shape, size):
            off = int(ptr) - base
            return self.block[off:off + count * size].view(dtype).view(shape)

        out = {"F": F, "V": V,
               "x0": sub(mv.x0, F * 9, self.dtype, (F, 3, 3), esz),
               "x1": sub(mv.x1, F * 9, self.dtype, (F, 3, 3), esz),
               "masses": sub(mv.masses, F * 3, self.dtype, (F, 3), esz),
               "faces": sub(mv.faces, F * 3, torch.int32, (F, 3), 4),
               "rows": sub(mv.rows, F * self.maxcol * 3, torch.int64, (F * self.maxcol, 3), 8),
               "times": sub(mv.times, F * self.maxcol, self.dtype, (F * self.maxcol,), esz)}
        if V:
            out["verts0"] = sub(mv.verts0, V * 3, self.dtype, (V, 3), esz)
            out["verts1"] = sub(mv.verts1, V * 3, self.dtype, (V, 3), esz)
            out["vel"] = sub(mv.vel, V * 3, self.dtype, (V, 3), esz)
        self._views[sid] = out
        return out

    def _to(self, t, dtype=None):
        if not isinstance(t, torch.Tensor):
            t = torch.from_numpy(np.ascontiguousarray(t))
        return t.to(dtype or self.dtype)

    def upload_soup(self, sid: int, x0, x1, non_blocking: bool = False):
        v = self.view(sid)
        v["x0"].copy_(self._to(x0).reshape(v["x0"].shape), non_blocking=non_blocking)
        v["x1"].copy_(self._to(x1).reshape(v["x1"].shape), non_blocking=non_blocking)

    def upload_mesh(self, sid: int, verts0, verts1, vel, faces, masses, non_blocking: bool = False):
        v = self.view(sid)
        v["verts0"].copy_(self._to(verts0), non_blocking=non_blocking)
        v["verts1"].copy_(self._to(verts1), non_blocking=non_blocking)
        v["vel"].copy_(self._to(vel), non_blocking=non_blocking)
        v["faces"].copy_(self._to(faces, torch.int32), non_blocking=non_blocking)
        v["masses"].copy_(self._to(masses), non_blocking=non_blocking)

    # ---- steps ----
    def set_active(self, sids: Sequence[int]):
        a, p, n = _ids(sids)
        N.check(N.lib().ccc_engine_set_active(self.handle, p, n, _stream(self.device)), "ccc_engine_set_active")
        self._active = a

    def build(self, sids: Sequence[int]):
        a, p, n = _ids(sids)
        N.check(N.lib().ccc_engine_build(self.handle, p, n, _stream(self.device)), "ccc_engine_build")

    def ccd(self):
        N.check(N.lib().ccc_engine_ccd(self.handle, _stream(self.device)), "ccc_engine_ccd")

    def loop_prepare(self, sids: Sequence[int]):
        a, p, n = _ids(sids)
        N.check(N.lib().ccc_engine_loop_prepare(self.handle, p, n, _stream(self.device)), "ccc_engine_loop_prepare")

    def loop_step(self, max_iter: int = 50):
        N.check(N.lib().ccc_engine_loop_step(self.handle, int(max_iter), _stream(self.device)), "ccc_engine_loop_step")

    def capture(self, op: int, max_iter: int = 50, stream: torch.cuda.Stream | None = None):
        s = stream or torch.cuda.current_stream(self.device)
        if s.cuda_stream == 0:
            raise RuntimeError("capture needs a non-default stream")
        N.check(N.lib().ccc_engine_capture(self.handle, int(op), int(max_iter), ctypes.c_void_p(s.cuda_stream)),
                "ccc_engine_capture")

    def replay(self, op: int):
        N.check(N.lib().ccc_engine_replay(self.handle, int(op), _stream(self.device)), "ccc_engine_replay")

    def autotune(self) -> int:
        c = ctypes.c_int32(-1)
        N.check(N.lib().ccc_engine_autotune(self.handle, _stream(self.device), ctypes.byref(c)), "ccc_engine_autotune")
        return int(c.value)

    @staticmethod
    def schedules() -> list[dict]:
        """The autotuner's candidate schedules: traversal blocks per SM, narrow-phase blocks
        per SM (in units of the resident count), the traversal form (0 one query per
        thread, 1 32 queries per warp), the tree levels below the root that each traversal
        block keeps in shared memory (0-2, one query per thread) and the narrow phase's
        batch in units of 256 sub-tests (1 or 2)."""
        out = []
        for i in range(N.lib().ccc_engine_schedule_count()):
            a = (ctypes.c_int32 * 5)()
            N.check(N.lib().ccc_engine_schedule_info(i, a), "ccc_engine_schedule_info")
            out.append({"traversal_blocks_per_sm": a[0], "narrow_blocks": a[1], "warp_traversal": a[2],
                        "staged_levels": a[3], "narrow_batch": a[4]})
        return out

    def set_schedule(self, choice: int):
        N.check(N.lib().ccc_engine_set_schedule(self.handle, int(choice)), "ccc_engine_set_schedule")

    def state(self, sids: Sequence[int]) -> dict:
        """Synchronises; status word and per-mesh rows, contacts, iterations, flags."""
        a, p, n = _ids(sids)
        st = ctypes.c_int32(0)
        rows = np.zeros(n, np.int32)
        con = np.zeros(n, np.int32)
        it = np.zeros(n, np.int32)
        fl = np.zeros(n, np.int32)
        P = lambda x: x.ctypes.data_as(ctypes.c_void_p)
        N.check(N.lib().ccc_engine_read_state(self.handle, p, n, ctypes.byref(st), P(rows), P(con), P(it), P(fl),
                                              _stream(self.device)), "ccc_engine_read_state")
        return {"status": int(st.value), "rows": rows, "contacts": con, "iterations": it, "flags": fl}

    def counters(self) -> dict:
        """Synchronises; work counters of the last step: status word, candidate pairs (in a
        collision step, those whose triangles share no vertex), sub-tests with overlapping
        sub-boxes, roots in [0, 1] filtered, sub-tests solved
        (each repeated sub-test is solved once for all the pairs that have it) and the
        candidate pairs with sub-tests to solve."""
        out = (ctypes.c_int32 * 6)()
        N.check(N.lib().ccc_engine_counters(self.handle, out, _stream(self.device)), "ccc_engine_counters")
        return {"status": int(out[0]), "candidates": int(out[1]), "subtests": int(out[2]), "roots": int(out[3]),
                "solved": int(out[4]), "live_pairs": int(out[5])}

    def pack_rows(self, out_rows: torch.Tensor, out_times: torch.Tensor, out_meta: torch.Tensor):
        """Packs the last ccd()'s rows of every active mesh back to back on the device (no
        synchronisation): out_rows (capacity, 3) int64, out_times (capacity,), out_meta
        (2 M + 2,) int32 = [row offset of each mesh in slot order, total, slot ids, status]."""
        if out_rows.dtype != torch.int64 or out_times.dtype != self.dtype or out_meta.dtype != torch.int32:
            raise RuntimeError("pack_rows: int64 rows, engine-dtype times and int32 meta expected")
        if not (out_rows.is_contiguous() and out_times.is_contiguous() and out_meta.is_contiguous()):
            raise RuntimeError("pack_rows: contiguous outputs expected")
        cap = min(out_rows.shape[0], out_times.shape[0])
        N.check(N.lib().ccc_engine_pack_rows(self.handle, ctypes.c_void_p(out_rows.data_ptr()),
                                             ctypes.c_void_p(out_times.data_ptr()), int(cap),
                                             ctypes.c_void_p(out_meta.data_ptr()), _stream(self.device)),
                "ccc_engine_pack_rows")

    def collisions(self, sid: int, count: int | None = None):
        """(rows (n, 3) int64, times (n,)) of the last ccd() for one mesh (views)."""
        if count is None:
            count = int(self.state([sid])["rows"][0])
        v = self.view(sid)
        return v["rows"][:count], v["times"][:count]


def _ranges(views, key):
    """Byte ranges of the given arrays in the engine block, adjacent ones merged."""
    spans = sorted((v[key].data_ptr(), v[key].data_ptr() + v[key].numel() * v[key].element_size()) for v in views)
    out = []
    for a, b in spans:
        if out and out[-1][1] == a:
            out[-1][1] = b
        else:
            out.append([a, b])
    return out


class StepPipeline:
    """Collision steps of a fixed active set, streamed from page-locked host memory to
    page-locked host memory.

    Step k's soups go up on one copy stream while step k-1 runs; step k's rows, packed on
    the device (``Engine.pack_rows``), come down on a second copy stream while step k+1
    runs.  The kernels of consecutive steps therefore run back to back, and a step's
    host-device traffic costs time only where it exceeds a step's kernel time.

    Device staging: one copy of the active meshes' soups and two packed-row buffers of
    (active triangles x max_collisions_per_triangle) rows.  The engine's step must have been
    captured (``Engine.capture(ENGINE_OP_CCD)``) for ``graph=True``; the active set and
    trees must be those of ``sids``.
    """

    def __init__(self, engine: Engine, sids: Sequence[int], graph: bool = True):
        self.e = engine
        self.sids = list(sids)
        self.graph = graph
        dev = engine.device
        views = [engine.view(s) for s in self.sids]
        self.M = len(self.sids)
        self.capacity = sum(v["F"] for v in views) * engine.maxcol
        base = engine.block.data_ptr()
        # device staging of the soups, laid out like the engine's slot ranges
        self._stage, self._pairs, self._slices = {}, [], []
        for key in ("x0", "x1"):
            for a, b in _ranges(views, key):
                st = torch.empty(b - a, dtype=torch.uint8, device=dev)
                self._pairs.append((engine.block[a - base:b - base], st))
                self._stage[(key, a)] = st
        for v in views:
            sl = []
            for key in ("x0", "x1"):
                p = v[key].data_ptr()
                a = max(k[1] for k in self._stage if k[0] == key and k[1] <= p)
                st = self._stage[(key, a)]
                n = v[key].numel() * v[key].element_size()
                sl.append(st[p - a:p - a + n].view(engine.dtype).view(v[key].shape))
            self._slices.append(tuple(sl))
        self._rows = [torch.empty((max(self.capacity, 1), 3), dtype=torch.int64, device=dev) for _ in range(2)]
        self._times = [torch.empty(max(self.capacity, 1), dtype=engine.dtype, device=dev) for _ in range(2)]
        self._meta = [torch.empty(2 * self.M + 2, dtype=torch.int32, device=dev) for _ in range(2)]
        # page-locked copies the host reads the counts from (step k in slot k % 2)
        self._meta_h = [torch.empty(2 * self.M + 2, dtype=torch.int32).pin_memory() for _ in range(2)]
        self.compute = torch.cuda.Stream(dev)
        self.copy_in = torch.cuda.Stream(dev)
        self.copy_out = torch.cuda.Stream(dev)

    def host_outputs(self):
        """Page-locked (rows, times, meta) host buffers sized for one step."""
        return (torch.empty((max(self.capacity, 1), 3), dtype=torch.int64).pin_memory(),
                torch.empty(max(self.capacity, 1), dtype=self.e.dtype).pin_memory(),
                torch.empty(2 * self.M + 2, dtype=torch.int32).pin_memory())

    def run(self, inputs, outputs) -> list[int]:
        """inputs[k]: one (x0, x1) pair of page-locked host tensors per mesh (order of sids)
        for step k; outputs[k]: (rows, times, meta) host tensors from host_outputs() that
        receive step k's rows (the same triple may serve several steps; each then holds the
        last of them).  meta = [row offset of each mesh in
        slot order, total, slot ids, status word].  Returns the row count of every step;
        raises if a step's status word reports an error."""
        e, K = self.e, len(inputs)
        if len(outputs) != K:
            raise ValueError("one output triple per step")
        ev = lambda: torch.cuda.Event()
        up, in_free, done, down = [ev() for _ in range(K)], [ev() for _ in range(K)], [ev() for _ in range(K)], \
            [ev() for _ in range(K)]
        totals, status = [0] * K, [0] * K

        def upload(k):
            with torch.cuda.stream(self.copy_in):
                if k > 0:
                    self.copy_in.wait_event(in_free[k - 1])
                for (d0, d1), (h0, h1) in zip(self._slices, inputs[k]):
                    d0.copy_(h0.view(d0.shape), non_blocking=True)
                    d1.copy_(h1.view(d1.shape), non_blocking=True)
                up[k].record(self.copy_in)

        def download(k):
            done[k].synchronize()
            rows_h, times_h, meta_h = outputs[k]
            meta = self._meta_h[k % 2]
            meta_h.copy_(meta)
            n = min(int(meta[self.M]), self.capacity)
            totals[k] = int(meta[self.M])
            status[k] = int(meta[2 * self.M + 1])
            with torch.cuda.stream(self.copy_out):
                self.copy_out.wait_event(done[k])
                if n:
                    rows_h[:n].copy_(self._rows[k % 2][:n], non_blocking=True)
                    times_h[:n].copy_(self._times[k % 2][:n], non_blocking=True)
                down[k].record(self.copy_out)

        self.compute.wait_stream(torch.cuda.current_stream(e.device))
        if K:
            upload(0)
        for k in range(K):
            with torch.cuda.stream(self.compute):
                self.compute.wait_event(up[k])
                for dst, src in self._pairs:
                    dst.copy_(src, non_blocking=True)
                in_free[k].record(self.compute)
                if self.graph:
                    e.replay(N.ENGINE_OP_CCD)
                else:
                    e.ccd()
                if k >= 2:
                    self.compute.wait_event(down[k - 2])
                e.pack_rows(self._rows[k % 2], self._times[k % 2], self._meta[k % 2])
                self._meta_h[k % 2].copy_(self._meta[k % 2], non_blocking=True)
                done[k].record(self.compute)
            if k + 1 < K:
                upload(k + 1)
            if k >= 1:
                download(k - 1)
        if K:
            download(K - 1)
        self.copy_out.synchronize()
        bad = [(k, st) for k, st in enumerate(status) if st & ~N.CCC_ST_NONFINITE]
        if bad:
            raise RuntimeError(f"engine status {bad[0][1]:#x} in step {bad[0][0]}")
        return totals
