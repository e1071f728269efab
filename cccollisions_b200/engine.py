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
        """Synchronises; work counters of the last step."""
        out = (ctypes.c_int32 * 4)()
        N.check(N.lib().ccc_engine_counters(self.handle, out, _stream(self.device)), "ccc_engine_counters")
        return {"status": int(out[0]), "candidates": int(out[1]), "subtests": int(out[2]), "roots": int(out[3])}

    def collisions(self, sid: int, count: int | None = None):
        """(rows (n, 3) int64, times (n,)) of the last ccd() for one mesh (views)."""
        if count is None:
            count = int(self.state([sid])["rows"][0])
        v = self.view(sid)
        return v["rows"][:count], v["times"][:count]
