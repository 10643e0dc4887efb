"""Python front end of the request loop (pppm_server_* in include/pppm.h)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import (REQ_ADVANCE, REQ_EVAL, PppmRequestInfo, PppmServerConfig, check, default_params, load)


class Server:
    """Resident scenes served by `slots` worker streams under an HBM budget."""

    def __init__(self, hbm_budget_bytes: int = 150 << 30, slots: int = 8):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("the request loop needs a CUDA device; no CPU path exists")
        self._lib = load()
        cfg = PppmServerConfig(hbm_budget_bytes=int(hbm_budget_bytes), slots=int(slots))
        h = C.c_void_p()
        check(self._lib.pppm_server_create(C.byref(cfg), C.byref(h)), "pppm_server_create")
        self._h = h
        self._N = {}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pppm_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_scene(self, n: int, pos4: np.ndarray, alpha: np.ndarray, **params) -> int:
        pos4 = np.ascontiguousarray(pos4, dtype=np.float32)
        al = np.ascontiguousarray(alpha, dtype=np.float64)
        if al.shape[0] != 3:
            al = np.ascontiguousarray(al.T)
        N = pos4.shape[0]
        p = default_params(n, **params)
        sid = C.c_uint64()
        check(self._lib.pppm_server_add_scene(self._h, C.byref(p), N, pos4.ctypes.data, al[0].ctypes.data,
                                              al[1].ctypes.data, al[2].ctypes.data, C.byref(sid)),
              "pppm_server_add_scene")
        self._N[sid.value] = N
        return sid.value

    def submit_eval(self, scene: int) -> int:
        t = C.c_uint64()
        check(self._lib.pppm_server_submit(self._h, scene, REQ_EVAL, 0, 0.0, C.byref(t)), "pppm_server_submit")
        return (t.value, scene)

    def submit_advance(self, scene: int, steps: int, dt: float) -> int:
        t = C.c_uint64()
        check(self._lib.pppm_server_submit(self._h, scene, REQ_ADVANCE, steps, dt, C.byref(t)), "pppm_server_submit")
        return (t.value, scene)

    def wait(self, ticket, timeout_s: float = 600.0):
        """Returns (info dict, velocities (N,3) for EVAL else None)."""
        tk, scene = ticket
        info = PppmRequestInfo()
        vel = np.empty((3, self._N[scene]), dtype=np.float64)
        check(self._lib.pppm_server_wait(self._h, tk, timeout_s, C.byref(info), vel.ctypes.data), "pppm_server_wait")
        d = {"submit_s": info.submit_s, "start_s": info.start_s, "end_s": info.end_s,
             "latency_s": info.end_s - info.submit_s}
        return d, vel.T

    def positions(self, scene: int) -> np.ndarray:
        out = np.empty((self._N[scene], 4), dtype=np.float32)
        check(self._lib.pppm_server_read_positions(self._h, scene, out.ctypes.data), "pppm_server_read_positions")
        return out

    def stats(self):
        rb, done = C.c_uint64(), C.c_uint64()
        check(self._lib.pppm_server_stats(self._h, C.byref(rb), C.byref(done)), "pppm_server_stats")
        return {"resident_bytes": rb.value, "completed": done.value}
