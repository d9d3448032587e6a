"""Served form: a request loop with continuous batching over resident
meshes (vfr_server_* in include/vfray.h).  Requests submitted from any
thread are admitted by memory footprint and folded into one running
persistent traversal launch, meshes and image sizes mixed; each completed
request carries its submit / admission / done times."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import Request, RequestInfo, ServerStats, check

__all__ = ["Server", "percentiles"]


class Server:
    def __init__(self, renderer, budget_bytes: int = 120 << 30, max_batch: int = 256):
        self.r = renderer
        self.lib = renderer.lib
        h = C.c_void_p()
        check(self.lib.vfr_server_create(renderer.h, budget_bytes, max_batch, C.byref(h)),
              renderer.h, "vfr_server_create")
        self.h = h
        self._outs = {}

    def submit(self, mesh_id: int, W: int, H: int, mv=None, mode: int = _lib.MODE_REF,
               out: np.ndarray | None = None) -> int:
        """Queue a request; the image lands in ``out`` (uint8 H x W x 3, kept
        alive here until ``wait``) or in a new array returned by ``wait``."""
        if out is None:
            out = np.empty((H, W, 3), np.uint8)
        assert out.dtype == np.uint8 and out.flags.c_contiguous and out.size == W * H * 3
        q = Request()
        q.mesh_id, q.W, q.H, q.mode = mesh_id, W, H, mode
        q.use_mv = 0 if mv is None else 1
        if mv is not None:
            m = np.ascontiguousarray(mv, np.float32).reshape(16)
            for k in range(16):
                q.mv[k] = float(m[k])
        q.rgb8_host = out.ctypes.data
        t = C.c_uint64()
        check(self.lib.vfr_server_submit(self.h, C.byref(q), C.byref(t)), None, "vfr_server_submit")
        self._outs[t.value] = out
        return int(t.value)

    def wait(self, ticket: int, timeout_ms: int = -1):
        """(image, info) of a request; raises VfrError on its status."""
        info = RequestInfo()
        rc = self.lib.vfr_server_wait(self.h, ticket, timeout_ms, C.byref(info))
        # after a timeout the request is still in flight and the server will
        # write its image later: its buffer stays referenced until a wait
        # that returns the request's own status
        if rc == _lib.VFR_ERR_TIMEOUT:
            out = self._outs.get(ticket)
        else:
            out = self._outs.pop(ticket, None)
        check(rc, None, "vfr_server_wait")
        return out, info.as_dict()

    def set_idle(self, drain_idle_us: int, linger_ms: int):
        """The drain's bounded idle wait (microseconds) and how long an
        idle drain runs before the server stops it."""
        check(self.lib.vfr_server_set_idle(self.h, drain_idle_us, linger_ms), None,
              "vfr_server_set_idle")

    def stats(self) -> dict:
        s = ServerStats()
        check(self.lib.vfr_server_stats(self.h, C.byref(s)), None, "vfr_server_stats")
        return s.as_dict()

    def close(self):
        if getattr(self, "h", None):
            self.lib.vfr_server_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def percentiles(latencies_ms, qs=(50, 99)):
    a = np.asarray(latencies_ms, np.float64)
    return {f"p{q}": float(np.percentile(a, q)) for q in qs} if len(a) else {}
