"""Serving loop (include/pdeb200_server.h): submit Poisson / heat / projection
requests as they arrive; the library admits them against an HBM budget and
runs them concurrently on several lanes, batching mixed-precision Poisson
requests that wait together.

    with Server(lanes=4) as s:
        rid = s.submit_poisson(problem)          # returns at once
        u, res = s.wait(rid)                      # solution and timing record
        print(s.stats().p99_ms)

`single_below=n` (MIXED only): while fewer than n Poisson requests wait, a
free lane solves one on its own grid in mixed precision instead of as a
batched group (lower latency at light load; results then agree with a
batched solve to the tolerance rather than bitwise).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .batch import default_options as batch_default_options


class ServerError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{message} (status {status})")
        self.status = status


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Server:
    def __init__(self, lanes=4, max_batch=64, precision=abi.MIXED, hbm_budget_bytes=0, device=0,
                 queue_capacity=0, single_below=0, **batch_kw):
        self.lib = abi.load()
        o = abi.ServerOptions()
        o.device, o.lanes, o.max_batch, o.precision = device, lanes, max_batch, precision
        o.hbm_budget_bytes, o.queue_capacity = hbm_budget_bytes, queue_capacity
        o.single_below = single_below
        o.batch = batch_default_options(**batch_kw)
        self._h = C.c_void_p()
        msg = C.create_string_buffer(512)
        st = self.lib.pdeb200_server_create(C.byref(o), C.byref(self._h), msg, len(msg))
        if st != abi.OK:
            raise ServerError(st, msg.value.decode(errors="replace"))
        self._out = {}

    def _submit(self, req, out, keep):
        rid = C.c_int64()
        # a device result buffer is passed as an int (device pointer)
        req.out = C.cast(C.c_void_p(out), C.POINTER(C.c_double)) if isinstance(out, int) else _dp(out)
        st = self.lib.pdeb200_server_submit(self._h, C.byref(req), C.byref(rid))
        if st != abi.OK:
            raise ServerError(st, "submit refused")
        self._out[rid.value] = (out, keep)
        return rid.value

    def submit_poisson(self, problem, tol=1e-10, out=None):
        """Device-resident problems (mem_space MEM_DEVICE) need `out`, a device
        pointer for the result; their arrays must outlive the request."""
        cp = problem.to_c()
        req = abi.Request()
        req.kind = abi.REQ_POISSON
        req.problem = C.pointer(cp)
        req.tol = tol
        if problem.mem_space == abi.MEM_DEVICE:
            if out is None:
                raise ValueError("device-resident requests need a device result pointer")
            return self._submit(req, int(out), (problem, cp))
        return self._submit(req, np.empty(problem.n) if out is None else out, (problem, cp))

    def submit_heat(self, problem, dt, steps, t_start=0.0):
        cp = problem.to_c()
        req = abi.Request()
        req.kind = abi.REQ_HEAT
        req.problem = C.pointer(cp)
        req.dt, req.steps, req.t_start = dt, steps, t_start
        return self._submit(req, np.empty(problem.n), (problem, cp))

    def submit_projection(self, u, v, w, p, nx, ny, nz, dx, dy, dz, dt, max_iter=10000, tol=1e-10):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, p)]
        wa = np.ascontiguousarray(w, dtype=np.float64) if w is not None else None
        req = abi.Request()
        req.kind = abi.REQ_PROJECTION
        req.nx, req.ny, req.nz, req.max_iter = nx, ny, nz, max_iter
        req.dx, req.dy, req.dz, req.proj_dt, req.proj_tol = dx, dy, dz, dt, tol
        req.u, req.v, req.p = _dp(arrs[0]), _dp(arrs[1]), _dp(arrs[2])
        if wa is not None:
            req.w = _dp(wa)
        n = nx * ny * max(nz, 1)
        nf = 4 if nz > 1 else 3
        return self._submit(req, np.empty(nf * n), (arrs, wa))

    def wait(self, rid, timeout_ms=-1.0):
        res = abi.Result()
        st = self.lib.pdeb200_server_wait(self._h, rid, timeout_ms, C.byref(res))
        if st == abi.ERR_TIMEOUT:
            return None, None
        out, _ = self._out.pop(rid)
        return out, res

    def drain(self, timeout_ms=-1.0):
        return self.lib.pdeb200_server_drain(self._h, timeout_ms)

    def stats(self, reset=False) -> abi.ServerStats:
        s = abi.ServerStats()
        self.lib.pdeb200_server_get_stats(self._h, C.byref(s), 1 if reset else 0)
        return s

    def close(self):
        if self._h:
            self.lib.pdeb200_server_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
