"""Batched solves of many independent grids (include/pdeb200_batch.h).

    b = Batch(problems, tile_y=16, autotune=False)
    reports = b.solve(1e-10)          # FP32 MG-PCG inside FP64 refinement
    fields = b.read()                 # list of flat arrays, one per member

There is no reference counterpart: the reference solves one SolveInput per
call. Every member reaches |b - A u| / |b| <= tol of its boundary-folded
system in FP64, and its result does not depend on the other members.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi


class BatchError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{message} (status {status})")
        self.status = status


def default_options(**kw) -> abi.BatchOptions:
    lib = abi.load()
    o = abi.BatchOptions()
    lib.pdeb200_batch_default_options(C.byref(o))
    for k, v in kw.items():
        if k == "tune_cache" and isinstance(v, str):
            v = v.encode()
        setattr(o, k, v)
    return o


class Batch:
    def __init__(self, problems, options: abi.BatchOptions | None = None, **kw):
        self.lib = abi.load()
        self.problems = list(problems)
        self._cprobs = (abi.Problem * len(self.problems))()
        for q, p in enumerate(self.problems):
            self._cprobs[q] = p.to_c()
        self._opts = options if options is not None else default_options(**kw)
        self._h = C.c_void_p()
        msg = C.create_string_buffer(512)
        st = self.lib.pdeb200_batch_create(self._cprobs, len(self.problems), C.byref(self._opts),
                                           C.byref(self._h), msg, len(msg))
        if st != abi.OK:
            raise BatchError(st, msg.value.decode(errors="replace"))
        self.nodes = int(self.lib.pdeb200_batch_nodes(self._h))
        self.offsets = [int(self.lib.pdeb200_batch_offset(self._h, q)) for q in range(len(self.problems))]
        self.stats = abi.BatchStats()

    @property
    def handle(self):
        return self._h

    def options(self) -> abi.BatchOptions:
        o = abi.BatchOptions()
        self.lib.pdeb200_batch_get_options(self._h, C.byref(o))
        return o

    def load_rhs(self, f_packed, mem_space=abi.MEM_HOST):
        if mem_space == abi.MEM_HOST:
            f = np.ascontiguousarray(f_packed, dtype=np.float64)
            assert f.size == self.nodes
            ptr = f.ctypes.data_as(C.c_void_p)
        else:
            ptr = C.c_void_p(int(f_packed))
        st = self.lib.pdeb200_batch_load_rhs(self._h, ptr, mem_space)
        if st != abi.OK:
            raise BatchError(st, "load_rhs failed")

    def solve(self, tol=1e-10, raise_on_error=True):
        reps = (abi.Report * len(self.problems))()
        st = self.lib.pdeb200_batch_solve(self._h, tol, reps, C.byref(self.stats))
        if st != abi.OK and raise_on_error:
            bad = [q for q in range(len(self.problems)) if not reps[q].converged]
            raise BatchError(st, f"{len(bad)} members did not converge, first {bad[:5]}: "
                                 f"{reps[bad[0]].message.decode(errors='replace') if bad else ''}")
        return list(reps)

    def read_packed(self, out=None):
        out = np.empty(self.nodes) if out is None else out
        st = self.lib.pdeb200_batch_read(self._h, out.ctypes.data_as(C.c_void_p), abi.MEM_HOST)
        if st != abi.OK:
            raise BatchError(st, "read failed")
        return out

    def read(self):
        flat = self.read_packed()
        return [flat[o:o + p.n].copy() for o, p in zip(self.offsets, self.problems)]

    def close(self):
        if self._h:
            self.lib.pdeb200_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
