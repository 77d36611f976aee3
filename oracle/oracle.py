"""Test infrastructure only: ctypes loaders for the two CPU oracles.

  restatement  oracle/_build/liborestate.so  (plain C, oracle/restate.c)
  reference    oracle/_ref/libpderef.so      (the reference's own CPU solver,
                                              built from its sources by oracle/Makefile)

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from pde_solver_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATE_SO = os.path.join(HERE, "_build", "liborestate.so")
REF_SO = os.path.join(HERE, "_ref", "libpderef.so")

P = C.POINTER
DP = P(C.c_double)


def _makefile_ref() -> str:
    """The reference source tree oracle/Makefile compiles by default (its `REF ?=` line)."""
    with open(os.path.join(HERE, "Makefile")) as fh:
        for line in fh:
            if line.startswith("REF ?="):
                return line.split("=", 1)[1].strip()
    return ""


# Where the reference's sources lie: $PDE_SOLVER_REF, else the Makefile's default.
REF_SRC = os.environ.get("PDE_SOLVER_REF") or _makefile_ref()


def have_reference_sources() -> bool:
    """True where the reference's CPU solver sources can be compiled (not on a box without them)."""
    return bool(REF_SRC) and os.path.exists(os.path.join(REF_SRC, "src", "backends", "cpu", "solver.cpp"))


def build(ref: bool = True) -> None:
    """make -C oracle (restatement always; the reference when its sources exist)."""
    target = "all" if ref else "restate"
    subprocess.run(["make", "-s", "-C", HERE, "-j8", target, f"REF={REF_SRC}"], check=True)


_restate = None
_ref = None


def restate() -> C.CDLL:
    global _restate
    if _restate is None:
        if not os.path.exists(RESTATE_SO):
            build(ref=False)
        lib = C.CDLL(RESTATE_SO)
        lib.rs_solve.restype = C.c_int
        lib.rs_solve.argtypes = [P(abi.Problem), P(abi.Options), DP, P(abi.Report)]
        lib.rs_apply.restype = C.c_int
        lib.rs_apply.argtypes = [P(abi.Problem), DP, DP]
        lib.rs_residual_norms.restype = C.c_int
        lib.rs_residual_norms.argtypes = [P(abi.Problem), DP, DP, DP]
        lib.rs_time_series.restype = C.c_int
        lib.rs_time_series.argtypes = [P(abi.Problem), P(abi.TimeOptions), DP, DP]
        lib.rs_project.restype = C.c_int
        lib.rs_project.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                   C.c_double, DP, DP, DP, DP, P(abi.ProjectionOptions),
                                   P(abi.ProjectionReport)]
        lib.rs_folded_rhs.restype = C.c_int
        lib.rs_folded_rhs.argtypes = [P(abi.Problem), DP]
        lib.rs_folded_apply.restype = C.c_int
        lib.rs_folded_apply.argtypes = [P(abi.Problem), DP, DP]
        lib.rs_fill_boundary.restype = C.c_int
        lib.rs_fill_boundary.argtypes = [P(abi.Problem), DP]
        lib.rs_sizeof.restype = C.c_long
        lib.rs_sizeof.argtypes = [C.c_int]
        lib.rs_set_threads.restype = None
        lib.rs_set_threads.argtypes = [C.c_int]
        _restate = lib
    return _restate


def have_reference() -> bool:
    return os.path.exists(REF_SO)


def reference() -> C.CDLL:
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise RuntimeError("oracle/_ref/libpderef.so not built (needs the reference sources)")
        lib = C.CDLL(REF_SO)
        lib.pderef_solve.restype = C.c_int
        lib.pderef_solve.argtypes = [P(abi.Problem), C.c_char_p, P(C.c_char_p), P(abi.Options), DP,
                                     DP, DP, C.c_char_p, C.c_size_t]
        lib.pderef_time_series.restype = C.c_int
        lib.pderef_time_series.argtypes = [P(abi.Problem), C.c_char_p, C.c_double, C.c_double,
                                           C.c_int, DP, DP, C.c_char_p, C.c_size_t]
        lib.pderef_residual_norms.restype = C.c_int
        lib.pderef_residual_norms.argtypes = [P(abi.Problem), C.c_char_p, DP, DP, DP, C.c_char_p,
                                              C.c_size_t]
        lib.pderef_materialize.restype = C.c_int
        lib.pderef_materialize.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int] + [C.c_double] * 7 + [
            DP, C.c_char_p, C.c_size_t]
        lib.pderef_project.restype = C.c_int
        lib.pderef_project.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                       C.c_double, DP, DP, DP, DP, C.c_int, C.c_double, C.c_int, DP]
        lib.pderef_self_test.restype = C.c_int
        lib.pderef_write_vtk.restype = C.c_int
        lib.pderef_write_vtk.argtypes = [C.c_char_p, P(abi.Problem), DP, C.c_char_p, C.c_size_t]
        lib.pderef_write_vti.restype = C.c_int
        lib.pderef_write_vti.argtypes = [C.c_char_p, P(abi.Problem), DP, C.c_int, C.c_char_p, C.c_size_t]
        lib.pderef_set_threads.argtypes = [C.c_int]
        lib.pderef_max_threads.restype = C.c_int
        _ref = lib
    return _ref


def _dp(a):
    return a.ctypes.data_as(DP) if a is not None else None


# ---------------------------------------------------------------- helpers

def rs_solve(prob, opt):
    out = np.zeros(prob.n)
    rep = abi.Report()
    cp = prob.to_c()
    st = restate().rs_solve(C.byref(cp), C.byref(opt), _dp(out), C.byref(rep))
    return st, out, rep


def rs_apply(prob, x):
    y = np.zeros(prob.n)
    cp = prob.to_c()
    x = np.ascontiguousarray(x, dtype=np.float64)
    assert restate().rs_apply(C.byref(cp), _dp(x), _dp(y)) == 0
    return y


def rs_folded(prob, x=None):
    cp = prob.to_c()
    b = np.zeros(prob.n)
    assert restate().rs_folded_rhs(C.byref(cp), _dp(b)) == 0
    if x is None:
        return b
    y = np.zeros(prob.n)
    x = np.ascontiguousarray(x, dtype=np.float64)
    assert restate().rs_folded_apply(C.byref(cp), _dp(x), _dp(y)) == 0
    return b, y


def rs_residual_norms(prob, grid):
    cp = prob.to_c()
    l2, linf = C.c_double(), C.c_double()
    grid = np.ascontiguousarray(grid, dtype=np.float64)
    assert restate().rs_residual_norms(C.byref(cp), _dp(grid), C.byref(l2), C.byref(linf)) == 0
    return l2.value, linf.value


def rs_time_series(prob, t_start, dt, frames, keep_frames=False):
    cp = prob.to_c()
    to = abi.TimeOptions(t_start=t_start, dt=dt, frames=frames, frame_stride=1)
    out = np.zeros(prob.n)
    fr = np.zeros(prob.n * frames) if keep_frames else None
    st = restate().rs_time_series(C.byref(cp), C.byref(to), _dp(out), _dp(fr))
    assert st == 0
    return (out, fr.reshape(frames, -1)) if keep_frames else out


def rs_project(u, v, w, p, nx, ny, nz, dx, dy, dz, dt, max_iter=1000, tol=1e-8, fix_corner=1):
    u, v, p = (np.array(a, dtype=np.float64) for a in (u, v, p))
    w = np.array(w, dtype=np.float64) if w is not None else np.zeros(1)
    po = abi.ProjectionOptions(max_iter=max_iter, fix_pressure_corner=fix_corner, tol=tol)
    rep = abi.ProjectionReport()
    st = restate().rs_project(nx, ny, nz, dx, dy, dz, dt, _dp(u), _dp(v), _dp(w), _dp(p),
                              C.byref(po), C.byref(rep))
    return st, u, v, w, p, rep


def ref_solve(prob, opt, rhs_latex=None, coef_latex=None):
    out = np.zeros(prob.n)
    l2, linf = C.c_double(), C.c_double()
    err = C.create_string_buffer(512)
    cl = None
    if coef_latex is not None:
        arr = (C.c_char_p * 7)(*[(s.encode() if s else None) for s in coef_latex])
        cl = C.cast(arr, P(C.c_char_p))
    cp = prob.to_c()
    st = reference().pderef_solve(C.byref(cp), rhs_latex.encode() if rhs_latex else None, cl,
                                  C.byref(opt), _dp(out), C.byref(l2), C.byref(linf), err, 512)
    return st, out, (l2.value, linf.value), err.value.decode()


def ref_time_series(prob, t_start, dt, frames, rhs_latex=None, keep_frames=False):
    out = np.zeros(prob.n)
    fr = np.zeros(prob.n * frames) if keep_frames else None
    err = C.create_string_buffer(512)
    cp = prob.to_c()
    st = reference().pderef_time_series(C.byref(cp), rhs_latex.encode() if rhs_latex else None,
                                        t_start, dt, frames, _dp(out), _dp(fr), err, 512)
    if st != 0:
        raise RuntimeError(err.value.decode())
    return (out, fr.reshape(frames, -1)) if keep_frames else out


def ref_residual_norms(prob, grid, rhs_latex=None):
    l2, linf = C.c_double(), C.c_double()
    err = C.create_string_buffer(512)
    grid = np.ascontiguousarray(grid, dtype=np.float64)
    cp = prob.to_c()
    st = reference().pderef_residual_norms(C.byref(cp), rhs_latex.encode() if rhs_latex else None,
                                           _dp(grid), C.byref(l2), C.byref(linf), err, 512)
    if st != 0:
        raise RuntimeError(err.value.decode())
    return l2.value, linf.value


def ref_materialize(latex, prob, t=0.0):
    out = np.zeros(prob.n)
    err = C.create_string_buffer(512)
    b = prob.bounds
    st = reference().pderef_materialize(latex.encode(), prob.nx, prob.ny, prob.nz, *b, t, _dp(out), err, 512)
    if st != 0:
        raise RuntimeError(err.value.decode())
    return out


def ref_write_vtk(path, prob, grid):
    """WriteVtkStructuredPoints (src/vtk_writer.cpp:28-82) of `grid` on prob's geometry."""
    grid = np.ascontiguousarray(grid, dtype=np.float64)
    err = C.create_string_buffer(256)
    cp = prob.to_c()
    if reference().pderef_write_vtk(str(path).encode(), C.byref(cp), _dp(grid), err, 256) != 0:
        raise RuntimeError(err.value.decode())


def ref_write_vti(path, prob, grid, derived=True):
    """WriteVtkXmlImageData (src/vtk_writer.cpp:176-268) with the CLI's derived fields."""
    grid = np.ascontiguousarray(grid, dtype=np.float64)
    err = C.create_string_buffer(256)
    cp = prob.to_c()
    if reference().pderef_write_vti(str(path).encode(), C.byref(cp), _dp(grid), 1 if derived else 0, err, 256) != 0:
        raise RuntimeError(err.value.decode())


def ref_project(u, v, w, p, nx, ny, nz, dx, dy, dz, dt, max_iter=1000, tol=1e-8, fix_corner=1):
    u, v, p = (np.array(a, dtype=np.float64) for a in (u, v, p))
    w = np.array(w, dtype=np.float64) if w is not None else np.zeros(1)
    rep = np.zeros(6)
    st = reference().pderef_project(nx, ny, nz, dx, dy, dz, dt, _dp(u), _dp(v), _dp(w), _dp(p),
                                    max_iter, tol, fix_corner, _dp(rep))
    return st, u, v, w, p, rep


# ------------------------------------------------------------ drop-in harness

DROPIN_SO = os.path.join(HERE, "_ref", "libdropin.so")
_dropin = None


def have_dropin() -> bool:
    return os.path.exists(DROPIN_SO)


def dropin() -> C.CDLL:
    """oracle/_ref/libdropin.so: the reference's SolveWithBackend with its CUDA
    backend served by pde_solver_b200/shim/cuda_solver_shim.cpp."""
    global _dropin
    if _dropin is None:
        lib = C.CDLL(DROPIN_SO)
        cpp = P(C.c_char_p)
        lib.dropin_solve_with_backend.restype = C.c_int
        lib.dropin_solve_with_backend.argtypes = [P(abi.Problem), C.c_char_p, cpp, cpp, P(abi.Options), C.c_int, DP,
                                                  DP, DP, P(C.c_int), C.c_char_p, C.c_size_t]
        lib.dropin_solve_cuda.restype = C.c_int
        lib.dropin_solve_cuda.argtypes = [P(abi.Problem), C.c_char_p, cpp, cpp, P(abi.Options), DP, C.c_char_p,
                                          C.c_size_t]
        lib.dropin_time_series_cuda.restype = C.c_int
        lib.dropin_time_series_cuda.argtypes = [P(abi.Problem), C.c_char_p, C.c_double, C.c_double, C.c_int, DP, DP,
                                                C.c_char_p, C.c_size_t]
        lib.dropin_probe.restype = C.c_int
        lib.dropin_probe.argtypes = [C.c_char_p, C.c_size_t]
        _dropin = lib
    return _dropin


def _cstrs(items, count):
    if items is None:
        return None
    arr = (C.c_char_p * count)(*[(s.encode() if s else None) for s in items])
    return C.cast(arr, P(C.c_char_p))


def dropin_solve(prob, opt, backend, rhs_latex=None, coef_latex=None, face_latex=None):
    """backend 1 = CUDA (the B200 shim), 0 = CPU; returns (status, grid, (l2, linf), selected_cuda, error)."""
    out = np.zeros(prob.n)
    l2, linf = C.c_double(), C.c_double()
    sel = C.c_int(-1)
    err = C.create_string_buffer(512)
    cp = prob.to_c()
    st = dropin().dropin_solve_with_backend(C.byref(cp), rhs_latex.encode() if rhs_latex else None,
                                            _cstrs(coef_latex, 7), _cstrs(face_latex, 6), C.byref(opt), backend,
                                            _dp(out), C.byref(l2), C.byref(linf), C.byref(sel), err, 512)
    return st, out, (l2.value, linf.value), sel.value == 1, err.value.decode()


def dropin_solve_cuda(prob, opt, rhs_latex=None, coef_latex=None, face_latex=None):
    out = np.zeros(prob.n)
    err = C.create_string_buffer(512)
    cp = prob.to_c()
    st = dropin().dropin_solve_cuda(C.byref(cp), rhs_latex.encode() if rhs_latex else None, _cstrs(coef_latex, 7),
                                    _cstrs(face_latex, 6), C.byref(opt), _dp(out), err, 512)
    return st, out, err.value.decode()


def dropin_time_series_cuda(prob, t_start, dt, frames, rhs_latex=None):
    out = np.zeros(prob.n)
    fr = np.zeros(prob.n * frames)
    err = C.create_string_buffer(512)
    cp = prob.to_c()
    st = dropin().dropin_time_series_cuda(C.byref(cp), rhs_latex.encode() if rhs_latex else None, t_start, dt, frames,
                                          _dp(out), _dp(fr), err, 512)
    return st, out, fr.reshape(frames, -1), err.value.decode()
