"""Python host API over the C ABI (include/pdeb200.h).

Mirrors the reference's solve entry (SolveWithBackend / SolvePDECuda,
src/backend_solve.cpp:53, src/backends/cuda/CudaSolve.cu:31): a problem and
solver options in, the full grid field out, errors as a status and message.
Every call goes through libpdeb200.so; there is no other implementation.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .problem import GridProblem, default_options


class SolveError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"[{status}] {message}")
        self.status = status
        self.message = message


def _lib():
    return abi.load()


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def solve(problem: GridProblem, options: abi.Options | None = None, out=None, raise_on_error=True, **kw):
    """Steady solve. Returns (field, report). With MEM_DEVICE problems `out`
    must be a device pointer (int) and is returned as given."""
    lib = _lib()
    opt = options if options is not None else default_options(**kw)
    rep = abi.Report()
    cp = problem.to_c()
    if problem.mem_space == abi.MEM_DEVICE:
        assert out is not None, "device problems need a device output pointer"
        st = lib.pdeb200_solve(C.byref(cp), C.byref(opt), C.c_void_p(out), C.byref(rep))
        res = out
    else:
        res = np.empty(problem.n) if out is None else out
        st = lib.pdeb200_solve(C.byref(cp), C.byref(opt), res.ctypes.data_as(C.c_void_p), C.byref(rep))
    if st != abi.OK and raise_on_error and st != abi.ERR_NOT_CONVERGED:
        raise SolveError(st, rep.message.decode() or lib.pdeb200_status_string(st).decode())
    rep.status = st
    return res, rep


def apply(problem: GridProblem, x, device: int = 0):
    lib = _lib()
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    cp = problem.to_c()
    st = lib.pdeb200_apply(C.byref(cp), x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p), device)
    if st != abi.OK:
        raise SolveError(st, lib.pdeb200_status_string(st).decode())
    return y


def residual_norms(problem: GridProblem, grid, device: int = 0):
    lib = _lib()
    grid = np.ascontiguousarray(grid, dtype=np.float64)
    l2, linf = C.c_double(), C.c_double()
    cp = problem.to_c()
    st = lib.pdeb200_residual_norms(C.byref(cp), grid.ctypes.data_as(C.c_void_p), device, C.byref(l2), C.byref(linf))
    if st != abi.OK:
        raise SolveError(st, lib.pdeb200_status_string(st).decode())
    return l2.value, linf.value


def eval_expression(latex: str, problem: GridProblem, t: float = 0.0, device: int = 0, out=None):
    """The LaTeX expression at every node of `problem`'s grid, computed on the
    GPU (ExpressionEvaluator::Eval per node, src/expression_eval.cpp:841-978).
    Host array result unless `out` is a device pointer (int)."""
    lib = _lib()
    cp = problem.to_c()
    msg = C.create_string_buffer(256)
    if out is not None and not isinstance(out, np.ndarray):
        st = lib.pdeb200_eval_expression(latex.encode(), C.byref(cp), t, device, C.c_void_p(out), abi.MEM_DEVICE,
                                         msg, 256)
        res = out
    else:
        res = np.empty(problem.n) if out is None else out
        st = lib.pdeb200_eval_expression(latex.encode(), C.byref(cp), t, device, res.ctypes.data_as(C.c_void_p),
                                         abi.MEM_HOST, msg, 256)
    if st != abi.OK:
        raise SolveError(st, msg.value.decode() or lib.pdeb200_status_string(st).decode())
    return res


def eval_face_expression(latex: str | None, problem: GridProblem, face: int, linear=(0.0, 0.0, 0.0, 0.0),
                         t: float = 0.0, device: int = 0):
    """A boundary expression on the nodes of one face in pdeb200_face order,
    with the reference's EvalExpr fallback to the linear form
    (src/backends/cpu/cpu_utils.cpp:520-530)."""
    lib = _lib()
    cp = problem.to_c()
    msg = C.create_string_buffer(256)
    nx, ny, nz = problem.nx, problem.ny, max(problem.nz, 1)
    n = (ny * nz) if face <= 1 else (nx * nz if face <= 3 else nx * ny)
    res = np.empty(n)
    lin = (C.c_double * 4)(*[float(v) for v in linear])
    st = lib.pdeb200_eval_face_expression(latex.encode() if latex is not None else None, lin, C.byref(cp), face, t,
                                          device, res.ctypes.data_as(C.c_void_p), abi.MEM_HOST, msg, 256)
    if st != abi.OK:
        raise SolveError(st, msg.value.decode() or lib.pdeb200_status_string(st).decode())
    return res


def _write(fn, path, problem, field, extra, device, progress):
    lib = _lib()
    cp = problem.to_c()
    msg = C.create_string_buffer(256)
    cb = abi.WRITE_PROGRESS(lambda f, u: progress(f)) if progress else abi.WRITE_PROGRESS()
    if isinstance(field, np.ndarray):
        field = np.ascontiguousarray(field, dtype=np.float64)
        ptr, mem = field.ctypes.data_as(C.c_void_p), abi.MEM_HOST
    else:
        ptr, mem = C.c_void_p(field), abi.MEM_DEVICE
    st = getattr(lib, fn)(str(path).encode(), C.byref(cp), ptr, *extra, mem, device, cb, None, msg, 256)
    if st != abi.OK:
        raise SolveError(st, msg.value.decode() or lib.pdeb200_status_string(st).decode())


def write_vtk(path, problem: GridProblem, field, device: int = 0, progress=None):
    """Legacy ASCII VTK file of `field` (host array, or device pointer as int),
    byte-identical to WriteVtkStructuredPoints (src/vtk_writer.cpp:28-82);
    formatted on the GPU."""
    _write("pdeb200_write_vtk", path, problem, field, (), device, progress)


def write_vti(path, problem: GridProblem, field, derived: bool = True, device: int = 0, progress=None):
    """VTK XML ImageData file (base64 Float32), byte-identical to
    WriteVtkXmlImageData (src/vtk_writer.cpp:176-268) with the derived fields
    the reference CLI adds (flux coefficients problem.a, problem.b, problem.az)."""
    _write("pdeb200_write_vti", path, problem, field, (1 if derived else 0,), device, progress)


def vtk_values_host(field, nx: int) -> bytes:
    """The legacy file's value text from the host copy of the GPU formatter."""
    lib = _lib()
    field = np.ascontiguousarray(field, dtype=np.float64)
    n = C.c_size_t()
    assert lib.pdeb200_vtk_values_host(field.ctypes.data_as(C.c_void_p), field.size, nx, None, 0, C.byref(n)) == 0
    buf = C.create_string_buffer(n.value)
    st = lib.pdeb200_vtk_values_host(field.ctypes.data_as(C.c_void_p), field.size, nx, buf, n.value, C.byref(n))
    assert st == abi.OK
    return buf.raw[:n.value]


def expression_value(latex: str, x: float, y: float, z: float = 0.0, t: float = 0.0) -> float:
    """One host evaluation of the compiled expression (no GPU needed)."""
    lib = _lib()
    v = C.c_double()
    msg = C.create_string_buffer(256)
    st = lib.pdeb200_expression_value(latex.encode(), x, y, z, t, C.byref(v), msg, 256)
    if st != abi.OK:
        raise SolveError(st, msg.value.decode())
    return v.value


def time_series(problem: GridProblem, t_start: float, dt: float, frames: int, on_frame=None, device: int = 0,
                frame_stride: int = 1):
    """Forward-Euler frames (SolvePDETimeSeries). on_frame(frame, t, grid) -> bool."""
    lib = _lib()
    to = abi.TimeOptions(t_start=t_start, dt=dt, frames=frames, frame_stride=frame_stride, device=device)
    out = np.empty(problem.n)
    n = problem.n

    def _cb(frame, t, ptr, user):
        if on_frame is None:
            return 1
        arr = np.ctypeslib.as_array(ptr, shape=(n,)).copy()
        return 1 if on_frame(frame, t, arr) is not False else 0

    cb = abi.FRAME_CB(_cb)
    rep = abi.Report()
    cp = problem.to_c()
    st = lib.pdeb200_time_series(C.byref(cp), C.byref(to), cb, None, out.ctypes.data_as(C.c_void_p), C.byref(rep))
    if st != abi.OK:
        raise SolveError(st, rep.message.decode() or lib.pdeb200_status_string(st).decode())
    return out, rep


def project_velocity(u, v, w, p, nx, ny, nz, dx, dy, dz, dt, max_iter=1000, tol=1e-8, fix_corner=True,
                     device=0):
    """ProjectVelocity2D/3D; arrays are updated copies (u, v, w, p, report)."""
    lib = _lib()
    u, v, p = (np.array(a, dtype=np.float64) for a in (u, v, p))
    w = np.array(w, dtype=np.float64) if w is not None else None
    po = abi.ProjectionOptions(max_iter=max_iter, fix_pressure_corner=int(fix_corner), tol=tol, device=device,
                               mem_space=abi.MEM_HOST)
    rep = abi.ProjectionReport()
    st = lib.pdeb200_project_velocity(nx, ny, nz, dx, dy, dz, dt, u.ctypes.data_as(C.c_void_p),
                                      v.ctypes.data_as(C.c_void_p),
                                      w.ctypes.data_as(C.c_void_p) if w is not None else None,
                                      p.ctypes.data_as(C.c_void_p), C.byref(po), C.byref(rep))
    rep.status = st
    return u, v, w, p, rep
