"""ctypes mirror of include/pdeb200.h (and pdeb200_batch.h, pdeb200_server.h)
and the loader for libpdeb200.so.

The structures here must stay byte-identical to the C header; tests check
their sizes against the library's own sizeof values (pdeb200_sizeof_*).
"""
from __future__ import annotations

import ctypes as C
import os

PDEB200_ABI_VERSION = 2

# pdeb200_status
OK, ERR_INVALID, ERR_UNSUPPORTED, ERR_NO_DEVICE, ERR_CUDA, ERR_OOM = 0, 1, 2, 3, 4, 5
ERR_NOT_CONVERGED, ERR_BREAKDOWN, ERR_DEGENERATE, ERR_CANCELLED, ERR_TIMEOUT, ERR_BUSY = 6, 7, 8, 9, 10, 11

# boundary kinds (BCKind order)
BC_DIRICHLET, BC_NEUMANN, BC_ROBIN = 0, 1, 2
# coefficient forms
COEF_CONST, COEF_DIVK, COEF_NODAL = 0, 1, 2
MEM_HOST, MEM_DEVICE = 0, 1
# methods (SolveMethod order, then the B200 forms)
JACOBI, GAUSS_SEIDEL, SOR, CG, BICGSTAB, GMRES, MG_VCYCLE, MG_PCG, MG_BICGSTAB = range(9)
TOL_REFERENCE, TOL_RELATIVE = 0, 1
FP64, MIXED = 0, 1
ORDER_LEXICOGRAPHIC, ORDER_REDBLACK = 0, 1
# pointwise nonlinear term kinds (NonlinearKind order)
NL_POWER, NL_SIN, NL_COS, NL_EXP, NL_ABS = range(5)
MAX_NONLINEAR = 8

FACE_NAMES = ("left", "right", "bottom", "top", "front", "back")


class Face(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("reserved", C.c_int32),
        ("value", C.c_double),
        ("alpha", C.c_double),
        ("beta", C.c_double),
        ("gamma", C.c_double),
        ("value_arr", C.POINTER(C.c_double)),
        ("alpha_arr", C.POINTER(C.c_double)),
        ("beta_arr", C.POINTER(C.c_double)),
        ("gamma_arr", C.POINTER(C.c_double)),
    ]


class NonlinearTerm(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("power", C.c_int32),
        ("coeff", C.c_double),
    ]


class Problem(C.Structure):
    _fields_ = [
        ("nx", C.c_int32),
        ("ny", C.c_int32),
        ("nz", C.c_int32),
        ("coef_kind", C.c_int32),
        ("mem_space", C.c_int32),
        ("reserved", C.c_int32),
        ("xmin", C.c_double),
        ("xmax", C.c_double),
        ("ymin", C.c_double),
        ("ymax", C.c_double),
        ("zmin", C.c_double),
        ("zmax", C.c_double),
        ("a", C.c_double),
        ("b", C.c_double),
        ("az", C.c_double),
        ("c", C.c_double),
        ("d", C.c_double),
        ("dz", C.c_double),
        ("e", C.c_double),
        ("f_const", C.c_double),
        ("ut", C.c_double),
        ("k", C.POINTER(C.c_double)),
        ("nodal", C.POINTER(C.c_double)),
        ("f", C.POINTER(C.c_double)),
        ("u0", C.POINTER(C.c_double)),
        ("face", Face * 6),
        ("n_nonlinear", C.c_int32),
        ("reserved2", C.c_int32),
        ("nonlinear", C.POINTER(NonlinearTerm)),
    ]


class Options(C.Structure):
    _fields_ = [
        ("method", C.c_int32),
        ("max_iter", C.c_int32),
        ("tol", C.c_double),
        ("tol_mode", C.c_int32),
        ("precision", C.c_int32),
        ("sor_omega", C.c_double),
        ("gmres_restart", C.c_int32),
        ("mg_pre_smooth", C.c_int32),
        ("mg_post_smooth", C.c_int32),
        ("mg_coarse_iters", C.c_int32),
        ("mg_max_levels", C.c_int32),
        ("gs_ordering", C.c_int32),
        ("device", C.c_int32),
        ("check_interval", C.c_int32),
        ("inner_tol", C.c_double),
        ("bf16_coefficients", C.c_int32),
        ("max_outer", C.c_int32),
        ("cancel", C.POINTER(C.c_int32)),
    ]


class Report(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32),
        ("outer_iterations", C.c_int32),
        ("converged", C.c_int32),
        ("kernel_launches", C.c_int32),
        ("residual_l2", C.c_double),
        ("rhs_l2", C.c_double),
        ("rel_residual", C.c_double),
        ("last_delta", C.c_double),
        ("device_ms", C.c_double),
        ("total_ms", C.c_double),
        ("message", C.c_char * 256),
    ]


class TimeOptions(C.Structure):
    _fields_ = [
        ("t_start", C.c_double),
        ("dt", C.c_double),
        ("frames", C.c_int32),
        ("frame_stride", C.c_int32),
        ("device", C.c_int32),
        ("reserved", C.c_int32),
    ]


class ProjectionOptions(C.Structure):
    _fields_ = [
        ("max_iter", C.c_int32),
        ("fix_pressure_corner", C.c_int32),
        ("tol", C.c_double),
        ("reference_pressure", C.c_double),
        ("device", C.c_int32),
        ("mem_space", C.c_int32),
    ]


class ProjectionReport(C.Structure):
    _fields_ = [
        ("success", C.c_int32),
        ("poisson_iterations", C.c_int32),
        ("poisson_residual", C.c_double),
        ("max_divergence_before", C.c_double),
        ("max_divergence_after", C.c_double),
        ("l2_divergence_before", C.c_double),
        ("l2_divergence_after", C.c_double),
        ("device_ms", C.c_double),
        ("message", C.c_char * 256),
    ]


class KernelStat(C.Structure):
    _fields_ = [
        ("name", C.c_char * 48),
        ("launches", C.c_int64),
        ("total_ms", C.c_double),
        ("bytes_per_launch", C.c_double),
    ]


class BatchOptions(C.Structure):
    """pdeb200_batch_options (include/pdeb200_batch.h)."""
    _fields_ = [
        ("device", C.c_int32),
        ("tile_x", C.c_int32),
        ("tile_y", C.c_int32),
        ("tile_z", C.c_int32),
        ("pre_smooth", C.c_int32),
        ("post_smooth", C.c_int32),
        ("coarse_sweeps", C.c_int32),
        ("max_inner", C.c_int32),
        ("max_outer", C.c_int32),
        ("bf16_coefficients", C.c_int32),
        ("no_graph", C.c_int32),
        ("autotune", C.c_int32),
        ("inner_tol", C.c_double),
        ("tune_cache", C.c_char_p),
        ("stream", C.c_void_p),
        ("no_compact", C.c_int32),
        ("reserved", C.c_int32 * 7),
    ]


class BatchStats(C.Structure):
    """pdeb200_batch_stats (include/pdeb200_batch.h)."""
    _fields_ = [
        ("members", C.c_int32),
        ("converged", C.c_int32),
        ("cycles", C.c_int32),
        ("max_levels", C.c_int32),
        ("kernel_launches", C.c_int64),
        ("tiles_level0", C.c_int64),
        ("nodes", C.c_int64),
        ("device_bytes", C.c_int64),
        ("device_ms", C.c_double),
        ("tune_ms", C.c_double),
        ("tuned_from_cache", C.c_int32),
        ("graph", C.c_int32),
        ("compactions", C.c_int32),
        ("reserved", C.c_int32 * 5),
    ]


REQ_POISSON, REQ_HEAT, REQ_PROJECTION = 0, 1, 2


class ServerOptions(C.Structure):
    """pdeb200_server_options (include/pdeb200_server.h)."""
    _fields_ = [
        ("device", C.c_int32),
        ("lanes", C.c_int32),
        ("max_batch", C.c_int32),
        ("precision", C.c_int32),
        ("hbm_budget_bytes", C.c_int64),
        ("queue_capacity", C.c_int32),
        ("single_below", C.c_int32),
        ("batch", BatchOptions),
        ("reserved", C.c_int32 * 8),
    ]


class Request(C.Structure):
    """pdeb200_request (include/pdeb200_server.h)."""
    _fields_ = [
        ("kind", C.c_int32),
        ("steps", C.c_int32),
        ("problem", C.POINTER(Problem)),
        ("tol", C.c_double),
        ("t_start", C.c_double),
        ("dt", C.c_double),
        ("nx", C.c_int32),
        ("ny", C.c_int32),
        ("nz", C.c_int32),
        ("max_iter", C.c_int32),
        ("dx", C.c_double),
        ("dy", C.c_double),
        ("dz", C.c_double),
        ("proj_dt", C.c_double),
        ("proj_tol", C.c_double),
        ("u", C.POINTER(C.c_double)),
        ("v", C.POINTER(C.c_double)),
        ("w", C.POINTER(C.c_double)),
        ("p", C.POINTER(C.c_double)),
        ("out", C.POINTER(C.c_double)),
    ]


class Result(C.Structure):
    """pdeb200_result (include/pdeb200_server.h)."""
    _fields_ = [
        ("id", C.c_int64),
        ("status", C.c_int32),
        ("kind", C.c_int32),
        ("queue_ms", C.c_double),
        ("run_ms", C.c_double),
        ("latency_ms", C.c_double),
        ("iterations", C.c_int32),
        ("group_size", C.c_int32),
        ("rel_residual", C.c_double),
        ("message", C.c_char * 128),
    ]


class ServerStats(C.Structure):
    """pdeb200_server_stats (include/pdeb200_server.h)."""
    _fields_ = [
        ("submitted", C.c_int64),
        ("completed", C.c_int64),
        ("failed", C.c_int64),
        ("rejected", C.c_int64),
        ("in_flight", C.c_int64),
        ("queued", C.c_int64),
        ("bytes_in_use", C.c_int64),
        ("bytes_peak", C.c_int64),
        ("budget_bytes", C.c_int64),
        ("lanes_busy_peak", C.c_int32),
        ("reserved0", C.c_int32),
        ("p50_ms", C.c_double),
        ("p99_ms", C.c_double),
        ("max_ms", C.c_double),
        ("elapsed_s", C.c_double),
        ("solves_per_s", C.c_double),
        ("reserved", C.c_int32 * 8),
    ]


WRITE_PROGRESS = C.CFUNCTYPE(None, C.c_double, C.c_void_p)
FRAME_CB = C.CFUNCTYPE(C.c_int32, C.c_int32, C.c_double, C.POINTER(C.c_double), C.c_void_p)

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libpdeb200.so")

_LIB = None


def declare(lib: C.CDLL) -> C.CDLL:
    """Attach argtypes/restype of every exported entry point."""
    P = C.POINTER
    lib.pdeb200_abi_version.restype = C.c_int32
    lib.pdeb200_abi_version.argtypes = []
    lib.pdeb200_probe.restype = C.c_int32
    lib.pdeb200_probe.argtypes = [C.c_char_p, C.c_size_t]
    lib.pdeb200_status_string.restype = C.c_char_p
    lib.pdeb200_status_string.argtypes = [C.c_int32]
    lib.pdeb200_default_options.restype = None
    lib.pdeb200_default_options.argtypes = [P(Options)]
    lib.pdeb200_release_all.restype = None
    lib.pdeb200_release_all.argtypes = []
    lib.pdeb200_solve.restype = C.c_int32
    lib.pdeb200_solve.argtypes = [P(Problem), P(Options), C.c_void_p, P(Report)]
    lib.pdeb200_residual_norms.restype = C.c_int32
    lib.pdeb200_residual_norms.argtypes = [P(Problem), C.c_void_p, C.c_int32, P(C.c_double), P(C.c_double)]
    lib.pdeb200_apply.restype = C.c_int32
    lib.pdeb200_apply.argtypes = [P(Problem), C.c_void_p, C.c_void_p, C.c_int32]
    lib.pdeb200_time_series.restype = C.c_int32
    lib.pdeb200_time_series.argtypes = [P(Problem), P(TimeOptions), FRAME_CB, C.c_void_p, C.c_void_p, P(Report)]
    lib.pdeb200_project_velocity.restype = C.c_int32
    lib.pdeb200_project_velocity.argtypes = [
        C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double,
        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, P(ProjectionOptions), P(ProjectionReport)]
    lib.pdeb200_set_stream.restype = C.c_int32
    lib.pdeb200_set_stream.argtypes = [C.c_int32, C.c_void_p]
    lib.pdeb200_profile_enable.restype = None
    lib.pdeb200_profile_enable.argtypes = [C.c_int32, C.c_int32]
    lib.pdeb200_profile_read.restype = C.c_int32
    lib.pdeb200_profile_read.argtypes = [C.c_int32, P(KernelStat), C.c_int32]
    lib.pdeb200_jacobi_noalloc.restype = C.c_int32
    lib.pdeb200_jacobi_noalloc.argtypes = [P(Problem), C.c_int32, C.c_double, C.c_int32, C.c_void_p, C.c_void_p,
                                           P(Report)]
    lib.pdeb200_eval_expression.restype = C.c_int32
    lib.pdeb200_eval_expression.argtypes = [C.c_char_p, P(Problem), C.c_double, C.c_int32, C.c_void_p, C.c_int32,
                                            C.c_char_p, C.c_size_t]
    lib.pdeb200_eval_face_expression.restype = C.c_int32
    lib.pdeb200_eval_face_expression.argtypes = [C.c_char_p, P(C.c_double), P(Problem), C.c_int32, C.c_double,
                                                 C.c_int32, C.c_void_p, C.c_int32, C.c_char_p, C.c_size_t]
    lib.pdeb200_write_vtk.restype = C.c_int32
    lib.pdeb200_write_vtk.argtypes = [C.c_char_p, P(Problem), C.c_void_p, C.c_int32, C.c_int32, WRITE_PROGRESS,
                                      C.c_void_p, C.c_char_p, C.c_size_t]
    lib.pdeb200_write_vti.restype = C.c_int32
    lib.pdeb200_write_vti.argtypes = [C.c_char_p, P(Problem), C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                                      WRITE_PROGRESS, C.c_void_p, C.c_char_p, C.c_size_t]
    lib.pdeb200_vtk_values_host.restype = C.c_int32
    lib.pdeb200_vtk_values_host.argtypes = [C.c_void_p, C.c_int64, C.c_int32, C.c_char_p, C.c_size_t,
                                            P(C.c_size_t)]
    lib.pdeb200_expression_value.restype = C.c_int32
    lib.pdeb200_expression_value.argtypes = [C.c_char_p, C.c_double, C.c_double, C.c_double, C.c_double,
                                             P(C.c_double), C.c_char_p, C.c_size_t]
    lib.pdeb200_batch_default_options.restype = None
    lib.pdeb200_batch_default_options.argtypes = [P(BatchOptions)]
    lib.pdeb200_batch_create.restype = C.c_int32
    lib.pdeb200_batch_create.argtypes = [P(Problem), C.c_int32, P(BatchOptions), P(C.c_void_p), C.c_char_p,
                                         C.c_size_t]
    lib.pdeb200_batch_nodes.restype = C.c_int64
    lib.pdeb200_batch_nodes.argtypes = [C.c_void_p]
    lib.pdeb200_batch_offset.restype = C.c_int64
    lib.pdeb200_batch_offset.argtypes = [C.c_void_p, C.c_int32]
    lib.pdeb200_batch_load_rhs.restype = C.c_int32
    lib.pdeb200_batch_load_rhs.argtypes = [C.c_void_p, C.c_void_p, C.c_int32]
    lib.pdeb200_batch_solve.restype = C.c_int32
    lib.pdeb200_batch_solve.argtypes = [C.c_void_p, C.c_double, P(Report), P(BatchStats)]
    lib.pdeb200_batch_read.restype = C.c_int32
    lib.pdeb200_batch_read.argtypes = [C.c_void_p, C.c_void_p, C.c_int32]
    lib.pdeb200_batch_read_member.restype = C.c_int32
    lib.pdeb200_batch_read_member.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32]
    lib.pdeb200_batch_get_options.restype = C.c_int32
    lib.pdeb200_batch_get_options.argtypes = [C.c_void_p, P(BatchOptions)]
    lib.pdeb200_batch_destroy.restype = None
    lib.pdeb200_batch_destroy.argtypes = [C.c_void_p]
    lib.pdeb200_server_create.restype = C.c_int32
    lib.pdeb200_server_create.argtypes = [P(ServerOptions), P(C.c_void_p), C.c_char_p, C.c_size_t]
    lib.pdeb200_server_submit.restype = C.c_int32
    lib.pdeb200_server_submit.argtypes = [C.c_void_p, P(Request), P(C.c_int64)]
    lib.pdeb200_server_wait.restype = C.c_int32
    lib.pdeb200_server_wait.argtypes = [C.c_void_p, C.c_int64, C.c_double, P(Result)]
    lib.pdeb200_server_drain.restype = C.c_int32
    lib.pdeb200_server_drain.argtypes = [C.c_void_p, C.c_double]
    lib.pdeb200_server_get_stats.restype = C.c_int32
    lib.pdeb200_server_get_stats.argtypes = [C.c_void_p, P(ServerStats), C.c_int32]
    lib.pdeb200_server_destroy.restype = None
    lib.pdeb200_server_destroy.argtypes = [C.c_void_p]
    return lib


def load(path: str | None = None) -> C.CDLL:
    """Load libpdeb200.so. Raises if the library has not been built: there is
    no fallback implementation."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"libpdeb200.so not built at {p}; run __graft_entry__.build()")
    lib = declare(C.CDLL(p))
    if lib.pdeb200_abi_version() != PDEB200_ABI_VERSION:
        raise RuntimeError("libpdeb200.so ABI version mismatch")
    if path is None:
        _LIB = lib
    return lib
