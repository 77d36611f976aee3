"""Host-side problem description mirroring the reference's SolveInput fields
that reach the solve path (include/pde_types.h:10-58, 148-228, 282-303).

GridProblem holds numpy arrays and constants and produces the ctypes
`Problem` of include/pdeb200.h; the arrays stay referenced by the object so
the pointers handed to the library remain valid for its lifetime.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import abi


def _dptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


@dataclass
class FaceBC:
    """One face's boundary condition (BoundaryCondition, include/pde_types.h:181-196)."""
    kind: int = abi.BC_DIRICHLET
    value: float = 0.0
    alpha: float = 0.0
    beta: float = 0.0
    gamma: float = 0.0
    value_arr: np.ndarray | None = None
    alpha_arr: np.ndarray | None = None
    beta_arr: np.ndarray | None = None
    gamma_arr: np.ndarray | None = None

    @staticmethod
    def dirichlet(v=0.0):
        return FaceBC(abi.BC_DIRICHLET, value=v)

    @staticmethod
    def neumann(g=0.0):
        return FaceBC(abi.BC_NEUMANN, value=g)

    @staticmethod
    def robin(alpha, beta, gamma):
        return FaceBC(abi.BC_ROBIN, alpha=alpha, beta=beta, gamma=gamma)


@dataclass
class GridProblem:
    nx: int
    ny: int
    nz: int = 1
    bounds: tuple = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    a: float = 0.0
    b: float = 0.0
    az: float = 0.0
    c: float = 0.0
    d: float = 0.0
    dz: float = 0.0
    e: float = 0.0
    f_const: float = 0.0
    ut: float = 0.0
    coef_kind: int = abi.COEF_CONST
    k: np.ndarray | None = None
    nodal: np.ndarray | None = None
    f: np.ndarray | None = None
    u0: np.ndarray | None = None
    faces: list = field(default_factory=lambda: [FaceBC() for _ in range(6)])
    # pointwise nonlinear terms (NonlinearTerm, include/pde_types.h:96-100):
    # (kind, coeff, power) with kind one of abi.NL_*
    nonlinear: list = field(default_factory=list)
    mem_space: int = abi.MEM_HOST
    # device pointers (MEM_DEVICE): ints
    k_dev: int = 0
    f_dev: int = 0
    u0_dev: int = 0
    nodal_dev: int = 0

    @property
    def dims(self):
        return self.nx, self.ny, max(self.nz, 1)

    @property
    def n(self):
        return self.nx * self.ny * max(self.nz, 1)

    @property
    def is3d(self):
        return self.nz > 1

    def spacing(self):
        x0, x1, y0, y1, z0, z1 = self.bounds
        dx = (x1 - x0) / (self.nx - 1)
        dy = (y1 - y0) / (self.ny - 1)
        dz = (z1 - z0) / (self.nz - 1) if self.nz > 1 else 0.0
        return dx, dy, dz

    def coords(self):
        """Node coordinates as broadcastable arrays, shape (nz,ny,nx) order."""
        x0, x1, y0, y1, z0, z1 = self.bounds
        dx, dy, dz = self.spacing()
        x = x0 + np.arange(self.nx) * dx
        y = y0 + np.arange(self.ny) * dy
        z = z0 + np.arange(max(self.nz, 1)) * dz if self.nz > 1 else np.zeros(1)
        return x[None, None, :], y[None, :, None], z[:, None, None]

    def _contig(self, a):
        if a is None:
            return None
        return np.ascontiguousarray(a, dtype=np.float64).reshape(-1)

    def to_c(self) -> abi.Problem:
        p = abi.Problem()
        p.nx, p.ny, p.nz = self.nx, self.ny, self.nz
        p.coef_kind = self.coef_kind
        p.mem_space = self.mem_space
        (p.xmin, p.xmax, p.ymin, p.ymax, p.zmin, p.zmax) = [float(v) for v in self.bounds]
        p.a, p.b, p.az, p.c, p.d, p.dz, p.e = self.a, self.b, self.az, self.c, self.d, self.dz, self.e
        p.f_const = self.f_const
        p.ut = self.ut
        self._keep = []
        if self.mem_space == abi.MEM_DEVICE:
            p.k = C.cast(C.c_void_p(self.k_dev or None), C.POINTER(C.c_double))
            p.f = C.cast(C.c_void_p(self.f_dev or None), C.POINTER(C.c_double))
            p.u0 = C.cast(C.c_void_p(self.u0_dev or None), C.POINTER(C.c_double))
            p.nodal = C.cast(C.c_void_p(self.nodal_dev or None), C.POINTER(C.c_double))
        else:
            for name in ("k", "nodal", "f", "u0"):
                arr = self._contig(getattr(self, name))
                self._keep.append(arr)
                setattr(p, name, _dptr(arr))
        for i, fc in enumerate(self.faces):
            cf = p.face[i]
            cf.kind = fc.kind
            cf.value, cf.alpha, cf.beta, cf.gamma = fc.value, fc.alpha, fc.beta, fc.gamma
            for name in ("value_arr", "alpha_arr", "beta_arr", "gamma_arr"):
                arr = self._contig(getattr(fc, name))
                self._keep.append(arr)
                setattr(cf, name, _dptr(arr))
        if self.nonlinear:
            terms = (abi.NonlinearTerm * len(self.nonlinear))()
            for t, (kind, coeff, power) in zip(terms, self.nonlinear):
                t.kind, t.coeff, t.power = int(kind), float(coeff), int(power)
            self._keep.append(terms)
            p.n_nonlinear = len(self.nonlinear)
            p.nonlinear = C.cast(terms, C.POINTER(abi.NonlinearTerm))
        return p


def default_options(lib=None, **kw) -> abi.Options:
    """SolverConfig defaults (include/pde_types.h:282-303) overridden by kw."""
    o = abi.Options()
    o.method = abi.JACOBI
    o.max_iter = 10000
    o.tol = 1e-6
    o.tol_mode = abi.TOL_REFERENCE
    o.precision = abi.FP64
    o.sor_omega = 1.5
    o.gmres_restart = 30
    o.mg_pre_smooth = 2
    o.mg_post_smooth = 2
    o.mg_coarse_iters = 50
    o.mg_max_levels = 10
    o.gs_ordering = abi.ORDER_LEXICOGRAPHIC
    o.device = 0
    o.check_interval = 0
    o.inner_tol = 1e-5
    o.bf16_coefficients = 0
    o.max_outer = 50
    for k, v in kw.items():
        if not hasattr(o, k):
            raise AttributeError(k)
        setattr(o, k, v)
    return o
