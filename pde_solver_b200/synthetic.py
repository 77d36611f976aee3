"""Seeded synthetic inputs of the benchmark shapes.

The reference publishes no dataset; every field here is generated from a seed
with numpy's PCG64 so the CPU oracle and the GPU see identical inputs.
"""
from __future__ import annotations

import numpy as np

from . import abi
from .problem import FaceBC, GridProblem


def box_smooth(a: np.ndarray, passes: int = 3) -> np.ndarray:
    """`passes` applications of a 3^d box filter with clamped (edge-replicated) borders."""
    from scipy.ndimage import uniform_filter

    out = a
    for _ in range(passes):
        out = uniform_filter(out, size=3, mode="nearest")
    return out


def lognormal_k(shape, sigma: float, seed: int, passes: int = 3) -> np.ndarray:
    """k = exp(sigma*g), g iid N(0,1), then `passes` box-filter passes."""
    rng = np.random.Generator(np.random.PCG64(seed))
    g = rng.standard_normal(shape)
    return np.ascontiguousarray(box_smooth(np.exp(sigma * g), passes))


def gaussian(shape, seed: int) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.ascontiguousarray(rng.standard_normal(shape))


def poisson_mms_2d(n: int = 129) -> GridProblem:
    """-Laplace(u) = 2 pi^2 sin(pi x) sin(pi y) on [0,1]^2, Dirichlet 0.
    Reference form a=b=-1, f = -2 pi^2 sin sin (the rhs_latex
    "-2*\\pi^2*\\sin(\\pi*x)*\\sin(\\pi*y)")."""
    p = GridProblem(n, n, 1, a=-1.0, b=-1.0)
    x, y, _ = p.coords()
    p.f = (-2.0 * np.pi ** 2 * np.sin(np.pi * x) * np.sin(np.pi * y)).reshape(-1)
    return p


MMS_RHS_LATEX = "-2*\\pi^2*\\sin(\\pi*x)*\\sin(\\pi*y)"


def varcoef_poisson_3d(n: int = 257, seed: int = 1234, sigma: float = 1.0) -> GridProblem:
    """-div(k grad u) = F on [0,1]^3; k log-normal (sigma) smoothed by 3 box
    passes; F ~ N(0,1); faces: left/right Dirichlet 0, bottom/top Neumann 0,
    front Robin(alpha=1, beta=1, gamma=0), back Dirichlet 0 (Robin on a min face,
    where every closure of the reference agrees)."""
    shape = (n, n, n)
    p = GridProblem(n, n, n, coef_kind=abi.COEF_DIVK)
    p.k = lognormal_k(shape, sigma, seed).reshape(-1)
    p.f = (-gaussian(shape, seed + 1)).reshape(-1)  # reference sign: f = -F
    p.faces = [FaceBC.dirichlet(0.0), FaceBC.dirichlet(0.0),
               FaceBC.neumann(0.0), FaceBC.neumann(0.0),
               FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(0.0)]
    return p


def convection_diffusion_3d(n: int = 513, seed: int = 99, eps: float = 1e-2) -> GridProblem:
    """-eps Laplace(u) + b.grad(u) = F, b a seeded unit vector, F ~ U[-1,1],
    Dirichlet 0 (centred convection, src/backends/cpu/solver.cpp:857-859)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    bv = rng.standard_normal(3)
    bv /= np.linalg.norm(bv)
    p = GridProblem(n, n, n, a=-eps, b=-eps, az=-eps, c=float(bv[0]), d=float(bv[1]), dz=float(bv[2]))
    p.f = (-rng.uniform(-1.0, 1.0, size=(n, n, n))).reshape(-1)
    return p


def varcoef_poisson_2d(n: int, seed: int, sigma: float = 0.5) -> GridProblem:
    """2D member of the batched set: k log-normal sigma, f Gaussian, Dirichlet 0."""
    p = GridProblem(n, n, 1, coef_kind=abi.COEF_DIVK)
    p.k = lognormal_k((n, n), sigma, seed).reshape(-1)
    p.f = gaussian((n, n), seed + 1).reshape(-1)
    return p


def batch_sides(n2d: int, n3d: int, seed: int, lo2=33, hi2=513, lo3=17, hi3=129):
    """Sides of the batched workload: 2D sides round(exp(U[ln lo2, ln hi2])),
    3D sides round(exp(U[ln lo3, ln hi3]))."""
    rng = np.random.Generator(np.random.PCG64(seed))
    s2 = np.rint(np.exp(rng.uniform(np.log(lo2), np.log(hi2), n2d))).astype(int)
    s3 = np.rint(np.exp(rng.uniform(np.log(lo3), np.log(hi3), n3d))).astype(int)
    return s2, s3


def batch_members(n2d: int = 2048, n3d: int = 256, seed: int = 4242, sigma: float = 0.5,
                  lo2=33, hi2=513, lo3=17, hi3=129) -> list:
    """Independent Poisson/diffusion grids -div(k grad u) = F with k = exp(sigma g)
    (g iid N(0,1) per node, no smoothing), F ~ N(0,1), Dirichlet 0, each seeded
    by its index: n2d square 2D grids then n3d cubic 3D grids."""
    s2, s3 = batch_sides(n2d, n3d, seed, lo2, hi2, lo3, hi3)
    out = []
    for q, n in enumerate(list(s2) + list(s3)):
        rng = np.random.Generator(np.random.PCG64([seed, q]))
        is3 = q >= n2d
        shape = (n, n, n) if is3 else (n, n)
        p = GridProblem(n, n, n if is3 else 1, coef_kind=abi.COEF_DIVK)
        p.k = np.exp(sigma * rng.standard_normal(shape)).reshape(-1)
        p.f = (-rng.standard_normal(shape)).reshape(-1)
        out.append(p)
    return out
