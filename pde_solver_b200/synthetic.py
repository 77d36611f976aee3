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


def gaussian_bump(p: GridProblem, width: float = 40.0) -> np.ndarray:
    """u0 = exp(-width |x - c|^2) around the domain centre."""
    x, y, z = p.coords()
    x0, x1, y0, y1, z0, z1 = p.bounds
    r2 = (x - 0.5 * (x0 + x1)) ** 2 + (y - 0.5 * (y0 + y1)) ** 2
    if p.nz > 1:
        r2 = r2 + (z - 0.5 * (z0 + z1)) ** 2
    return np.ascontiguousarray(np.broadcast_to(np.exp(-width * r2), (max(p.nz, 1), p.ny, p.nx))).reshape(-1)


def heat_problem(n: int, dim: int = 2) -> tuple:
    """u_t = Laplace(u) (reference form a=b[=az]=-1, ut=1), Dirichlet 0, Gaussian
    bump u0; returns (problem, dt) with dt = 0.9 h^2 / (2 dim), the forward-Euler
    limit scaled by 0.9."""
    p = GridProblem(n, n, n if dim == 3 else 1, a=-1.0, b=-1.0, az=-1.0 if dim == 3 else 0.0, ut=1.0)
    p.u0 = gaussian_bump(p)
    h = 1.0 / (n - 1)
    return p, 0.9 * h * h / (2 * dim)


def projection_fields(n: int, seed: int) -> tuple:
    """2D velocity (u, v) ~ N(0,1) and zero pressure on an n x n grid."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return rng.standard_normal(n * n), rng.standard_normal(n * n), np.zeros(n * n)


def serving_requests(count: int, seed: int, rate_hz: float, lo2=65, hi2=513, lo3=65, hi3=129,
                     heat_hi=257, proj_lo=256, proj_hi=1024, mix=(0.6, 0.25, 0.15)) -> list:
    """A seeded request stream: (arrival_s, kind, spec) with Poisson-process
    arrivals at `rate_hz`; kinds drawn with probabilities `mix` (Poisson solve,
    200-step heat, 2D projection). Poisson solves are 2D (sides lo2..hi2) or 3D
    (sides lo3..hi3) divergence-form problems with k log-normal sigma=0.5."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = 0.0
    out = []
    for q in range(count):
        t += rng.exponential(1.0 / rate_hz)
        kind = rng.choice(3, p=mix)
        if kind == 0:
            is3 = rng.random() < 0.3
            lo, hi = (lo3, hi3) if is3 else (lo2, hi2)
            n = int(np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi)))))
            out.append((t, "poisson", dict(n=n, dim=3 if is3 else 2, seed=int(rng.integers(1 << 30)))))
        elif kind == 1:
            n = int(np.rint(np.exp(rng.uniform(np.log(lo2), np.log(heat_hi)))))
            out.append((t, "heat", dict(n=n, steps=200)))
        else:
            n = int(np.rint(np.exp(rng.uniform(np.log(proj_lo), np.log(proj_hi)))))
            out.append((t, "projection", dict(n=n, seed=int(rng.integers(1 << 30)))))
    return out


def poisson_request_problem(n: int, dim: int, seed: int, sigma: float = 0.5) -> GridProblem:
    rng = np.random.Generator(np.random.PCG64(seed))
    shape = (n, n, n) if dim == 3 else (n, n)
    p = GridProblem(n, n, n if dim == 3 else 1, coef_kind=abi.COEF_DIVK)
    p.k = np.exp(sigma * rng.standard_normal(shape)).reshape(-1)
    p.f = (-rng.standard_normal(shape)).reshape(-1)
    return p
