"""Cases of the golden fixtures (reference_cases.npz). Each case builds its
problem and options deterministically; make_golden.py runs the reference's own
CPU solver (compiled from its sources into oracle/_ref) on them and stores the
results, so the fixtures pin this path without the reference sources present."""
import numpy as np

from pde_solver_b200 import abi, synthetic
from pde_solver_b200.problem import FaceBC, GridProblem, default_options


def faces_2d():
    return [FaceBC.robin(1.0, 0.5, 0.2), FaceBC.dirichlet(0.0), FaceBC.neumann(0.3), FaceBC.dirichlet(1.0),
            FaceBC(), FaceBC()]


def faces_3d():
    return [FaceBC.dirichlet(0.0), FaceBC.dirichlet(0.5), FaceBC.neumann(0.0), FaceBC.neumann(0.2),
            FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(0.0)]


def solve_cases():
    """name -> (problem, options, rhs_latex). The reference evaluates the LaTeX
    right-hand side; the fixture stores the materialised f it used."""
    out = {}
    p = GridProblem(33, 33, 1, a=-1.0, b=-1.0)
    out["cg_mms_33"] = (p, default_options(method=abi.CG, max_iter=8000, tol=1e-10), synthetic.MMS_RHS_LATEX)
    p = GridProblem(21, 17, 1, a=-1.0, b=-1.0, c=0.4)
    p.faces = faces_2d()
    out["jacobi_mixed_2d"] = (p, default_options(method=abi.JACOBI, max_iter=20000, tol=1e-9), "x+2*y")
    p = GridProblem(25, 21, 1, a=-1.0, b=-1.0, c=0.4)
    p.faces = faces_2d()
    out["sor_mixed_2d"] = (p, default_options(method=abi.SOR, sor_omega=1.7, max_iter=20000, tol=1e-11),
                           "\\sin(\\pi*x)*y")
    p = GridProblem(11, 9, 10, a=-1.0, b=-1.0, az=-1.0, c=0.4)
    p.faces = faces_3d()
    out["gs_mixed_3d"] = (p, default_options(method=abi.GAUSS_SEIDEL, max_iter=20000, tol=1e-11), "x*y+z")
    p = GridProblem(33, 33, 1, a=-1.0, b=-1.0)
    p.faces = [FaceBC.dirichlet(0.0), FaceBC.dirichlet(1.0), FaceBC.dirichlet(0.0), FaceBC.dirichlet(2.0),
               FaceBC(), FaceBC()]
    out["vcycle_2d"] = (p, default_options(method=abi.MG_VCYCLE, max_iter=1, tol=1e-8), "x+y")
    p = GridProblem(21, 19, 1, a=-1.0, b=-0.5, c=3.0, d=-2.0, e=-0.3)
    p.faces = [FaceBC.dirichlet(0.5), FaceBC.dirichlet(0.0), FaceBC.dirichlet(1.0), FaceBC.dirichlet(0.0),
               FaceBC(), FaceBC()]
    out["bicgstab_2d"] = (p, default_options(method=abi.BICGSTAB, max_iter=3000, tol=1e-10), "x-y+1")
    return out


def heat_case():
    n = 33
    p = GridProblem(n, n, 1, a=-1.0, b=-1.0, ut=1.0)
    p.faces = [FaceBC.dirichlet(0.0), FaceBC.neumann(0.0), FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(0.0),
               FaceBC(), FaceBC()]
    x, y, _ = p.coords()
    p.u0 = np.exp(-40 * ((x - 0.5) ** 2 + (y - 0.5) ** 2)).reshape(-1)
    h = 1.0 / (n - 1)
    return p, 0.0, 0.9 * h * h / 4, 25


def projection_case():
    nx, ny = 24, 20
    n = nx * ny
    rng = np.random.Generator(np.random.PCG64(5))
    u, v = rng.standard_normal(n), rng.standard_normal(n)
    return dict(u=u, v=v, w=None, p=np.zeros(n), nx=nx, ny=ny, nz=1, dx=1.0 / (nx - 1), dy=1.0 / (ny - 1), dz=1.0,
                dt=0.01, max_iter=2000, tol=1e-10)


def residual_case():
    p = GridProblem(19, 17, 1, a=-1.0, b=-2.0, c=0.3, e=0.2, f_const=0.7)
    p.faces = [FaceBC.robin(1.0, 0.5, 0.2), FaceBC.robin(2.0, 0.25, 0.1), FaceBC.neumann(0.3),
               FaceBC.dirichlet(1.0), FaceBC(), FaceBC()]
    grid = np.random.Generator(np.random.PCG64(3)).standard_normal(p.n)
    return p, grid
