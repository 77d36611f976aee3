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
    # Robin on the max faces (right, top, back): the closure there is
    # u_N = (gamma - beta/h u_{N-1}) / (alpha - beta/h) (cpu_utils.cpp:671-673,853-855,893-895);
    # alpha > 2 beta/h keeps |du_N/du_{N-1}| < 1, so the relaxation converges
    p = GridProblem(23, 19, 1, a=-1.0, b=-1.0, c=0.3)
    p.faces = [FaceBC.dirichlet(0.0), FaceBC.robin(2.0, 0.02, 0.3), FaceBC.dirichlet(0.5), FaceBC.robin(1.0, 0.02, 0.2),
               FaceBC(), FaceBC()]
    out["jacobi_maxrobin_2d"] = (p, default_options(method=abi.JACOBI, max_iter=40000, tol=1e-11), "x-y")
    p = GridProblem(11, 10, 9, a=-1.0, b=-1.0, az=-1.0)
    p.faces = [FaceBC.neumann(0.1), FaceBC.robin(2.0, 0.05, 0.2), FaceBC.dirichlet(0.0), FaceBC.robin(1.5, 0.03, 0.0),
               FaceBC.dirichlet(0.25), FaceBC.robin(2.0, 0.05, -0.1)]
    out["sor_maxrobin_3d"] = (p, default_options(method=abi.SOR, sor_omega=1.5, max_iter=40000, tol=1e-12), "1+x*z")
    # pointwise nonlinear terms (EvalNonlinear, relaxation.cpp:27-45, solver.cpp:234-256)
    p = GridProblem(25, 21, 1, a=-1.0, b=-1.0)
    p.faces = faces_2d()
    p.nonlinear = [(abi.NL_POWER, 0.5, 2)]
    out["jacobi_nl_u2_2d"] = (p, default_options(method=abi.JACOBI, max_iter=40000, tol=1e-11), "x*y-1")
    p = GridProblem(25, 21, 1, a=-1.0, b=-1.0, c=0.4)
    p.faces = faces_2d()
    p.nonlinear = [(abi.NL_SIN, 2.0, 2)]
    out["sor_nl_sin_2d"] = (p, default_options(method=abi.SOR, sor_omega=1.6, max_iter=40000, tol=1e-12), "1+x")
    p = GridProblem(11, 9, 10, a=-1.0, b=-1.0, az=-1.0)
    p.faces = faces_3d()
    p.nonlinear = [(abi.NL_EXP, 0.3, 2)]
    out["gs_nl_exp_3d"] = (p, default_options(method=abi.GAUSS_SEIDEL, max_iter=40000, tol=1e-12), "x-z")
    p = GridProblem(12, 11, 10, a=-1.0, b=-1.0, az=-1.0)
    p.faces = faces_3d()
    p.nonlinear = [(abi.NL_POWER, -0.4, 3), (abi.NL_COS, 0.5, 2), (abi.NL_ABS, 0.7, 2)]
    out["jacobi_nl_mixed_3d"] = (p, default_options(method=abi.JACOBI, max_iter=40000, tol=1e-11), "y+1")
    return out


def heat_nl_case():
    """2D heat step with a pointwise nonlinear source (solver.cpp:1298-1302)."""
    p, t0, dt, frames = heat_case()
    p.nonlinear = [(abi.NL_POWER, 0.8, 2), (abi.NL_SIN, -0.5, 2)]
    return p, t0, dt, frames


def residual_nl_case():
    """2D residual norms with nonlinear terms (residual.cpp:449-487)."""
    p, grid = residual_case()
    p.nonlinear = [(abi.NL_POWER, 0.25, 3), (abi.NL_EXP, 0.1, 2)]
    return p, grid


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


def expression_cases():
    """LaTeX expressions with the grid and time they are evaluated on:
    (latex, nx, ny, nz, bounds, t). They cover every command, function, alias,
    constant and guard of the reference's evaluator (src/expression_eval.cpp)."""
    b2 = (-1.0, 1.0, -0.5, 1.5, 0.0, 0.0)
    b3 = (0.0, 1.0, -1.0, 1.0, 0.25, 2.0)
    pos = (0.1, 2.0, 0.2, 3.0, 0.0, 0.0)
    return [
        (r"\sin(\pi*x)\sin(\pi*y)", 17, 13, 1, b2, 0.0),
        (r"-2\pi^2\sin(\pi*x)\cdot\sin(\pi*y)", 17, 13, 1, b2, 0.0),
        (r"\frac{x^2 + y^2}{1 + x^2}", 17, 13, 1, b2, 0.0),
        (r"\sqrt{x^2+y^2+z^2} \times e^{-t}", 9, 7, 5, b3, 0.75),
        (r"\exp(-(x^2+y^2)/0.1)", 17, 13, 1, b2, 0.0),
        (r"\left(x + 1\right)^{3} - 2 x", 17, 13, 1, b2, 0.0),
        (r"2(x)(y) + 3y\cdot z\,", 9, 7, 5, b3, 0.0),
        (r"x^y^2", 17, 13, 1, pos, 0.0),
        (r"-x^2", 17, 13, 1, b2, 0.0),
        (r"\tan(x) + \tanh(y) + \sinh(x) - \cosh(y)", 17, 13, 1, b2, 0.0),
        (r"\arcsin(x) + \arccos(y) + \arctan(x*y)", 17, 13, 1, b2, 0.0),
        (r"\operatorname{asin}(2x) + \operatorname{acos}(y/2)", 17, 13, 1, b2, 0.0),
        (r"\ln(x) + \log{y}", 17, 13, 1, b2, 0.0),
        (r"\ln(x) + \log{y}", 17, 13, 1, pos, 0.0),
        (r"\sqrt{x}", 17, 13, 1, b2, 0.0),
        (r"\frac{1}{x}", 17, 13, 1, b2, 0.0),
        (r"\frac{1}{x - y}", 17, 17, 1, (0.0, 1.0, 0.0, 1.0, 0.0, 0.0), 0.0),
        (r"\exp(800 x) + \exp(-800 x)", 17, 13, 1, b2, 0.0),
        (r"\floor(4x) + \ceil(4y) + \round(2.5x) + \abs(x\cdot y)", 17, 13, 1, b2, 0.0),
        (r"\sign(x) + \sgn{y} + \operatorname{sgn}(x+y)", 17, 13, 1, b2, 0.0),
        (r"\erf(x) \cdot \erf(2y)", 17, 13, 1, b2, 0.0),
        (r"\min{x,y} + \max(x, y^2)", 17, 13, 1, b2, 0.0),
        (r"\pow{x, 2} + \pow(y, 0.5) + \operatorname{pow}{x, y}", 17, 13, 1, b2, 0.0),
        (r"x^{0.5} + (-2)^{3} + (-8)^{1/3}", 17, 13, 1, b2, 0.0),
        (r"\sin{\pi} + \cos\pi + \sin x + \cos 2 + \exp .5", 17, 13, 1, b2, 0.0),
        (r"r\cdot\cos(\theta) + \phi + \vartheta*\varphi", 9, 7, 5, b3, 0.0),
        (r"$x + t$", 17, 13, 1, b2, 1.25),
        (r"\sin(x)^2 + \cos(x)^2", 17, 13, 1, b2, 0.0),
        (r"e^{x} - e", 17, 13, 1, b2, 0.0),
        (r"1.5e-3 + .25 + 3.", 17, 13, 1, b2, 0.0),
        (r"f(x) + 1", 17, 13, 1, b2, 0.0),
        (r"+-+x", 17, 13, 1, b2, 0.0),
        (r"\frac{\sin(\pi*x)}{\pi*(1 + t)}\frac{y}{2}", 9, 7, 5, b3, 2.0),
    ]


def expression_errors():
    """Expressions the reference rejects; the message must match."""
    return [
        r"\sin(\pi x)",
        r"2xy",
        r"\foo(x)",
        r"\frac{1}",
        r"\sqrt(x)",
        r"\min{x}",
        r"x + }",
        r"(x + 1",
        r"x + ",
        r"x $ # y",
        r"",
        r"\left(\right)",
        r"\sin",
        r"\sin\,",
        "(" * 60 + "x" + ")" * 60,
        "-" * 120 + "x",
        r"\max{x,",
        r"3y\,z",
        r"\atan2{y, x}",
        r"\operatorname{atan2}{y, x}",
    ]


def vtk_cases():
    """Fields for the VTK writers: (name, problem geometry, field). Values mix
    smooth data with the formatter's edge cases: exact decimal ties, negative
    zero, tiny negatives, subnormals, huge values, +-inf and NaN of both signs."""
    rng = np.random.default_rng(2024)
    special = np.array([0.0078125, -0.0078125, 2.0**-20, 0.5, 2.5, -0.0, -1e-9, 1e-45, 3.4e38, -3.4e38,
                        0.9999995, 123456.7890625, 1e300, -1e300, np.inf, -np.inf, np.nan,
                        -np.nan, 4.0e9, 16777217.0, 1.0 / 3.0, 2.0 / 3.0], dtype=np.float64)
    special[17] = np.copysign(np.nan, -1.0)
    out = []
    p = GridProblem(9, 7, 1, bounds=(-1.0, 1.0, 0.0, 3.0, 0.0, 1.0), a=-1.0, b=-2.0, az=-0.5)
    f = np.sin(np.linspace(0.0, 7.0, p.n)) * 10.0 ** rng.integers(-8, 6, p.n)
    f[:special.size] = special
    out.append(("field_2d", p, f))
    p = GridProblem(6, 5, 4, bounds=(0.0, 1.0, -0.5, 0.5, 0.25, 2.0), a=-1.0, b=-1.0, az=-3.0)
    x, y, z = p.coords()
    out.append(("smooth_3d", p, np.exp(-x) * np.cos(3.0 * y) + z * z))
    p = GridProblem(3, 3, 1, bounds=(0.0, 1e-3, 0.0, 2.5e6, 0.0, 0.0))
    out.append(("tiny_2d", p, rng.standard_normal(p.n)))
    p = GridProblem(1, 2, 1, bounds=(0.0, 0.0, 0.0, 1.0, 0.0, 1.0))
    out.append(("single_column", p, np.array([1.25, -7.5])))
    return out
