"""GPU parity at the configurations' own sizes, on the reference's nonlinear
relaxation terms and on Robin conditions on the max faces, through the C ABI
against the oracle (the reference's own CPU solver where it has the method,
else the restatement pinned to it in tests/test_oracle_pins.py).

Bars: reference methods rel L2 <= 1e-10 (Jacobi, SOR, nonlinear terms: the
same algorithm; FMA contraction and CUDA's transcendentals are the only
differences); MG-PCG, solved to 1e-12 relative residual on both sides,
<= 1e-9 rel L2 with iteration counts within one."""
import numpy as np
import pytest

from pde_solver_b200 import abi, solver, synthetic
from pde_solver_b200.problem import FaceBC, GridProblem, default_options

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    d = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (d if d > 0 else 1.0)


@pytest.fixture(scope="module", autouse=True)
def _lib(lib):
    return lib


# ------------------------------------------- configuration sizes

def test_config1_jacobi_129_matches_reference(ref_oracle):
    # 2D Poisson 129^2, MMS right side, Dirichlet 0, Jacobi to max|du| < 1e-10
    # (SolveJacobi2D, src/backends/cpu/solvers/relaxation.cpp:310-574): about 49.5k sweeps
    p = synthetic.poisson_mms_2d(129)
    p.f = None
    opt = default_options(method=abi.JACOBI, max_iter=200000, tol=1e-10)
    st, ref, _, err = ref_oracle.ref_solve(p, opt, rhs_latex=synthetic.MMS_RHS_LATEX)
    assert st == 0, err
    p.f = ref_oracle.ref_materialize(synthetic.MMS_RHS_LATEX, p)
    got, rep = solver.solve(p, opt)
    assert rep.status == abi.OK
    _, rs, rrep = ref_oracle.rs_solve(p, opt)
    assert abs(rep.iterations - rrep.iterations) <= 1
    assert rel_l2(got, ref) <= 1e-10
    x, y, _ = p.coords()
    exact = (np.sin(np.pi * x) * np.sin(np.pi * y)).reshape(-1)
    assert abs(np.abs(got - exact).max() - np.abs(ref - exact).max()) <= 1e-9


@pytest.mark.parametrize("n", [129, 257])
def test_config2_mgpcg_matches_oracle(oracle_mod, n):
    # 3D variable-k Poisson (k log-normal sigma=1, 3 box passes; f ~ N(0,1);
    # faces D0/D0/N0/N0/Robin(1,1,0) front/D0): the configuration's own size 257^3
    p = synthetic.varcoef_poisson_3d(n, seed=1234)
    opt = default_options(method=abi.MG_PCG, tol=1e-12, tol_mode=abi.TOL_RELATIVE, max_iter=300)
    got, rep = solver.solve(p, opt)
    st, ref, rrep = oracle_mod.rs_solve(p, opt)
    assert st == 0 and rep.status == abi.OK
    assert rep.rel_residual <= 1e-12
    assert abs(rep.iterations - rrep.iterations) <= 1
    assert rel_l2(got, ref) <= 1e-9


def test_config2_tolerance_1e10_solution_within_parity_bar(oracle_mod):
    # at the configuration's stopping tolerance (1e-10 relative) the field the
    # bench times agrees with the oracle's converged field to the 1e-9 bar
    p = synthetic.varcoef_poisson_3d(129, seed=1234)
    got, rep = solver.solve(p, default_options(method=abi.MG_PCG, tol=1e-10, tol_mode=abi.TOL_RELATIVE,
                                               max_iter=300))
    assert rep.status == abi.OK and rep.rel_residual <= 1e-10
    st, ref, _ = oracle_mod.rs_solve(p, default_options(method=abi.MG_PCG, tol=1e-13, tol_mode=abi.TOL_RELATIVE,
                                                        max_iter=300))
    assert st == 0
    assert rel_l2(got, ref) <= 1e-9


@pytest.mark.parametrize("n", [65, 129])
def test_config3_mixed_error_against_fp64_oracle(oracle_mod, n):
    # 3D convection-diffusion -eps Lap u + b.grad u = f (eps 1e-2, unit b from
    # the seed, f ~ U[-1,1], Dirichlet 0): the FP32-in-FP64 MG-BiCGStab result
    # (BF16 smoother coefficients off and on) against the oracle's FP64
    # BiCGStab solution of the same system, solved to 1e-13 relative
    p = synthetic.convection_diffusion_3d(n, seed=99)
    bnorm = np.linalg.norm(p.f.reshape(n, n, n)[1:-1, 1:-1, 1:-1])
    st, ref, rrep = oracle_mod.rs_solve(p, default_options(method=abi.BICGSTAB, tol=1e-13 * bnorm, max_iter=20000))
    assert st == 0, rrep.message
    for bf16 in (0, 1):
        got, rep = solver.solve(p, default_options(method=abi.MG_BICGSTAB, precision=abi.MIXED, tol=1e-10,
                                                   tol_mode=abi.TOL_RELATIVE, max_iter=200, bf16_coefficients=bf16))
        assert rep.status == abi.OK and rep.rel_residual <= 1e-10
        assert rel_l2(got, ref) <= 1e-8


# ----------------------------------------------- max-face Robin in solves

@pytest.mark.parametrize("dims", [(33, 29, 31), (65, 49, 1)])
def test_mgpcg_robin_on_max_faces(oracle_mod, dims):
    # Robin on right, top and back: closure u_N = (gamma - beta/h u_{N-1})/(alpha - beta/h)
    # (cpu_utils.cpp:671-673,853-855,893-895); alpha > beta/h keeps the folded system SPD
    nx, ny, nz = dims
    rng = np.random.Generator(np.random.PCG64(nx * ny))
    p = GridProblem(nx, ny, nz, coef_kind=abi.COEF_DIVK)
    p.k = np.exp(0.5 * rng.standard_normal(p.n))
    p.f = rng.standard_normal(p.n)
    p.faces = [FaceBC.dirichlet(0.0), FaceBC.robin(2.0, 0.02, 0.1), FaceBC.neumann(0.0), FaceBC.robin(3.0, 0.05, 0.0),
               FaceBC.dirichlet(0.2) if nz > 1 else FaceBC(), FaceBC.robin(1.5, 0.01, -0.2) if nz > 1 else FaceBC()]
    opt = default_options(method=abi.MG_PCG, tol=1e-12, tol_mode=abi.TOL_RELATIVE, max_iter=300)
    got, rep = solver.solve(p, opt)
    st, ref, rrep = oracle_mod.rs_solve(p, opt)
    assert st == 0 and rep.status == abi.OK
    assert abs(rep.iterations - rrep.iterations) <= 1
    assert rel_l2(got, ref) <= 1e-9


@pytest.mark.parametrize("method,omega", [(abi.JACOBI, 1.0), (abi.SOR, 1.6)])
def test_relaxation_robin_on_max_faces_matches_reference(ref_oracle, method, omega):
    p = GridProblem(13, 12, 11, a=-1.0, b=-1.0, az=-1.0, c=0.2)
    p.faces = [FaceBC.neumann(0.1), FaceBC.robin(2.0, 0.05, 0.2), FaceBC.dirichlet(0.0), FaceBC.robin(1.5, 0.03, 0.0),
               FaceBC.dirichlet(0.25), FaceBC.robin(2.0, 0.05, -0.1)]
    opt = default_options(method=method, max_iter=40000, tol=1e-12, sor_omega=omega)
    st, ref, _, err = ref_oracle.ref_solve(p, opt, rhs_latex="1+x*z")
    assert st == 0, err
    p.f = ref_oracle.ref_materialize("1+x*z", p)
    got, rep = solver.solve(p, opt)
    assert rep.status == abi.OK
    assert rel_l2(got, ref) <= 1e-10


# ------------------------------------------------- nonlinear terms

NONLINEAR = [
    ("u2", [(abi.NL_POWER, 0.5, 2)]),
    ("sin", [(abi.NL_SIN, 2.0, 2)]),
    ("exp", [(abi.NL_EXP, 0.3, 2)]),
    ("cube_cos_abs", [(abi.NL_POWER, -0.4, 3), (abi.NL_COS, 0.5, 2), (abi.NL_ABS, 0.7, 2)]),
]


# every term kind on the small grids, two kinds on the larger ones
NONLINEAR_CASES = [(dims, name, terms) for dims in [(21, 19, 1), (11, 10, 9), (70, 66, 1), (24, 22, 20)]
                   for name, terms in NONLINEAR if dims[0] * dims[1] * dims[2] <= 2000 or name in ("u2", "sin")]


@pytest.mark.parametrize("method,omega", [(abi.JACOBI, 1.0), (abi.GAUSS_SEIDEL, 1.0), (abi.SOR, 1.5)])
@pytest.mark.parametrize("dims,name,terms", NONLINEAR_CASES)
def test_relaxation_nonlinear_terms_match_reference(ref_oracle, dims, method, omega, name, terms):
    # sum(coeff * g(u_old)) inside every relaxation update (EvalNonlinear,
    # relaxation.cpp:27-45,217-218,476-477; solver.cpp:884-885)
    _nonlinear_case(ref_oracle, dims, method, omega, terms, 1e-11)


def test_nonlinear_sor_multi_launch_wavefront(ref_oracle):
    # more than 2^18 interior nodes: one launch per hyperplane instead of the single-block form
    _nonlinear_case(ref_oracle, (68, 66, 66), abi.SOR, 1.9, [(abi.NL_SIN, 2.0, 2), (abi.NL_POWER, 0.5, 2)], 1e-9)


def _nonlinear_case(ref_oracle, dims, method, omega, terms, tol):
    p = GridProblem(*dims, a=-1.0, b=-1.0, az=-1.0, c=0.3)
    p.faces = [FaceBC.robin(1.0, 0.5, 0.2), FaceBC.dirichlet(0.0), FaceBC.neumann(0.3), FaceBC.dirichlet(1.0),
               FaceBC(), FaceBC()] if dims[2] == 1 else [
        FaceBC.dirichlet(0.0), FaceBC.dirichlet(0.5), FaceBC.neumann(0.0), FaceBC.neumann(0.2),
        FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(0.0)]
    p.nonlinear = terms
    opt = default_options(method=method, max_iter=100000, tol=tol, sor_omega=omega)
    st, ref, _, err = ref_oracle.ref_solve(p, opt, rhs_latex="x*y-1")
    assert st == 0, err
    p.f = ref_oracle.ref_materialize("x*y-1", p)
    got, rep = solver.solve(p, opt)
    assert rep.status == abi.OK, rep.message
    assert rel_l2(got, ref) <= 1e-10


def test_nonlinear_residual_norms_3d_leave_terms_out(ref_oracle):
    # 3D ComputeResidualNorms is interior-only and has no nonlinear term (src/residual.cpp:592-719)
    p = GridProblem(9, 8, 7, a=-1.0, b=-1.0, az=-1.0, f_const=0.5)
    p.faces = [FaceBC.dirichlet(0.0), FaceBC.neumann(0.1), FaceBC.dirichlet(0.0), FaceBC.dirichlet(0.0),
               FaceBC.robin(1.0, 0.5, 0.0), FaceBC.dirichlet(0.0)]
    p.nonlinear = [(abi.NL_EXP, 0.5, 2)]
    grid = np.random.Generator(np.random.PCG64(4)).standard_normal(p.n)
    l2r, lir = ref_oracle.ref_residual_norms(p, grid)
    l2, li = solver.residual_norms(p, grid)
    assert l2 == pytest.approx(l2r, rel=1e-12) and li == pytest.approx(lir, rel=1e-12)


@pytest.mark.parametrize("method", [abi.CG, abi.MG_PCG, abi.MG_BICGSTAB])
def test_nonlinear_terms_rejected_by_linear_methods(method):
    p = GridProblem(17, 17, 1, a=-1.0, b=-1.0)
    p.nonlinear = [(abi.NL_POWER, 1.0, 2)]
    _, rep = solver.solve(p, default_options(method=method, tol_mode=abi.TOL_RELATIVE), raise_on_error=False)
    assert rep.status == abi.ERR_UNSUPPORTED
    assert b"linear PDEs" in rep.message


# --------------------------------------------------- projection at 256^2

def test_projection_256_matches_reference(ref_oracle):
    # the smallest projection size of the serving stream, 256^2 N(0,1) velocities,
    # against ProjectVelocity2D itself (src/pressure_projection.cpp:255-334)
    n = 256
    u, v, p0 = synthetic.projection_fields(n, seed=17)
    h = 1.0 / (n - 1)
    st, ur, vr, _, pr, rrep = ref_oracle.ref_project(u, v, None, p0, n, n, 1, h, h, 1.0, 0.01, 20000, 1e-10)
    assert st == 0
    ug, vg, _, pg, rep = solver.project_velocity(u, v, None, p0, n, n, 1, h, h, 1.0, 0.01, 20000, 1e-10)
    assert rep.success == 1
    assert rep.poisson_iterations == int(rrep[0])
    for name, a, b in (("u", ug, ur), ("v", vg, vr), ("p", pg, pr)):
        d = rel_l2(a, b)
        assert d <= 1e-10, (name, d)


# ------------------------------------------- anisotropic constant coefficients

@pytest.mark.parametrize("dims,coefs", [((33, 33, 33), (-1.0, -4.0, -0.25)), ((65, 33, 1), (-3.0, -0.5, 0.0)),
                                        ((41, 29, 23), (-0.5, -1.0, -2.0))])
def test_mgpcg_anisotropic_constant_matches_oracle(oracle_mod, dims, coefs):
    # a, b, az differ by up to 16x: the smoother and the hierarchy see a
    # strongly directional operator; both sides solve to 1e-12 relative
    nx, ny, nz = dims
    a, b, az = coefs
    p = GridProblem(nx, ny, nz, a=a, b=b, az=az)
    p.f = np.random.Generator(np.random.PCG64(nx * ny + nz)).standard_normal(p.n)
    # Robin on min faces only: there the closure weight (beta/h)/(alpha+beta/h)
    # stays below one and the folded operator stays definite
    if nz == 1:
        p.faces = [FaceBC.robin(1.0, 0.5, 0.1), FaceBC.dirichlet(0.0), FaceBC.neumann(0.2), FaceBC.dirichlet(0.3),
                   FaceBC(), FaceBC()]
    else:
        p.faces = [FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(0.5), FaceBC.neumann(0.0), FaceBC.neumann(0.1),
                   FaceBC.robin(2.0, 0.5, 0.1), FaceBC.dirichlet(0.0)]
    opt = default_options(method=abi.MG_PCG, tol=1e-12, tol_mode=abi.TOL_RELATIVE, max_iter=400)
    got, rep = solver.solve(p, opt)
    st, ref, rrep = oracle_mod.rs_solve(p, opt)
    assert st == 0 and rep.status == abi.OK
    assert rep.rel_residual <= 1e-12
    assert abs(rep.iterations - rrep.iterations) <= 1
    assert rel_l2(got, ref) <= 1e-9
