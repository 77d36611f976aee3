"""Pins the plain-C restatement (oracle/restate.c) to the reference's own CPU
solver compiled from its sources (oracle/_ref/libpderef.so). CPU only.

Each case runs the reference through SolveWithBackend(CPU) and the
restatement on the same input; the restatement follows the reference's
expression order, so the fields agree to rounding (most are bit-identical).
"""
import numpy as np
import pytest

from pde_solver_b200 import abi, synthetic
from pde_solver_b200.problem import FaceBC, GridProblem, default_options

REL = 1e-12


def rel_l2(a, b):
    d = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (d if d > 0 else 1.0)


def _pair(ref_oracle, prob, opt, rhs_latex=None, coef_latex=None, f_from_latex=True):
    st, ref, _, err = ref_oracle.ref_solve(prob, opt, rhs_latex=rhs_latex, coef_latex=coef_latex)
    assert st == 0, err
    if rhs_latex is not None and f_from_latex:
        prob.f = ref_oracle.ref_materialize(rhs_latex, prob)
    st2, rs, rep = ref_oracle.rs_solve(prob, opt)
    assert st2 in (abi.OK, abi.ERR_NOT_CONVERGED), rep.message
    return ref, rs, rep


def test_reference_self_test_known_failures(ref_oracle):
    # 9/11 pass; the two failures are reference defects (single-V-cycle "mg",
    # unary-minus/^ precedence in the MMS RHS), src/self_test.cpp:224-411.
    # RunSelfTest returns 1 when any case fails (:404-410).
    assert ref_oracle.reference().pderef_self_test() == 1


def test_cg_config1_mms(ref_oracle):
    prob = GridProblem(129, 129, 1, a=-1.0, b=-1.0)
    opt = default_options(method=abi.CG, max_iter=8000, tol=1e-10)
    ref, rs, rep = _pair(ref_oracle, prob, opt, rhs_latex=synthetic.MMS_RHS_LATEX)
    assert rel_l2(rs, ref) <= REL
    x, y, _ = prob.coords()
    exact = (np.sin(np.pi * x) * np.sin(np.pi * y)).reshape(-1)
    err_inf = np.abs(rs - exact).max()
    assert abs(err_inf - 5.02e-5) < 0.005e-5  # err_inf 5.02e-5 of the reference CG at 129^2


def test_cg_nonzero_dirichlet_reference_defect(ref_oracle):
    # The reference's CG keeps identity boundary rows with non-zero Dirichlet
    # data, which makes its operator nonsymmetric: it diverges
    # (src/backends/cpu/solvers/krylov.cpp:14-80 on cpu_utils.cpp:497-512 rows).
    # The restatement reproduces the failure.
    prob = GridProblem(33, 33, 1, a=-1.0, b=-1.0, f_const=3.0)
    prob.faces = [FaceBC.dirichlet(1.0), FaceBC.dirichlet(2.0), FaceBC.dirichlet(0.0), FaceBC.dirichlet(-1.5),
                  FaceBC(), FaceBC()]
    opt = default_options(method=abi.CG, max_iter=4000, tol=1e-10)
    st, _, _, err = ref_oracle.ref_solve(prob, opt)
    assert st != 0 and "converge" in err
    st2, _, _ = ref_oracle.rs_solve(prob, opt)
    assert st2 in (abi.ERR_BREAKDOWN, abi.ERR_NOT_CONVERGED)


def test_cg_zero_dirichlet_const_rhs(ref_oracle):
    prob = GridProblem(41, 33, 1, a=-1.0, b=-2.0, e=-0.5, f_const=3.0)
    opt = default_options(method=abi.CG, max_iter=4000, tol=1e-11)
    ref, rs, _ = _pair(ref_oracle, prob, opt)
    assert rel_l2(rs, ref) <= REL


@pytest.mark.parametrize("method,restart", [(abi.BICGSTAB, 30), (abi.GMRES, 400)])
def test_nonsymmetric_krylov(ref_oracle, method, restart):
    prob = GridProblem(21, 19, 1, a=-1.0, b=-0.5, c=3.0, d=-2.0, e=-0.3)
    prob.faces = [FaceBC.dirichlet(0.5), FaceBC.dirichlet(0.0), FaceBC.dirichlet(1.0), FaceBC.dirichlet(0.0),
                  FaceBC(), FaceBC()]
    opt = default_options(method=method, max_iter=3000, tol=1e-10, gmres_restart=restart)
    ref, rs, _ = _pair(ref_oracle, prob, opt, rhs_latex="\\sin(3*x)+y")
    assert rel_l2(rs, ref) <= 1e-10


def test_gmres_restart_reference_defect(ref_oracle):
    # After a restart the reference sizes the back-substitution with
    # y_dim = min(m, iter_total) (krylov.cpp:297) and fails; restated as is.
    prob = GridProblem(33, 29, 1, a=-1.0, b=-0.5, c=3.0, d=-2.0, e=-0.3)
    opt = default_options(method=abi.GMRES, max_iter=3000, tol=1e-10, gmres_restart=25)
    st, _, _, err = ref_oracle.ref_solve(prob, opt, rhs_latex="\\sin(3*x)+y")
    assert st != 0
    prob.f = ref_oracle.ref_materialize("\\sin(3*x)+y", prob)
    st2, _, _ = ref_oracle.rs_solve(prob, opt)
    assert st2 != abi.OK


def _mixed_faces_2d():
    return [FaceBC.robin(1.0, 0.5, 0.2), FaceBC.dirichlet(0.0), FaceBC.neumann(0.3), FaceBC.dirichlet(1.0),
            FaceBC(), FaceBC()]


@pytest.mark.parametrize("method,omega", [(abi.JACOBI, 1.0), (abi.GAUSS_SEIDEL, 1.0), (abi.SOR, 1.7)])
def test_relaxation_2d_mixed(ref_oracle, method, omega):
    prob = GridProblem(25, 21, 1, a=-1.0, b=-1.0, c=0.5)
    prob.faces = _mixed_faces_2d()
    opt = default_options(method=method, max_iter=20000, tol=1e-11, sor_omega=omega)
    ref, rs, rep = _pair(ref_oracle, prob, opt, rhs_latex="x*y-1")
    assert rel_l2(rs, ref) <= REL


def _mixed_faces_3d():
    return [FaceBC.dirichlet(0.0), FaceBC.dirichlet(0.5), FaceBC.neumann(0.0), FaceBC.neumann(0.2),
            FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(0.0)]


@pytest.mark.parametrize("method,omega", [(abi.JACOBI, 1.0), (abi.GAUSS_SEIDEL, 1.0), (abi.SOR, 1.5)])
def test_relaxation_3d_mixed(ref_oracle, method, omega):
    prob = GridProblem(13, 11, 9, a=-1.0, b=-1.0, az=-1.0, dz=0.4)
    prob.faces = _mixed_faces_3d()
    opt = default_options(method=method, max_iter=20000, tol=1e-11, sor_omega=omega)
    ref, rs, _ = _pair(ref_oracle, prob, opt, rhs_latex="x+y*z")
    assert rel_l2(rs, ref) <= REL


def test_divk_constant_k_equals_reference_const(ref_oracle):
    # Constant k reduces exactly to the reference 7-point stencil with a=b=az=-k.
    kval = 2.5
    ref_prob = GridProblem(11, 11, 11, a=-kval, b=-kval, az=-kval)
    ref_prob.faces = _mixed_faces_3d()
    opt = default_options(method=abi.SOR, max_iter=20000, tol=1e-12, sor_omega=1.6)
    st, ref, _, err = ref_oracle.ref_solve(ref_prob, opt, rhs_latex="1+x")
    assert st == 0, err
    prob = GridProblem(11, 11, 11, coef_kind=abi.COEF_DIVK)
    prob.faces = _mixed_faces_3d()
    prob.k = np.full(prob.n, kval)
    prob.f = ref_oracle.ref_materialize("1+x", prob)
    st2, rs, _ = ref_oracle.rs_solve(prob, opt)
    assert st2 == 0
    assert rel_l2(rs, ref) <= REL


@pytest.mark.parametrize("dim", [2, 3])
def test_nodal_variable_coefficients(ref_oracle, dim):
    n = (17, 15, 1) if dim == 2 else (11, 9, 10)
    lat = ["-(1+x*y)", "-(2+\\sin(x))", "-(1+z)" if dim == 3 else None, "x", None, "0.5" if dim == 3 else None, "-0.1"]
    prob = GridProblem(*n, a=-1.0, b=-1.0, az=-1.0)
    prob.faces = _mixed_faces_2d() if dim == 2 else _mixed_faces_3d()
    opt = default_options(method=abi.SOR, max_iter=20000, tol=1e-12, sor_omega=1.4)
    st, ref, _, err = ref_oracle.ref_solve(prob, opt, rhs_latex="1", coef_latex=lat)
    assert st == 0, err
    consts = [prob.a, prob.b, prob.az, prob.c, prob.d, prob.dz, prob.e]
    nodal = np.concatenate([ref_oracle.ref_materialize(s, prob) if s else np.full(prob.n, c)
                            for s, c in zip(lat, consts)])
    prob.coef_kind = abi.COEF_NODAL
    prob.nodal = nodal
    prob.f_const = 1.0
    st2, rs, _ = ref_oracle.rs_solve(prob, opt)
    assert st2 == 0
    assert rel_l2(rs, ref) <= REL


def test_mg_single_vcycle(ref_oracle):
    prob = GridProblem(33, 33, 1, a=-1.0, b=-1.0)
    prob.faces = [FaceBC.dirichlet(0.0), FaceBC.dirichlet(1.0), FaceBC.dirichlet(0.0), FaceBC.dirichlet(2.0),
                  FaceBC(), FaceBC()]
    opt = default_options(method=abi.MG_VCYCLE, max_iter=1, tol=1e-8)
    ref, rs, _ = _pair(ref_oracle, prob, opt, rhs_latex="x+y")
    assert rel_l2(rs, ref) <= REL


def test_time_series_heat(ref_oracle):
    n = 33
    prob = GridProblem(n, n, 1, a=-1.0, b=-1.0, ut=1.0)
    prob.faces = [FaceBC.dirichlet(0.0), FaceBC.neumann(0.0), FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(0.0),
                  FaceBC(), FaceBC()]
    x, y, _ = prob.coords()
    prob.u0 = np.exp(-40 * ((x - 0.5) ** 2 + (y - 0.5) ** 2)).reshape(-1)
    h = 1.0 / (n - 1)
    dt = 0.9 * h * h / 4
    ref, ref_frames = ref_oracle.ref_time_series(prob, 0.0, dt, 25, keep_frames=True)
    rs, rs_frames = ref_oracle.rs_time_series(prob, 0.0, dt, 25, keep_frames=True)
    assert np.array_equal(rs_frames, ref_frames) or rel_l2(rs, ref) <= REL


@pytest.mark.parametrize("dims", [(24, 20, 1), (10, 9, 8)])
def test_projection(ref_oracle, dims):
    nx, ny, nz = dims
    n = nx * ny * nz
    rng = np.random.Generator(np.random.PCG64(5))
    u, v = rng.standard_normal(n), rng.standard_normal(n)
    w = rng.standard_normal(n) if nz > 1 else None
    p = np.zeros(n)
    dx, dy, dz = 1.0 / (nx - 1), 1.0 / (ny - 1), (1.0 / (nz - 1) if nz > 1 else 1.0)
    st, ur, vr, wr, pr, rep = ref_oracle.ref_project(u, v, w, p, nx, ny, nz, dx, dy, dz, 0.01, 2000, 1e-10)
    st2, us, vs, ws, ps, rep2 = ref_oracle.rs_project(u, v, w, p, nx, ny, nz, dx, dy, dz, 0.01, 2000, 1e-10)
    assert st == 0 and st2 == 0
    assert rep2.poisson_iterations == int(rep[0])
    for a, b in ((us, ur), (vs, vr), (ps, pr)):
        assert rel_l2(a, b) <= 1e-10
    assert abs(rep2.max_divergence_after - rep[3]) <= 1e-8 * max(1.0, rep[3])


@pytest.mark.parametrize("dim", [2, 3])
def test_residual_norms(ref_oracle, dim):
    n = (19, 17, 1) if dim == 2 else (9, 8, 7)
    prob = GridProblem(*n, a=-1.0, b=-2.0, az=-1.0, c=0.3, e=0.2, f_const=0.7)
    prob.faces = [FaceBC.robin(1.0, 0.5, 0.2), FaceBC.robin(2.0, 0.25, 0.1), FaceBC.neumann(0.3),
                  FaceBC.dirichlet(1.0), FaceBC.dirichlet(0.0), FaceBC.neumann(0.1)]
    grid = np.random.Generator(np.random.PCG64(3)).standard_normal(prob.n)
    l2r, lir = ref_oracle.ref_residual_norms(prob, grid)
    l2s, lis = ref_oracle.rs_residual_norms(prob, grid)
    assert l2s == pytest.approx(l2r, rel=1e-14)
    assert lis == pytest.approx(lir, rel=1e-14)


NONLINEAR = [
    ("u2", [(abi.NL_POWER, 0.5, 2)]),
    ("sin", [(abi.NL_SIN, 2.0, 2)]),
    ("exp", [(abi.NL_EXP, 0.3, 2)]),
    ("cube_cos_abs", [(abi.NL_POWER, -0.4, 3), (abi.NL_COS, 0.5, 2), (abi.NL_ABS, 0.7, 2)]),
]


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("method,omega", [(abi.JACOBI, 1.0), (abi.GAUSS_SEIDEL, 1.0), (abi.SOR, 1.5)])
@pytest.mark.parametrize("name,terms", NONLINEAR)
def test_relaxation_nonlinear_terms(ref_oracle, dim, method, omega, name, terms):
    # EvalNonlinear at the node's old value inside every update
    # (relaxation.cpp:27-45,217-218,476-477; solver.cpp:884-885)
    dims = (21, 19, 1) if dim == 2 else (11, 10, 9)
    prob = GridProblem(*dims, a=-1.0, b=-1.0, az=-1.0, c=0.3)
    prob.faces = _mixed_faces_2d() if dim == 2 else _mixed_faces_3d()
    prob.nonlinear = terms
    opt = default_options(method=method, max_iter=40000, tol=1e-11, sor_omega=omega)
    ref, rs, rep = _pair(ref_oracle, prob, opt, rhs_latex="x*y-1")
    assert rel_l2(rs, ref) <= REL


@pytest.mark.parametrize("method", [abi.CG, abi.BICGSTAB, abi.MG_VCYCLE])
def test_nonlinear_terms_rejected_like_reference(ref_oracle, method):
    prob = GridProblem(17, 17, 1, a=-1.0, b=-1.0)
    prob.nonlinear = [(abi.NL_POWER, 1.0, 2)]
    opt = default_options(method=method, max_iter=100, tol=1e-8)
    # the reference's gate refuses first ("linear PDE required for this method",
    # backend_capability_matrix.cpp:265-267); SolvePDE itself says "... require
    # linear PDEs" (solver.cpp:502-504,550-552), the text the restatement gives
    st, _, _, err = ref_oracle.ref_solve(prob, opt)
    st2, _, rep = ref_oracle.rs_solve(prob, opt)
    assert st != 0 and st2 == abi.ERR_UNSUPPORTED
    assert "linear PDE" in err and "linear PDEs" in rep.message.decode()
