"""The drop-in boundary end to end: the reference's own dispatch
(SolveWithBackend, src/backend_solve.cpp:53) with its CUDA backend compiled in
(USE_CUDA) and served by pde_solver_b200/shim/cuda_solver_shim.cpp, against the
same call on the reference's CPU backend. Inputs are the reference's own
SolveInput forms: LaTeX right sides, LaTeX boundary values, LaTeX coefficients.
Fields agree to <= 1e-9 relative L2 at the same stopping tolerance."""
import numpy as np
import pytest

from pde_solver_b200 import abi, synthetic
from pde_solver_b200.problem import FaceBC, GridProblem, default_options

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def drop(ref_oracle, lib):
    if not ref_oracle.have_dropin():
        pytest.skip("oracle/_ref/libdropin.so not built")
    return ref_oracle


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_probe_reports_device(drop):
    import ctypes as C

    buf = C.create_string_buffer(256)
    assert drop.dropin().dropin_probe(buf, 256) == 1
    assert b"device" in buf.value


def test_config1_cg_through_solve_with_backend(drop):
    p = GridProblem(129, 129, 1, a=-1.0, b=-1.0)
    opt = default_options(method=abi.CG, max_iter=8000, tol=1e-10)
    st, gpu, res_gpu, sel, err = drop.dropin_solve(p, opt, 1, rhs_latex=synthetic.MMS_RHS_LATEX)
    assert st == 0 and sel, err
    st, cpu, res_cpu, _, err = drop.dropin_solve(p, opt, 0, rhs_latex=synthetic.MMS_RHS_LATEX)
    assert st == 0, err
    assert rel_l2(gpu, cpu) <= 1e-9
    x, y, _ = p.coords()
    exact = (np.sin(np.pi * x) * np.sin(np.pi * y)).reshape(-1)
    assert abs(np.abs(gpu - exact).max() - 5.02e-5) < 0.005e-5
    # SolveWithBackend's own post-solve residual (CPU ComputeResidualNorms) on the GPU field
    assert res_gpu[0] == pytest.approx(res_cpu[0], rel=0.1)


def test_sor_with_latex_boundary_values(drop):
    p = GridProblem(41, 33, 1, a=-1.0, b=-1.0, c=0.3)
    p.faces = [FaceBC.dirichlet(0.0), FaceBC.neumann(0.0), FaceBC.robin(1.0, 0.5, 0.2), FaceBC.dirichlet(0.0),
               FaceBC(), FaceBC()]
    faces = ["\\sin(\\pi*y)", "x*y", None, "1+x^2", None, None]
    opt = default_options(method=abi.SOR, sor_omega=1.6, max_iter=20000, tol=1e-11)
    st, gpu, _, sel, err = drop.dropin_solve(p, opt, 1, rhs_latex="\\cos(x)+y", face_latex=faces)
    assert st == 0 and sel, err
    st, cpu, _, _, err = drop.dropin_solve(p, opt, 0, rhs_latex="\\cos(x)+y", face_latex=faces)
    assert st == 0, err
    assert rel_l2(gpu, cpu) <= 1e-9


def test_3d_gauss_seidel_through_solve_pde_cuda(drop):
    # the reference's capability gate keeps CUDA to 2D, so 3D goes to SolvePDECuda directly
    p = GridProblem(13, 11, 10, a=-1.0, b=-1.0, az=-1.0)
    p.faces = [FaceBC.dirichlet(0.0), FaceBC.dirichlet(0.5), FaceBC.neumann(0.0), FaceBC.neumann(0.2),
               FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(0.0)]
    opt = default_options(method=abi.GAUSS_SEIDEL, max_iter=20000, tol=1e-11)
    st, gpu, err = drop.dropin_solve_cuda(p, opt, rhs_latex="x+y*z")
    assert st == 0, err
    st, cpu, _, _, err = drop.dropin_solve(p, opt, 0, rhs_latex="x+y*z")
    assert st == 0, err
    assert rel_l2(gpu, cpu) <= 1e-10


def test_latex_coefficients_jacobi(drop):
    p = GridProblem(17, 15, 1, a=-1.0, b=-1.0)
    lat = ["-(1+x*y)", "-(2+\\sin(x))", None, "x", None, None, "-0.1"]
    opt = default_options(method=abi.JACOBI, max_iter=40000, tol=1e-12)
    st, gpu, _, sel, err = drop.dropin_solve(p, opt, 1, rhs_latex="1", coef_latex=lat)
    assert st == 0 and sel, err
    st, cpu, _, _, err = drop.dropin_solve(p, opt, 0, rhs_latex="1", coef_latex=lat)
    assert st == 0, err
    assert rel_l2(gpu, cpu) <= 1e-10


def test_unsupported_reports_reference_error(drop):
    p = GridProblem(17, 17, 1, a=-1.0, b=-1.0)
    p.faces = [FaceBC.neumann(0.0), FaceBC.dirichlet(0.0), FaceBC.dirichlet(0.0), FaceBC.dirichlet(0.0),
               FaceBC(), FaceBC()]
    st, _, err = drop.dropin_solve_cuda(p, default_options(method=abi.CG))
    assert st != 0 and "Dirichlet" in err


def test_time_series_through_shim(drop):
    n = 33
    p = GridProblem(n, n, 1, a=-1.0, b=-1.0, ut=1.0)
    p.faces = [FaceBC.dirichlet(0.0), FaceBC.neumann(0.0), FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(0.0),
               FaceBC(), FaceBC()]
    x, y, _ = p.coords()
    p.u0 = np.exp(-40 * ((x - 0.5) ** 2 + (y - 0.5) ** 2)).reshape(-1)
    dt = 0.9 * (1.0 / (n - 1)) ** 2 / 4
    st, gpu, gframes, err = drop.dropin_time_series_cuda(p, 0.0, dt, 30)
    assert st == 0, err
    cpu, cframes = drop.ref_time_series(p, 0.0, dt, 30, keep_frames=True)
    assert rel_l2(gframes, cframes) <= 1e-12


def test_nonlinear_jacobi_through_solve_with_backend(drop):
    # pointwise nonlinear terms reach the CUDA backend: the reference's capability
    # row for CUDA advertises them (src/backend_capability_matrix.cpp:105)
    p = GridProblem(33, 29, 1, a=-1.0, b=-1.0)
    p.faces = [FaceBC.robin(1.0, 0.5, 0.2), FaceBC.dirichlet(0.0), FaceBC.neumann(0.3), FaceBC.dirichlet(1.0),
               FaceBC(), FaceBC()]
    p.nonlinear = [(abi.NL_POWER, 0.5, 2), (abi.NL_SIN, 1.0, 2)]
    opt = default_options(method=abi.JACOBI, max_iter=40000, tol=1e-11)
    st, gpu, _, sel, err = drop.dropin_solve(p, opt, 1, rhs_latex="x*y-1")
    assert st == 0 and sel, err
    st, cpu, _, _, err = drop.dropin_solve(p, opt, 0, rhs_latex="x*y-1")
    assert st == 0, err
    assert rel_l2(gpu, cpu) <= 1e-10


def test_nonlinear_sor_3d_through_solve_pde_cuda(drop):
    p = GridProblem(13, 11, 10, a=-1.0, b=-1.0, az=-1.0)
    p.faces = [FaceBC.dirichlet(0.0), FaceBC.dirichlet(0.5), FaceBC.neumann(0.0), FaceBC.neumann(0.2),
               FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(0.0)]
    p.nonlinear = [(abi.NL_EXP, 0.3, 2)]
    opt = default_options(method=abi.SOR, sor_omega=1.5, max_iter=40000, tol=1e-11)
    st, gpu, err = drop.dropin_solve_cuda(p, opt, rhs_latex="x-z")
    assert st == 0, err
    st, cpu, _, _, err = drop.dropin_solve(p, opt, 0, rhs_latex="x-z")
    assert st == 0, err
    assert rel_l2(gpu, cpu) <= 1e-10


def test_nonlinear_krylov_refused_with_reference_text(drop):
    p = GridProblem(17, 17, 1, a=-1.0, b=-1.0)
    p.nonlinear = [(abi.NL_POWER, 1.0, 2)]
    st, _, err = drop.dropin_solve_cuda(p, default_options(method=abi.CG))
    assert st != 0 and err == "Krylov solvers require linear PDEs"


def test_nonlinear_time_series_through_shim(drop):
    n = 33
    p = GridProblem(n, n, 1, a=-1.0, b=-1.0, ut=1.0)
    p.faces = [FaceBC.dirichlet(0.0), FaceBC.neumann(0.0), FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(0.0),
               FaceBC(), FaceBC()]
    x, y, _ = p.coords()
    p.u0 = np.exp(-40 * ((x - 0.5) ** 2 + (y - 0.5) ** 2)).reshape(-1)
    p.nonlinear = [(abi.NL_POWER, 0.8, 2), (abi.NL_SIN, -0.5, 2)]
    dt = 0.9 * (1.0 / (n - 1)) ** 2 / 4
    st, gpu, gframes, err = drop.dropin_time_series_cuda(p, 0.0, dt, 30)
    assert st == 0, err
    cpu, cframes = drop.ref_time_series(p, 0.0, dt, 30, keep_frames=True)
    assert rel_l2(gframes, cframes) <= 1e-12
