"""GPU parity of the core path through the C ABI against the oracle
(plain-C restatement pinned to the reference; tests/test_oracle_pins.py).

Tolerances: the reference methods run the reference's algorithm, so fields
agree to rounding (rel L2 <= 1e-10; FMA contraction on the GPU is the only
difference). The MG-PCG form solves the folded system to 1e-12 relative
residual on both sides and must agree to <= 1e-9 rel L2 (the plain FP64 path's parity bar)."""
import numpy as np
import pytest

from pde_solver_b200 import abi, solver, synthetic
from pde_solver_b200.problem import FaceBC, GridProblem, default_options

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    d = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (d if d > 0 else 1.0)


def mixed_faces_2d():
    return [FaceBC.robin(1.0, 0.5, 0.2), FaceBC.dirichlet(0.0), FaceBC.neumann(0.3), FaceBC.dirichlet(1.0),
            FaceBC(), FaceBC()]


def mixed_faces_3d():
    return [FaceBC.dirichlet(0.0), FaceBC.dirichlet(0.5), FaceBC.neumann(0.0), FaceBC.neumann(0.2),
            FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(0.0)]


@pytest.fixture(scope="module", autouse=True)
def _lib(lib):
    return lib


# ------------------------------------------------------------------ apply

def _problems_for_apply():
    rng = np.random.Generator(np.random.PCG64(11))
    out = []
    for dims in [(13, 11, 1), (9, 8, 7)]:
        p = GridProblem(*dims, a=-1.3, b=-0.7, az=-2.0, c=0.4, d=-0.2, dz=0.3, e=0.1)
        p.faces = mixed_faces_3d()
        out.append(("const", p))
        q = GridProblem(*dims, coef_kind=abi.COEF_DIVK, c=0.3, e=-0.2)
        q.k = np.exp(rng.standard_normal(q.n))
        out.append(("divk", q))
        r = GridProblem(*dims, coef_kind=abi.COEF_NODAL)
        r.nodal = rng.standard_normal(7 * r.n)
        out.append(("nodal", r))
    return out


@pytest.mark.parametrize("name,prob", _problems_for_apply())
def test_apply_matches_oracle(oracle_mod, name, prob):
    x = np.random.Generator(np.random.PCG64(3)).standard_normal(prob.n)
    got = solver.apply(prob, x)
    ref = oracle_mod.rs_apply(prob, x)
    assert rel_l2(got, ref) <= 1e-14, name


# ----------------------------------------------------------------- Jacobi

@pytest.mark.parametrize("dims", [(25, 21, 1), (13, 11, 9)])
def test_jacobi_mixed_bc(oracle_mod, dims):
    p = GridProblem(*dims, a=-1.0, b=-1.0, az=-1.0, c=0.5)
    p.faces = mixed_faces_2d() if dims[2] == 1 else mixed_faces_3d()
    x, y, z = p.coords()
    p.f = (x * y - 1.0 + 0 * z).reshape(-1)
    opt = default_options(method=abi.JACOBI, max_iter=20000, tol=1e-11)
    got, rep = solver.solve(p, opt)
    st, ref, rrep = oracle_mod.rs_solve(p, opt)
    assert st == 0 and rep.status == abi.OK
    assert abs(rep.iterations - rrep.iterations) <= 1
    assert rel_l2(got, ref) <= 1e-10


def test_jacobi_nodal_coefficients(oracle_mod):
    p = GridProblem(15, 13, 1, coef_kind=abi.COEF_NODAL)
    x, y, _ = p.coords()
    ones = np.ones(p.n)
    a = -(1 + (x * y)).reshape(-1) * ones
    b = -(2 + np.sin(x) + 0 * y).reshape(-1)
    p.nodal = np.concatenate([a, b, -ones, (x + 0 * y).reshape(-1), 0 * ones, 0 * ones, -0.1 * ones])
    p.faces = mixed_faces_2d()
    p.f_const = 1.0
    opt = default_options(method=abi.JACOBI, max_iter=40000, tol=1e-12)
    got, rep = solver.solve(p, opt)
    st, ref, _ = oracle_mod.rs_solve(p, opt)
    assert st == 0 and rel_l2(got, ref) <= 1e-10


# --------------------------------------------------------------------- CG

def test_cg_config1_mms(oracle_mod):
    p = synthetic.poisson_mms_2d(129)
    opt = default_options(method=abi.CG, max_iter=8000, tol=1e-10)
    got, rep = solver.solve(p, opt)
    st, ref, rrep = oracle_mod.rs_solve(p, opt)
    assert st == 0 and rep.status == abi.OK
    assert rel_l2(got, ref) <= 1e-9
    x, y, _ = p.coords()
    exact = (np.sin(np.pi * x) * np.sin(np.pi * y)).reshape(-1)
    assert abs(np.abs(got - exact).max() - 5.02e-5) < 0.005e-5


def test_cg_random_rhs(oracle_mod):
    p = GridProblem(65, 49, 1, a=-1.0, b=-2.0, e=-0.5)
    p.f = np.random.Generator(np.random.PCG64(9)).standard_normal(p.n)
    opt = default_options(method=abi.CG, max_iter=8000, tol=1e-9)
    got, rep = solver.solve(p, opt)
    st, ref, rrep = oracle_mod.rs_solve(p, opt)
    assert st == 0 and rep.status == abi.OK
    assert abs(rep.iterations - rrep.iterations) <= 2
    assert rel_l2(got, ref) <= 1e-9


def test_cg_rejects_non_dirichlet():
    p = GridProblem(17, 17, 1, a=-1.0, b=-1.0)
    p.faces = mixed_faces_2d()
    got, rep = solver.solve(p, default_options(method=abi.CG), raise_on_error=False)
    assert rep.status == abi.ERR_UNSUPPORTED


# ----------------------------------------------------------------- MG-PCG

@pytest.mark.parametrize("n", [17, 33])
def test_mgpcg_varcoef_3d(oracle_mod, n):
    p = synthetic.varcoef_poisson_3d(n, seed=5)
    opt = default_options(method=abi.MG_PCG, tol=1e-12, tol_mode=abi.TOL_RELATIVE, max_iter=300)
    got, rep = solver.solve(p, opt)
    st, ref, rrep = oracle_mod.rs_solve(p, opt)
    assert st == 0 and rep.status == abi.OK
    assert rep.rel_residual <= 1e-12
    assert abs(rep.iterations - rrep.iterations) <= 1
    assert rel_l2(got, ref) <= 1e-9


@pytest.mark.parametrize("dims", [(34, 34, 34), (24, 19, 30), (129, 20, 17), (100, 37, 1), (258, 131, 1)])
def test_mgpcg_uneven_sizes(oracle_mod, dims):
    # even and mixed sizes: non-nested levels and semi-coarsening
    nx, ny, nz = dims
    rng = np.random.Generator(np.random.PCG64(sum(dims)))
    p = GridProblem(nx, ny, nz, coef_kind=abi.COEF_DIVK)
    p.k = np.exp(0.5 * rng.standard_normal(p.n))
    p.f = rng.standard_normal(p.n)
    if nz == 1:
        p.faces = [FaceBC.dirichlet(0.0), FaceBC.neumann(0.0), FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(1.0),
                   FaceBC(), FaceBC()]
    else:
        p.faces = [FaceBC.dirichlet(0.0), FaceBC.neumann(0.0), FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(1.0),
                   FaceBC.neumann(0.1), FaceBC.dirichlet(0.0)]
    opt = default_options(method=abi.MG_PCG, tol=1e-12, tol_mode=abi.TOL_RELATIVE, max_iter=300)
    got, rep = solver.solve(p, opt)
    st, ref, rrep = oracle_mod.rs_solve(p, opt)
    assert st == 0 and rep.status == abi.OK
    assert rrep.iterations <= 20
    assert abs(rep.iterations - rrep.iterations) <= 1
    assert rel_l2(got, ref) <= 1e-9


def test_mgpcg_relative_1e10_true_residual(oracle_mod):
    p = synthetic.varcoef_poisson_3d(33, seed=8)
    opt = default_options(method=abi.MG_PCG, tol=1e-10, tol_mode=abi.TOL_RELATIVE, max_iter=300)
    got, rep = solver.solve(p, opt)
    b, ax = oracle_mod.rs_folded(p, got)
    true_rel = np.linalg.norm(b - ax) / np.linalg.norm(b)
    assert true_rel <= 1e-10
    assert rep.rel_residual == pytest.approx(true_rel, rel=1e-3)


def test_mgpcg_2d_poisson_matches_reference_cg_solution(oracle_mod):
    p = synthetic.poisson_mms_2d(129)
    got, rep = solver.solve(p, default_options(method=abi.MG_PCG, tol=1e-12, tol_mode=abi.TOL_RELATIVE))
    ref_opt = default_options(method=abi.CG, max_iter=8000, tol=1e-13)
    st, ref, _ = oracle_mod.rs_solve(p, ref_opt)
    assert rel_l2(got, ref) <= 1e-9


def test_fused_sweep_form_matches_color_passes(monkeypatch):
    # the single-pass red-black sweep and the two colour passes are the same
    # arithmetic; results agree to rounding and iteration counts match
    p = synthetic.varcoef_poisson_3d(33, seed=4)
    opt = default_options(method=abi.MG_PCG, tol=1e-11, tol_mode=abi.TOL_RELATIVE, max_iter=200)
    a, ra = solver.solve(p, opt)
    monkeypatch.setenv("PDEB200_FUSED_SWEEP", "1")
    b, rb = solver.solve(p, opt)
    assert ra.iterations == rb.iterations
    assert rel_l2(b, a) <= 1e-12


@pytest.mark.parametrize("dims", [(33, 33, 33), (129, 100, 1), (40, 30, 20)])
def test_single_block_tail_matches_per_level_launches(monkeypatch, dims):
    # the small levels run as one launch; the arithmetic is that of the
    # per-level kernels, so fields agree to rounding and iteration counts match
    nx, ny, nz = dims
    rng = np.random.Generator(np.random.PCG64(nx + ny + nz))
    p = GridProblem(nx, ny, nz, coef_kind=abi.COEF_DIVK)
    p.k = np.exp(0.5 * rng.standard_normal(p.n))
    p.f = rng.standard_normal(p.n)
    p.faces = [FaceBC.dirichlet(0.0), FaceBC.neumann(0.0), FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(1.0),
               FaceBC.neumann(0.1) if nz > 1 else FaceBC(), FaceBC.dirichlet(0.0) if nz > 1 else FaceBC()]
    opt = default_options(method=abi.MG_PCG, tol=1e-11, tol_mode=abi.TOL_RELATIVE, max_iter=200)
    a, ra = solver.solve(p, opt)
    monkeypatch.setenv("PDEB200_NO_TAIL", "1")
    b, rb = solver.solve(p, opt)
    assert ra.iterations == rb.iterations
    assert rel_l2(a, b) <= 1e-12


def test_graph_replay_matches_direct_launches(monkeypatch):
    # one MG-PCG iteration replayed as a CUDA graph runs the same kernels in
    # the same order as direct launches: identical fields and iteration counts
    p = synthetic.varcoef_poisson_3d(33, seed=12)
    opt = default_options(method=abi.MG_PCG, tol=1e-11, tol_mode=abi.TOL_RELATIVE, max_iter=200)
    a, ra = solver.solve(p, opt)
    monkeypatch.setenv("PDEB200_NO_GRAPH", "1")
    b, rb = solver.solve(p, opt)
    assert ra.iterations == rb.iterations
    assert np.array_equal(a, b)
    assert ra.kernel_launches == rb.kernel_launches


@pytest.mark.parametrize("which", ["divk", "const"])
def test_staged_sweep_matches_colour_passes(monkeypatch, which):
    # with PDEB200_STAGED_SWEEP, levels of 2^18+ nodes smooth with the
    # single-pass staged sweep; it does the arithmetic of two colour passes,
    # so fields agree to rounding
    if which == "divk":
        p = synthetic.varcoef_poisson_3d(65, seed=21)
    else:
        p = GridProblem(65, 70, 66, a=-1.0, b=-1.0, az=-1.0)
        p.f = np.random.Generator(np.random.PCG64(2)).standard_normal(p.n)
        p.faces = [FaceBC.dirichlet(0.0), FaceBC.neumann(0.0), FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(1.0),
                   FaceBC.neumann(0.1), FaceBC.dirichlet(0.0)]
    opt = default_options(method=abi.MG_PCG, tol=1e-11, tol_mode=abi.TOL_RELATIVE, max_iter=200)
    a, ra = solver.solve(p, opt)
    monkeypatch.setenv("PDEB200_STAGED_SWEEP", "1")
    b, rb = solver.solve(p, opt)
    assert abs(ra.iterations - rb.iterations) <= 1
    assert rel_l2(a, b) <= 1e-10


@pytest.mark.parametrize("which", ["divk", "const", "uneven"])
def test_marching_sweep_matches_colour_passes(monkeypatch, which):
    # with PDEB200_MARCH, levels of 2^18+ nodes smooth with the single-pass
    # marching sweep (k_rbgs_march); it does the arithmetic of two colour
    # passes, so the solve agrees with the colour-pass form to rounding at the
    # same iteration count
    if which == "divk":
        p = synthetic.varcoef_poisson_3d(65, seed=21)
    elif which == "const":
        p = GridProblem(65, 70, 66, a=-1.0, b=-1.0, az=-1.0, c=0.2)
        p.f = np.random.Generator(np.random.PCG64(2)).standard_normal(p.n)
        p.faces = [FaceBC.dirichlet(0.0), FaceBC.neumann(0.0), FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(1.0),
                   FaceBC.neumann(0.1), FaceBC.dirichlet(0.0)]
    else:
        rng = np.random.Generator(np.random.PCG64(8))
        p = GridProblem(131, 37, 70, coef_kind=abi.COEF_DIVK)
        p.k = np.exp(0.5 * rng.standard_normal(p.n))
        p.f = rng.standard_normal(p.n)
        p.faces = [FaceBC.robin(2.0, 0.02, 0.0), FaceBC.dirichlet(0.0), FaceBC.neumann(0.0), FaceBC.dirichlet(0.5),
                   FaceBC.dirichlet(0.0), FaceBC.neumann(0.2)]
    opt = default_options(method=abi.MG_PCG, tol=1e-11, tol_mode=abi.TOL_RELATIVE, max_iter=200)
    b, rb = solver.solve(p, opt)
    monkeypatch.setenv("PDEB200_MARCH", "1")
    a, ra = solver.solve(p, opt)
    assert ra.status == abi.OK and rb.status == abi.OK
    assert ra.iterations == rb.iterations
    assert rel_l2(a, b) <= 1e-12
