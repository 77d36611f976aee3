"""Golden fixtures from the reference's own CPU solver (tests/golden/, made by
tests/golden/make_golden.py from oracle/_ref): the oracle restatement must
reproduce them on the CPU, and the CUDA path through the C ABI on the GPU.
Tolerances: restatement rel L2 <= 1e-12 (same expression order as the
reference; 1e-10 for Krylov, whose OpenMP dot products follow the thread
count); CUDA path rel L2 <= 1e-10 for relaxation and the V-cycle, <= 1e-9
for Krylov (FMA contraction and reduction order are the only differences)."""
import os
import sys

import numpy as np
import pytest

from pde_solver_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import cases  # noqa: E402

FIX = np.load(os.path.join(HERE, "golden", "reference_cases.npz"))
SOLVE = sorted(cases.solve_cases().keys())


def rel_l2(a, b):
    d = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (d if d > 0 else 1.0)


def _case(name):
    p, opt, _ = cases.solve_cases()[name]
    p.f = FIX[f"{name}/f"].copy()
    return p, opt, FIX[f"{name}/grid"]


@pytest.mark.parametrize("name", SOLVE)
def test_restatement_matches_reference_fixture(oracle_mod, name):
    p, opt, ref = _case(name)
    st, got, _ = oracle_mod.rs_solve(p, opt)
    assert st in (abi.OK, abi.ERR_NOT_CONVERGED)
    # Krylov dot products are OpenMP reductions: their order follows the thread count
    tol = 1e-10 if opt.method in (abi.CG, abi.BICGSTAB, abi.GMRES) else 1e-12
    assert rel_l2(got, ref) <= tol


def test_restatement_heat_fixture(oracle_mod):
    p, t0, dt, frames = cases.heat_case()
    got, fr = oracle_mod.rs_time_series(p, t0, dt, frames, keep_frames=True)
    assert rel_l2(fr, FIX["heat_2d/frames"]) <= 1e-12


def test_restatement_projection_fixture(oracle_mod):
    c = cases.projection_case()
    st, u, v, w, pr, rep = oracle_mod.rs_project(c["u"], c["v"], c["w"], c["p"], c["nx"], c["ny"], c["nz"], c["dx"],
                                                c["dy"], c["dz"], c["dt"], c["max_iter"], c["tol"])
    assert st == 0
    for a, key in ((u, "u"), (v, "v"), (pr, "p")):
        assert rel_l2(a, FIX[f"projection_2d/{key}"]) <= 1e-10
    assert rep.poisson_iterations == int(FIX["projection_2d/report"][0])


@pytest.mark.parametrize("case,key", [(cases.residual_case, "residual_2d"), (cases.residual_nl_case, "residual_nl_2d")])
def test_restatement_residual_fixture(oracle_mod, case, key):
    p, grid = case()
    l2, linf = oracle_mod.rs_residual_norms(p, grid)
    assert l2 == pytest.approx(FIX[f"{key}/norms"][0], rel=1e-12)
    assert linf == pytest.approx(FIX[f"{key}/norms"][1], rel=1e-12)


def test_restatement_heat_nonlinear_fixture(oracle_mod):
    p, t0, dt, frames = cases.heat_nl_case()
    got, fr = oracle_mod.rs_time_series(p, t0, dt, frames, keep_frames=True)
    assert rel_l2(fr, FIX["heat_nl_2d/frames"]) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("name", SOLVE)
def test_cuda_path_matches_reference_fixture(lib, name):
    from pde_solver_b200 import solver

    p, opt, ref = _case(name)
    got, rep = solver.solve(p, opt, raise_on_error=False)
    assert rep.status in (abi.OK, abi.ERR_NOT_CONVERGED)
    tol = 1e-9 if opt.method in (abi.CG, abi.BICGSTAB, abi.GMRES) else 1e-10
    assert rel_l2(got, ref) <= tol


@pytest.mark.gpu
@pytest.mark.parametrize("case,key", [(cases.heat_case, "heat_2d"), (cases.heat_nl_case, "heat_nl_2d")])
def test_cuda_heat_matches_reference_fixture(lib, case, key):
    from pde_solver_b200 import solver

    p, t0, dt, frames = case()
    got, _ = solver.time_series(p, t0, dt, frames)
    assert rel_l2(got, FIX[f"{key}/grid"]) <= 1e-12


@pytest.mark.gpu
def test_cuda_projection_matches_reference_fixture(lib):
    from pde_solver_b200 import solver

    c = cases.projection_case()
    u, v, _, pr, rep = solver.project_velocity(c["u"], c["v"], c["w"], c["p"], c["nx"], c["ny"], c["nz"], c["dx"],
                                              c["dy"], c["dz"], c["dt"], c["max_iter"], c["tol"])
    # the same CG in the same order: only FMA contraction and the reduction
    # order differ, which moves the fields by about 1e-13
    assert rep.poisson_iterations == int(FIX["projection_2d/report"][0])
    for a, key in ((u, "u"), (v, "v"), (pr, "p")):
        d = rel_l2(a, FIX[f"projection_2d/{key}"])
        assert d <= 1e-10, (key, d)


@pytest.mark.gpu
@pytest.mark.parametrize("case,key", [(cases.residual_case, "residual_2d"), (cases.residual_nl_case, "residual_nl_2d")])
def test_cuda_residual_norms_match_reference_fixture(lib, case, key):
    from pde_solver_b200 import solver

    p, grid = case()
    l2, linf = solver.residual_norms(p, grid)
    assert l2 == pytest.approx(FIX[f"{key}/norms"][0], rel=1e-12)
    assert linf == pytest.approx(FIX[f"{key}/norms"][1], rel=1e-12)
