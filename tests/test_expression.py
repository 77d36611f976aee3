"""Expressions of x, y, z, t compiled once and evaluated at every node
(include/pdeb200.h: pdeb200_eval_expression / pdeb200_expression_value).

Fixtures: tests/golden/expression_cases.npz, the reference's own
ExpressionEvaluator (src/expression_eval.cpp) on the grids of
cases.expression_cases(), made by tests/golden/make_expression_golden.py.
Tolerances: the host evaluation calls the same C library functions as the
reference and must match bit for bit; the GPU evaluation uses CUDA's double
functions (a few ulp from the C library), so values agree to rel 1e-13 with
an absolute floor of 1e-14 * max|value| for results near zero, and the
NaN / inf pattern must be identical."""
import os
import sys

import numpy as np
import pytest

from pde_solver_b200 import abi, solver
from pde_solver_b200.problem import GridProblem

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import cases  # noqa: E402

FIX = np.load(os.path.join(HERE, "golden", "expression_cases.npz"))
CASES = cases.expression_cases()
ERRORS = cases.expression_errors()


def _grid(nx, ny, nz, b):
    return GridProblem(nx=nx, ny=ny, nz=nz, bounds=b)


def _nodes(nx, ny, nz, b):
    """Node coordinates in grid order, with the reference's xmin + i*dx."""
    nzz = nz if nz > 1 else 1
    dx = (b[1] - b[0]) / (nx - 1)
    dy = (b[3] - b[2]) / (ny - 1)
    dz = (b[5] - b[4]) / (nzz - 1) if nzz > 1 else 0.0
    for k in range(nzz):
        for j in range(ny):
            for i in range(nx):
                yield b[0] + i * dx, b[2] + j * dy, (b[4] + k * dz if nzz > 1 else 0.0)


def _same(got, ref, rtol=0.0, afloor=0.0):
    nan_g, nan_r = np.isnan(got), np.isnan(ref)
    assert np.array_equal(nan_g, nan_r), "NaN pattern differs"
    inf_g, inf_r = np.isinf(got), np.isinf(ref)
    assert np.array_equal(inf_g, inf_r), "inf pattern differs"
    assert np.array_equal(got[inf_g], ref[inf_r])
    fin = ~(nan_r | inf_r)
    if not fin.any():
        return
    g, r = got[fin], ref[fin]
    if rtol == 0.0:
        assert np.array_equal(g, r), f"max |diff| {np.max(np.abs(g - r))}"
    else:
        tol = rtol * np.abs(r) + afloor * np.max(np.abs(r))
        assert np.all(np.abs(g - r) <= tol), f"max |diff| {np.max(np.abs(g - r))}"


@pytest.mark.parametrize("q", range(len(CASES)))
def test_host_evaluation_matches_reference_fixture(lib, q):
    latex, nx, ny, nz, b, t = CASES[q]
    got = np.array([solver.expression_value(latex, x, y, z, t) for x, y, z in _nodes(nx, ny, nz, b)])
    _same(got, FIX[f"value/{q}"])


def test_parse_errors_match_reference_messages(lib):
    for latex, msg in zip(ERRORS, FIX["errors"]):
        with pytest.raises(solver.SolveError) as e:
            solver.expression_value(latex, 0.5, 0.5)
        assert e.value.status == abi.ERR_INVALID
        assert e.value.message == str(msg), latex


def test_host_evaluation_matches_live_reference(ref_oracle, lib):
    """Random nodes and times against the reference library itself."""
    rng = np.random.default_rng(7)
    for latex, nx, ny, nz, b, _ in CASES[:12]:
        t = float(rng.uniform(0.0, 2.0))
        g = _grid(nx, ny, nz, b)
        ref = ref_oracle.ref_materialize(latex, g, t)
        got = np.array([solver.expression_value(latex, x, y, z, t) for x, y, z in _nodes(nx, ny, nz, b)])
        _same(got, ref)


def test_program_size_limit(lib):
    """A sum of 256 terms (511 operations) fits the 512-operation program; 257 do not."""
    ok = "+".join(["x"] * 256)
    assert solver.expression_value(ok, 2.0, 0.0) == 512.0
    with pytest.raises(solver.SolveError) as e:
        solver.expression_value("+".join(["x"] * 257), 1.0, 0.0)
    assert "too large" in e.value.message


@pytest.mark.gpu
@pytest.mark.parametrize("q", range(len(CASES)))
def test_gpu_grid_matches_reference_fixture(lib, q):
    latex, nx, ny, nz, b, t = CASES[q]
    got = solver.eval_expression(latex, _grid(nx, ny, nz, b), t)
    _same(got, FIX[f"value/{q}"], rtol=1e-13, afloor=1e-14)


@pytest.mark.gpu
def test_gpu_errors_and_device_output(lib):
    import torch

    g = _grid(65, 33, 17, (0.0, 1.0, 0.0, 2.0, -1.0, 1.0))
    with pytest.raises(solver.SolveError) as e:
        solver.eval_expression(r"\sin(\pi x)", g)
    assert e.value.message == "unknown identifier: pix"
    latex = r"\exp(-x)\cos(\pi*y)\sinh(z) + t"
    host = solver.eval_expression(latex, g, 0.5)
    dev = torch.full((g.n,), float("nan"), dtype=torch.float64, device="cuda:0")
    solver.eval_expression(latex, g, 0.5, out=dev.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(dev.cpu().numpy(), host)
    ref = np.array([solver.expression_value(latex, x, y, z, 0.5) for x, y, z in _nodes(65, 33, 17, g.bounds)])
    _same(host, ref, rtol=1e-13, afloor=1e-14)


@pytest.mark.gpu
def test_gpu_large_grid_sampled(lib):
    """257^3 nodes: sampled nodes against the host evaluation."""
    g = _grid(257, 257, 257, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0))
    latex = r"-3\pi^2\sin(\pi*x)\sin(\pi*y)\sin(\pi*z)"
    got = solver.eval_expression(latex, g)
    rng = np.random.default_rng(3)
    idx = rng.integers(0, g.n, 2000)
    h = 1.0 / 256
    for q in idx:
        i, j, k = q % 257, (q // 257) % 257, q // (257 * 257)
        ref = solver.expression_value(latex, i * h, j * h, k * h)
        assert abs(got[q] - ref) <= 1e-13 * abs(ref) + 1e-14 * 3 * np.pi**2


def _face_nodes(face, nx, ny, nz, b):
    """Face-local nodes in pdeb200_face order, coordinates as the reference computes them."""
    nzz = nz if nz > 1 else 1
    dx = (b[1] - b[0]) / (nx - 1)
    dy = (b[3] - b[2]) / (ny - 1)
    dz = (b[5] - b[4]) / (nzz - 1) if nzz > 1 else 0.0
    w = ny if face <= 1 else nx
    h = nzz if face <= 3 else ny
    for q in range(h):
        for a in range(w):
            if face <= 1:
                yield (b[0] if face == 0 else b[1]), b[2] + a * dy, (b[4] + q * dz if nzz > 1 else 0.0)
            elif face <= 3:
                yield b[0] + a * dx, (b[2] if face == 2 else b[3]), (b[4] + q * dz if nzz > 1 else 0.0)
            else:
                yield b[0] + a * dx, b[2] + q * dy, (b[4] if face == 4 else b[5])


def _eval_bc(latex, lin, x, y, z):
    """EvalExpr (src/backends/cpu/cpu_utils.cpp:520-530) over the host evaluation."""
    if latex:
        try:
            v = solver.expression_value(latex, x, y, z)
            if np.isfinite(v):
                return v
        except solver.SolveError:
            pass
    return lin[0] + lin[1] * x + lin[2] * y + lin[3] * z


@pytest.mark.gpu
@pytest.mark.parametrize("nz", [1, 9])
def test_gpu_face_expressions_with_linear_fallback(lib, nz):
    b = (-1.0, 2.0, 0.5, 1.5, -0.25, 0.75)
    g = _grid(17, 11, nz, b)
    lin = (0.5, -1.25, 2.0, 0.75)
    forms = [r"\sin(\pi*x)\cos(y) + z", r"\frac{1}{x}", r"\log(y - 1)", r"\sin(\pi x)", "", None]
    for face in range(6 if nz > 1 else 4):
        for latex in forms:
            got = solver.eval_face_expression(latex, g, face, lin)
            ref = np.array([_eval_bc(latex, lin, x, y, z) for x, y, z in _face_nodes(face, 17, 11, nz, b)])
            _same(got, ref, rtol=1e-13, afloor=1e-14)
