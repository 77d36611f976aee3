"""The launch forms of the MG-PCG solve change no numbers: replaying each PCG
iteration as a captured CUDA graph or launching kernel by kernel, and
launching with programmatic stream serialization (each kernel may be
scheduled while its predecessor drains, and waits for it before touching
memory) or in plain stream order, give bit-identical fields and the same
iteration count."""
import os
import subprocess
import sys

import numpy as np
import pytest

from pde_solver_b200 import abi, solver, synthetic
from pde_solver_b200.problem import FaceBC, default_options

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _problem(n=65):
    p = synthetic.varcoef_poisson_3d(n, seed=5)
    p.faces = [FaceBC.dirichlet(0.0), FaceBC.neumann(0.1), FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(0.5),
               FaceBC.neumann(0.0), FaceBC.robin(2.0, 0.5, 0.1)]
    return p


def _opt():
    return default_options(method=abi.MG_PCG, tol=1e-10, tol_mode=abi.TOL_RELATIVE, max_iter=200)


@pytest.fixture(scope="module", autouse=True)
def _lib(lib):
    return lib


def test_graph_replay_changes_no_numbers(monkeypatch):
    p = _problem()
    a, ra = solver.solve(p, _opt())
    monkeypatch.setenv("PDEB200_NO_GRAPH", "1")
    b, rb = solver.solve(p, _opt())
    assert ra.iterations == rb.iterations and ra.iterations > 0
    assert np.array_equal(a, b)


def test_programmatic_launch_changes_no_numbers(tmp_path):
    # the launch attribute is chosen once per device context, so the plain
    # stream-order solve runs in a child process
    p = _problem()
    a, ra = solver.solve(p, _opt())
    out = tmp_path / "plain.npy"
    code = (
        "import sys, numpy as np\n"
        f"sys.path.insert(0, {REPO!r})\n"
        f"sys.path.insert(0, {os.path.join(REPO, 'tests')!r})\n"
        "from test_gpu_launch_forms import _problem, _opt\n"
        "from pde_solver_b200 import solver\n"
        "u, r = solver.solve(_problem(), _opt())\n"
        f"np.save({str(out)!r}, u)\n"
        "print(r.iterations)\n"
    )
    env = dict(os.environ, PDEB200_NO_PDL="1")
    res = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    assert int(res.stdout.strip().splitlines()[-1]) == ra.iterations
    assert np.array_equal(np.load(out), a)
