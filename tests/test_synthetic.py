"""CPU checks of the seeded synthetic workloads: each generator gives the
shapes, ranges and distributions its benchmark configuration names, and the
same seed gives the same bits."""
import numpy as np
import pytest

from pde_solver_b200 import abi, synthetic


def test_varcoef_poisson_3d_fields_and_faces():
    p = synthetic.varcoef_poisson_3d(33, seed=5)
    q = synthetic.varcoef_poisson_3d(33, seed=5)
    assert p.n == 33 ** 3 and p.coef_kind == abi.COEF_DIVK
    assert np.array_equal(p.k, q.k) and np.array_equal(p.f, q.f)
    # k = box^3(exp(g)), sigma 1: positive, smoothed (narrower than the raw
    # log-normal: log-variance well below 1)
    assert p.k.min() > 0.0
    assert np.var(np.log(p.k)) < 0.5
    raw = np.exp(np.random.Generator(np.random.PCG64(5)).standard_normal((33, 33, 33)))
    assert np.allclose(p.k.reshape(33, 33, 33), synthetic.box_smooth(raw, 3))
    # f = -F with F ~ N(0,1)
    assert abs(p.f.mean()) < 0.02 and abs(p.f.std() - 1.0) < 0.02
    kinds = [f.kind for f in p.faces]
    assert kinds == [abi.BC_DIRICHLET, abi.BC_DIRICHLET, abi.BC_NEUMANN, abi.BC_NEUMANN, abi.BC_ROBIN,
                     abi.BC_DIRICHLET]
    robin = p.faces[4]
    assert (robin.alpha, robin.beta, robin.gamma) == (1.0, 1.0, 0.0)
    assert all(f.value == 0.0 for f in p.faces)


def test_convection_diffusion_3d():
    p = synthetic.convection_diffusion_3d(17, seed=99)
    assert p.n == 17 ** 3 and p.coef_kind == abi.COEF_CONST
    assert (p.a, p.b, p.az) == (-1e-2, -1e-2, -1e-2)
    assert abs(np.sqrt(p.c ** 2 + p.d ** 2 + p.dz ** 2) - 1.0) < 1e-12  # unit convection vector
    assert p.f.min() >= -1.0 and p.f.max() <= 1.0 and p.f.std() > 0.5  # uniform on [-1, 1]
    q = synthetic.convection_diffusion_3d(17, seed=99)
    assert np.array_equal(p.f, q.f) and (p.c, p.d, p.dz) == (q.c, q.d, q.dz)


def test_batch_sides_log_uniform():
    s2, s3 = synthetic.batch_sides(2048, 256, seed=4242)
    assert len(s2) == 2048 and len(s3) == 256
    assert s2.min() >= 33 and s2.max() <= 513 and s3.min() >= 17 and s3.max() <= 129
    # log-uniform: the median is near the geometric mean of the range
    assert abs(np.log(np.median(s2)) - 0.5 * np.log(33 * 513)) < 0.15
    assert abs(np.log(np.median(s3)) - 0.5 * np.log(17 * 129)) < 0.2
    a2, a3 = synthetic.batch_sides(2048, 256, seed=4242)
    assert np.array_equal(s2, a2) and np.array_equal(s3, a3)


def test_batch_members_per_member_seeds():
    ms = synthetic.batch_members(6, 2)
    assert [m.nz > 1 for m in ms] == [False] * 6 + [True] * 2
    assert all(m.coef_kind == abi.COEF_DIVK and m.k.min() > 0 for m in ms)
    again = synthetic.batch_members(6, 2)
    assert all(np.array_equal(a.k, b.k) and np.array_equal(a.f, b.f) for a, b in zip(ms, again))
    # member q's fields depend on (seed, q) only, not on the batch size
    more = synthetic.batch_members(7, 2)
    assert np.array_equal(ms[3].k, more[3].k)


def test_serving_requests_stream():
    stream = synthetic.serving_requests(3000, seed=11, rate_hz=100.0)
    t = np.array([a for a, _, _ in stream])
    assert np.all(np.diff(t) > 0)
    # Poisson process: mean inter-arrival 1/rate
    assert abs(np.mean(np.diff(t)) - 0.01) < 0.001
    kinds = [k for _, k, _ in stream]
    share = {k: kinds.count(k) / len(kinds) for k in ("poisson", "heat", "projection")}
    assert abs(share["poisson"] - 0.6) < 0.03 and abs(share["heat"] - 0.25) < 0.03
    assert abs(share["projection"] - 0.15) < 0.03
    for _, k, sp in stream:
        if k == "poisson":
            lo, hi = (65, 129) if sp["dim"] == 3 else (65, 513)
            assert lo <= sp["n"] <= hi
        elif k == "heat":
            assert 65 <= sp["n"] <= 257 and sp["steps"] == 200
        else:
            assert 256 <= sp["n"] <= 1024
    assert synthetic.serving_requests(50, seed=11, rate_hz=100.0) == stream[:50]


@pytest.mark.parametrize("dim", [2, 3])
def test_heat_problem_dt_at_0_9_cfl(dim):
    p, dt = synthetic.heat_problem(33, dim)
    h = 1.0 / 32
    assert dt == pytest.approx(0.9 * h * h / (2 * dim), rel=1e-15)
    assert p.ut == 1.0 and p.a == -1.0 and p.b == -1.0 and p.az == (-1.0 if dim == 3 else 0.0)
    assert p.u0.max() == pytest.approx(1.0, abs=0.05) and p.u0.min() >= 0.0
