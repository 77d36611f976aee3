"""GPU checks of the batched solver (include/pdeb200_batch.h) through the C ABI.

Each member is solved by FP32 MG-PCG inside FP64 refinement to a relative
FP64 residual of 1e-10; the oracle (FP64 restatement, solved to 1e-13) gives
the reference solution: the FP64 residual of every batch result is checked
with the oracle's folded operator, and its error against the oracle solution
must stay within the conditioning of the problem (rel L2 <= 1e-7). A member's
result must be bitwise the same alone, in a mixed batch, and with or without
the CUDA graph."""
import numpy as np
import pytest

from pde_solver_b200 import abi, synthetic
from pde_solver_b200.batch import Batch, BatchError
from pde_solver_b200.problem import FaceBC, GridProblem, default_options

pytestmark = pytest.mark.gpu

TOL = 1e-10
FIXED = dict(tile_x=32, tile_y=16, tile_z=8, pre_smooth=2, post_smooth=2, inner_tol=1e-4)


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def mixed_members():
    rng = np.random.Generator(np.random.PCG64(77))
    out = []
    # 2D divergence form, Dirichlet 0 (odd and even sides)
    for n in (33, 50):
        p = GridProblem(n, n, 1, coef_kind=abi.COEF_DIVK)
        p.k = np.exp(0.5 * rng.standard_normal(p.n))
        p.f = rng.standard_normal(p.n)
        out.append(p)
    # 2D rectangle with Neumann / Robin / non-zero Dirichlet faces
    p = GridProblem(61, 37, 1, coef_kind=abi.COEF_DIVK)
    p.k = np.exp(0.5 * rng.standard_normal(p.n))
    p.f = rng.standard_normal(p.n)
    p.faces = [FaceBC.dirichlet(0.5), FaceBC.neumann(0.2), FaceBC.robin(1.0, 1.0, 0.1), FaceBC.dirichlet(0.0),
               FaceBC(), FaceBC()]
    out.append(p)
    # 3D divergence form with mixed faces (the 257^3 workload's faces)
    out.append(synthetic.varcoef_poisson_3d(17, seed=3, sigma=0.5))
    # 3D constant coefficients, uneven sides
    p = GridProblem(20, 18, 16, a=-1.0, b=-1.0, az=-1.0)
    p.f = rng.standard_normal(p.n)
    # Robin on a min face: the reference's max-face Robin closure amplifies
    # (u_N = (gamma - beta/h u_N-1)/(alpha - beta/h)) and leaves no SPD system
    p.faces = [FaceBC.dirichlet(0.0), FaceBC.neumann(0.0), FaceBC.robin(2.0, 1.0, 0.0), FaceBC.dirichlet(0.0),
               FaceBC.neumann(0.1), FaceBC.dirichlet(1.0)]
    out.append(p)
    # 2D constant coefficients, large side
    p = GridProblem(129, 129, 1, a=-1.0, b=-1.0)
    p.f = rng.standard_normal(p.n)
    out.append(p)
    return out


@pytest.fixture(scope="module")
def members():
    return mixed_members()


@pytest.fixture(scope="module")
def batch_result(members):
    b = Batch(members, **FIXED)
    reps = b.solve(TOL)
    fields = b.read()
    stats = b.stats
    b.close()
    return reps, fields, stats


def test_batch_converges_and_matches_oracle(oracle_mod, members, batch_result):
    reps, fields, stats = batch_result
    assert stats.converged == len(members) and stats.graph == 1
    for p, r, u in zip(members, reps, fields):
        assert r.converged and r.rel_residual <= TOL
        assert r.outer_iterations >= 1
        b, ax = oracle_mod.rs_folded(p, u)
        true_rel = np.linalg.norm(b - ax) / np.linalg.norm(b)
        assert true_rel <= 1.01 * TOL
        assert true_rel == pytest.approx(r.rel_residual, rel=1e-3)
        opt = default_options(method=abi.MG_PCG, tol=1e-13, tol_mode=abi.TOL_RELATIVE, max_iter=400)
        st, ref, _ = oracle_mod.rs_solve(p, opt)
        assert st == 0
        assert rel_l2(u, ref) <= 1e-7


def test_member_alone_equals_member_in_mix(members, batch_result):
    _, fields, _ = batch_result
    for j in (1, 3, 4):
        with Batch([members[j]], **FIXED) as b:
            b.solve(TOL)
            alone = b.read()[0]
        assert np.array_equal(alone, fields[j])
    # a different mix (members reordered, one repeated)
    order = [4, 0, 4, 2]
    with Batch([members[q] for q in order], **FIXED) as b:
        b.solve(TOL)
        got = b.read()
    for q, u in zip(order, got):
        assert np.array_equal(u, fields[q])


def test_graph_and_direct_launches_agree(members, batch_result):
    _, fields, _ = batch_result
    with Batch(members, no_graph=1, **FIXED) as b:
        b.solve(TOL)
        assert b.stats.graph == 0
        got = b.read()
    for u, v in zip(got, fields):
        assert np.array_equal(u, v)


def test_bf16_hierarchy_coefficients(oracle_mod, members):
    with Batch(members, bf16_coefficients=1, **FIXED) as b:
        reps = b.solve(TOL)
        fields = b.read()
    for p, r, u in zip(members, reps, fields):
        assert r.converged and r.rel_residual <= TOL
        bb, ax = oracle_mod.rs_folded(p, u)
        assert np.linalg.norm(bb - ax) / np.linalg.norm(bb) <= 1.01 * TOL


def test_load_rhs_replaces_every_member(oracle_mod, members):
    with Batch(members, **FIXED) as b:
        rng = np.random.Generator(np.random.PCG64(5))
        f = rng.standard_normal(b.nodes)
        b.load_rhs(f)
        b.solve(TOL)
        got = b.read()
    for q, (p, u) in enumerate(zip(members, got)):
        p2 = GridProblem(**{k: getattr(p, k) for k in ("nx", "ny", "nz", "a", "b", "az", "coef_kind", "k")})
        p2.faces = p.faces
        p2.f = f[b.offsets[q]:b.offsets[q] + p.n].copy()
        bb, ax = oracle_mod.rs_folded(p2, u)
        assert np.linalg.norm(bb - ax) / np.linalg.norm(bb) <= 1.01 * TOL


def test_autotune_cache_round_trip(tmp_path, members):
    cache = str(tmp_path / "tune.txt")
    with Batch(members[:3], autotune=1, tune_cache=cache) as b:
        b.solve(TOL)
        first = b.options()
        assert b.stats.tuned_from_cache == 0 and b.stats.tune_ms > 0
    with Batch(members[:3], autotune=1, tune_cache=cache) as b:
        b.solve(TOL)
        again = b.options()
        assert b.stats.tuned_from_cache == 1
    for k in ("tile_x", "tile_y", "tile_z", "pre_smooth", "post_smooth"):
        assert getattr(first, k) == getattr(again, k)
    assert first.inner_tol == again.inner_tol


def test_batch_of_the_batched_workload_shapes(oracle_mod):
    # a scaled-down draw of the batched workload (sides 33..129 2D, 17..33 3D)
    ms = synthetic.batch_members(24, 6, seed=11, hi2=129, hi3=33)
    with Batch(ms, **FIXED) as b:
        reps = b.solve(TOL)
        fields = b.read()
    for p, r, u in zip(ms, reps, fields):
        assert r.converged
        bb, ax = oracle_mod.rs_folded(p, u)
        assert np.linalg.norm(bb - ax) / np.linalg.norm(bb) <= 1.01 * TOL


def test_batch_rejects_unsupported_members():
    p = GridProblem(9, 9, 1, coef_kind=abi.COEF_NODAL)
    p.nodal = np.zeros(7 * p.n)
    with pytest.raises(BatchError) as e:
        Batch([p])
    assert e.value.status == abi.ERR_UNSUPPORTED
    q = GridProblem(4, 4, 1, a=-1.0, b=-1.0)
    with pytest.raises(BatchError) as e:
        Batch([q])
    assert e.value.status == abi.ERR_UNSUPPORTED


def test_compaction_changes_no_numbers(batch_result, members):
    # rebuilding the tables for the unfinished members keeps every member's
    # tiles and their order, so the fields are the same bits
    _, fields, stats = batch_result
    with Batch(members, no_compact=1, **FIXED) as b:
        b.solve(TOL)
        assert b.stats.compactions == 0
        got = b.read()
    for u, v in zip(got, fields):
        assert np.array_equal(u, v)
    ms = synthetic.batch_members(40, 8, seed=3, hi2=257, hi3=49)
    for p in ms[::2]:
        p.f = np.zeros(p.n)  # these finish at the first outer step
    with Batch(ms, **FIXED) as b:
        b.solve(TOL)
        compacted = b.read()
        assert b.stats.compactions >= 1
    with Batch(ms, no_compact=1, **FIXED) as b:
        b.solve(TOL)
        plain = b.read()
    for u, v in zip(compacted, plain):
        assert np.array_equal(u, v)
