"""GPU checks of the serving loop (include/pdeb200_server.h) through the C ABI.

Requests of all three kinds run concurrently on several lanes; each result is
checked against the oracle (Poisson: FP64 folded residual <= 1e-10 by the
oracle's operator; heat: the oracle's forward-Euler series, rel L2 <= 1e-12)
or against the single-call entry point (projection, bitwise), and each
request's result must be bitwise the same alone and in a mixed stream."""
import numpy as np
import pytest

from pde_solver_b200 import abi, solver, synthetic
from pde_solver_b200.problem import FaceBC, default_options
from pde_solver_b200.server import Server, ServerError

pytestmark = pytest.mark.gpu


def folded_rel(oracle_mod, p, u):
    b, ax = oracle_mod.rs_folded(p, u)
    return np.linalg.norm(b - ax) / np.linalg.norm(b)


def poisson_mix():
    ps = [synthetic.poisson_request_problem(n, d, seed=100 + q)
          for q, (n, d) in enumerate([(65, 2), (100, 2), (33, 3), (129, 2), (24, 3), (257, 2)])]
    ps[1].faces = [FaceBC.dirichlet(0.3), FaceBC.neumann(0.0), FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(0.0),
                   FaceBC(), FaceBC()]
    return ps


def test_mixed_stream_results(oracle_mod):
    ps = poisson_mix()
    hp, hdt = synthetic.heat_problem(65)
    u, v, p0 = synthetic.projection_fields(96, seed=9)
    h = 1.0 / 95
    with Server(lanes=3) as s:
        pid = [s.submit_poisson(p) for p in ps[:3]]
        hid = s.submit_heat(hp, hdt, 200)
        jid = s.submit_projection(u, v, None, p0, 96, 96, 1, h, h, 1.0, 0.01)
        pid += [s.submit_poisson(p) for p in ps[3:]]
        pres = [s.wait(i) for i in pid]
        hout, hres = s.wait(hid)
        jout, jres = s.wait(jid)
        st = s.stats()
    for p, (out, res) in zip(ps, pres):
        assert res.status == abi.OK and res.rel_residual <= 1e-10
        assert folded_rel(oracle_mod, p, out) <= 1.01e-10
    assert hres.status == abi.OK
    ref = oracle_mod.rs_time_series(hp, 0.0, hdt, 201)  # u0 plus 200 steps
    assert np.linalg.norm(hout - ref) / np.linalg.norm(ref) <= 1e-12
    assert jres.status == abi.OK
    ug, vg, _, pg, _ = solver.project_velocity(u, v, None, p0, 96, 96, 1, h, h, 1.0, 0.01, 10000, 1e-10)
    n = 96 * 96
    assert np.array_equal(jout[:n], ug) and np.array_equal(jout[n:2 * n], vg) and np.array_equal(jout[2 * n:], pg)
    assert st.completed == len(ps) + 2 and st.failed == 0
    assert 0 < st.p50_ms <= st.p99_ms <= st.max_ms


def test_each_result_same_alone_and_in_the_mix():
    ps = poisson_mix()
    hp, hdt = synthetic.heat_problem(49)
    u, v, p0 = synthetic.projection_fields(64, seed=3)
    h = 1.0 / 63
    # alone: one request at a time
    alone = {}
    with Server(lanes=1) as s:
        for q, p in enumerate(ps):
            alone[("p", q)] = s.wait(s.submit_poisson(p))[0]
        alone["h"] = s.wait(s.submit_heat(hp, hdt, 200))[0]
        alone["j"] = s.wait(s.submit_projection(u, v, None, p0, 64, 64, 1, h, h, 1.0, 0.01))[0]
    # in a mix: everything at once, with extra traffic around it
    extra = [synthetic.poisson_request_problem(n, 2, seed=500 + n) for n in (70, 90, 150, 45)]
    with Server(lanes=4) as s:
        ids = {}
        for q, e in enumerate(extra[:2]):
            ids[("x", q)] = s.submit_poisson(e)
        for q, p in enumerate(ps):
            ids[("p", q)] = s.submit_poisson(p)
            if q == 2:
                ids["h"] = s.submit_heat(hp, hdt, 200)
                ids["j"] = s.submit_projection(u, v, None, p0, 64, 64, 1, h, h, 1.0, 0.01)
        for q, e in enumerate(extra[2:]):
            ids[("x", q + 2)] = s.submit_poisson(e)
        got = {k: s.wait(i) for k, i in ids.items()}
    groups = [r.group_size for k, (o, r) in got.items() if k[0] in ("p", "x")]
    assert max(groups) > 1  # some requests really were batched together
    for k, ref in alone.items():
        assert np.array_equal(got[k][0], ref), k


def test_light_load_runs_single_grid_mixed(oracle_mod):
    # with single_below set, a Poisson request that waits alone runs on its own
    # grid in mixed precision: the bits of pdeb200_solve with precision MIXED,
    # FP64 residual <= 1e-10 by the oracle's operator, and within 1e-8 of the
    # batched result of the same request
    ps = poisson_mix()[:3]
    with Server(lanes=2, single_below=4) as s:
        outs = [s.wait(s.submit_poisson(p)) for p in ps]
    with Server(lanes=1) as s:
        batched = [s.wait(s.submit_poisson(p))[0] for p in ps]
    opt = default_options(method=abi.MG_PCG, tol=1e-10, tol_mode=abi.TOL_RELATIVE, max_iter=500,
                          precision=abi.MIXED)
    for p, (out, res), b in zip(ps, outs, batched):
        assert res.status == abi.OK and res.group_size == 1 and res.rel_residual <= 1e-10
        assert folded_rel(oracle_mod, p, out) <= 1.01e-10
        ref, _ = solver.solve(p, opt)
        assert np.array_equal(out, ref)
        assert np.linalg.norm(out - b) <= 1e-8 * np.linalg.norm(b)


def test_admission_respects_the_hbm_budget():
    ps = [synthetic.poisson_request_problem(129, 2, seed=q) for q in range(8)]
    one = 80 * ps[0].n + (1 << 20)
    budget = int(2.5 * one)
    with Server(lanes=4, hbm_budget_bytes=budget) as s:
        ids = [s.submit_poisson(p) for p in ps]
        res = [s.wait(i)[1] for i in ids]
        st = s.stats()
        big = synthetic.poisson_request_problem(129, 3, seed=1)
        with pytest.raises(ServerError) as e:
            s.submit_poisson(big)
        assert e.value.status == abi.ERR_OOM
    assert all(r.status == abi.OK for r in res)
    assert st.bytes_peak <= budget
    assert max(r.group_size for r in res) <= 2


def test_fp64_lanes_match_single_call():
    ps = poisson_mix()[:3]
    with Server(lanes=2, precision=abi.FP64) as s:
        outs = [s.wait(s.submit_poisson(p)) for p in ps]
    opt = default_options(method=abi.MG_PCG, tol=1e-10, tol_mode=abi.TOL_RELATIVE, max_iter=500)
    for p, (out, res) in zip(ps, outs):
        assert res.status == abi.OK and res.group_size == 1
        ref, _ = solver.solve(p, opt)
        assert np.array_equal(out, ref)


@pytest.mark.parametrize("precision", [abi.MIXED, abi.FP64])
def test_device_resident_requests_match_host_requests(precision):
    # k and f already in HBM are used in place, and the result is written to
    # a device buffer; the numbers are those of the same request from host data
    import copy

    import torch

    ps = poisson_mix()[:4]
    dev = torch.device("cuda", 0)
    keep, dps, outs = [], [], []
    for p in ps:
        q = copy.copy(p)
        k = torch.from_numpy(p.k).to(dev)
        f = torch.from_numpy(p.f).to(dev)
        keep += [k, f]
        q.k, q.f, q.mem_space, q.k_dev, q.f_dev = None, None, abi.MEM_DEVICE, k.data_ptr(), f.data_ptr()
        dps.append(q)
        outs.append(torch.empty(p.n, dtype=torch.float64, device=dev))
    torch.cuda.synchronize()
    with Server(lanes=2, precision=precision) as s:
        host = [s.wait(s.submit_poisson(p))[0] for p in ps]
        ids = [s.submit_poisson(q, out=o.data_ptr()) for q, o in zip(dps, outs)]
        res = [s.wait(i)[1] for i in ids]
    assert all(r.status == abi.OK for r in res)
    for h, o in zip(host, outs):
        assert np.array_equal(h, o.cpu().numpy())
