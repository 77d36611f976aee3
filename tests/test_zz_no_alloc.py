"""The Jacobi entry point that allocates nothing (pdeb200_jacobi_noalloc).

It exists for callers that cannot let a library allocate device memory, such
as code running inside another runtime's fixed memory arena or hosts that
forbid allocation after start-up; its scratch is a fixed device array inside
the library. This file runs last so a failure here leaves every other test
already run. The inputs and outputs are device buffers the test owns (torch);
the two calls in a row must match the allocating entry point (pdeb200_solve,
same Jacobi semantics) to 1e-12 relative L2: the same kernels run in the same
order, so only the scratch location differs."""
import ctypes as C

import numpy as np
import pytest

from pde_solver_b200 import abi, solver
from pde_solver_b200.problem import FaceBC, GridProblem, default_options

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _problem():
    p = GridProblem(17, 15, 13, coef_kind=abi.COEF_DIVK)
    rng = np.random.Generator(np.random.PCG64(17))
    p.k = np.exp(0.5 * rng.standard_normal(p.n))
    p.f = rng.standard_normal(p.n)
    p.faces = [FaceBC.dirichlet(0.0), FaceBC.dirichlet(0.5), FaceBC.neumann(0.0), FaceBC.neumann(0.2),
               FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(0.0)]
    return p


def test_noalloc_jacobi_matches_allocating_entry_twice():
    import torch

    lib = abi.load()
    p = _problem()
    max_iter, tol = 20000, 1e-10
    ref, rep = solver.solve(p, default_options(method=abi.JACOBI, max_iter=max_iter, tol=tol))
    assert rep.status == abi.OK

    dev = torch.device("cuda", 0)
    k_d = torch.from_numpy(p.k).to(dev)
    f_d = torch.from_numpy(p.f).to(dev)
    out_d = torch.empty(p.n, dtype=torch.float64, device=dev)
    dp = GridProblem(p.nx, p.ny, p.nz, coef_kind=abi.COEF_DIVK, mem_space=abi.MEM_DEVICE)
    dp.faces = p.faces
    dp.k_dev, dp.f_dev = k_d.data_ptr(), f_d.data_ptr()
    cp = dp.to_c()
    torch.cuda.synchronize()
    results = []
    for _ in range(2):
        out_d.fill_(123.0)  # stale contents must not leak into the result
        torch.cuda.synchronize()
        r = abi.Report()
        st = lib.pdeb200_jacobi_noalloc(C.byref(cp), max_iter, tol, 0, None, C.c_void_p(out_d.data_ptr()),
                                        C.byref(r))
        assert st == abi.OK, r.message
        assert r.iterations == rep.iterations
        results.append(out_d.cpu().numpy().copy())
    for got in results:
        assert rel_l2(got, ref) <= 1e-12
    assert np.array_equal(results[0], results[1])


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch

    lib = abi.load()
    dev = torch.device("cuda", 0)
    big = GridProblem(129, 129, 129, a=-1.0, b=-1.0, az=-1.0, mem_space=abi.MEM_DEVICE)
    out_d = torch.empty(8, dtype=torch.float64, device=dev)  # never written: rejected before any launch
    cp = big.to_c()
    r = abi.Report()
    st = lib.pdeb200_jacobi_noalloc(C.byref(cp), 10, 1e-6, 0, None, C.c_void_p(out_d.data_ptr()), C.byref(r))
    assert st == abi.ERR_UNSUPPORTED
    assert b"1048576" in r.message
