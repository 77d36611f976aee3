"""The Jacobi entry point that allocates nothing (pdeb200_jacobi_noalloc).

It exists for callers that cannot let a library allocate device memory, such
as code running inside another runtime's fixed memory arena or hosts that
forbid allocation after start-up; its scratch is a fixed device array inside
the library. This file runs last so a failure here leaves every other test
already run. The inputs and outputs are device buffers the test owns (torch);
two calls in a row must match the allocating entry point (pdeb200_solve, same
Jacobi semantics) to 1e-12 relative L2: the same kernels run in the same
order, so only the scratch location differs. The cases cover the three
coefficient forms, 2D and 3D, and runs that end on an odd and on an even
iteration (the last field is then in the scratch array or in the output)."""
import ctypes as C

import numpy as np
import pytest

from pde_solver_b200 import abi, solver
from pde_solver_b200.problem import FaceBC, GridProblem, default_options

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _divk_3d():
    p = GridProblem(17, 15, 13, coef_kind=abi.COEF_DIVK)
    rng = np.random.Generator(np.random.PCG64(17))
    p.k = np.exp(0.5 * rng.standard_normal(p.n))
    p.f = rng.standard_normal(p.n)
    p.faces = [FaceBC.dirichlet(0.0), FaceBC.dirichlet(0.5), FaceBC.neumann(0.0), FaceBC.neumann(0.2),
               FaceBC.robin(1.0, 1.0, 0.0), FaceBC.dirichlet(0.0)]
    return p


def _const_2d():
    p = GridProblem(41, 29, a=-1.0, b=-1.0, e=0.0)
    rng = np.random.Generator(np.random.PCG64(5))
    p.f = rng.standard_normal(p.n)
    p.faces = [FaceBC.dirichlet(0.25), FaceBC.neumann(0.1), FaceBC.dirichlet(0.0), FaceBC.robin(1.0, 1.0, 0.0),
               FaceBC(), FaceBC()]
    return p


def _nodal_3d():
    p = GridProblem(13, 11, 9, coef_kind=abi.COEF_NODAL)
    rng = np.random.Generator(np.random.PCG64(11))
    n = p.n
    nodal = np.zeros(7 * n)
    nodal[0:n] = -1.0 - 0.3 * rng.random(n)       # a
    nodal[n:2 * n] = -1.0 - 0.3 * rng.random(n)   # b
    nodal[2 * n:3 * n] = -0.8 - 0.2 * rng.random(n)  # az
    nodal[3 * n:4 * n] = 0.2 * rng.standard_normal(n)  # c
    nodal[6 * n:7 * n] = -0.1 * rng.random(n)     # e
    p.nodal = nodal
    p.f = rng.standard_normal(n)
    p.faces = [FaceBC.dirichlet(0.0), FaceBC.dirichlet(1.0), FaceBC.neumann(0.0), FaceBC.dirichlet(0.0),
               FaceBC.dirichlet(0.0), FaceBC.robin(1.0, 0.5, 0.2)]
    return p


CASES = {"divk_3d": _divk_3d, "const_2d": _const_2d, "nodal_3d": _nodal_3d}


def _device_problem(p, dev):
    import torch

    dp = GridProblem(p.nx, p.ny, p.nz, coef_kind=p.coef_kind, mem_space=abi.MEM_DEVICE,
                     a=p.a, b=p.b, az=p.az, c=p.c, d=p.d, dz=p.dz, e=p.e, f_const=p.f_const)
    dp.faces = p.faces
    keep = []
    for name in ("k", "f", "nodal"):
        arr = getattr(p, name)
        if arr is not None:
            t = torch.from_numpy(np.ascontiguousarray(arr)).to(dev)
            keep.append(t)
            setattr(dp, name + "_dev", t.data_ptr())
    return dp, keep


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("stop", ["converged", "odd", "even"])
def test_noalloc_jacobi_matches_allocating_entry_twice(case, stop):
    import torch

    lib = abi.load()
    p = CASES[case]()
    # "odd"/"even": tol 0 never stops early, so exactly max_iter iterations run
    max_iter, tol = {"converged": (100000, 1e-10), "odd": (301, 0.0), "even": (300, 0.0)}[stop]
    ref, rep = solver.solve(p, default_options(method=abi.JACOBI, max_iter=max_iter, tol=tol))
    want = abi.OK if stop == "converged" else abi.ERR_NOT_CONVERGED
    assert rep.status == want, rep.message
    if stop != "converged":
        assert rep.iterations == max_iter

    dev = torch.device("cuda", 0)
    dp, keep = _device_problem(p, dev)
    out_d = torch.empty(p.n, dtype=torch.float64, device=dev)
    cp = dp.to_c()
    torch.cuda.synchronize()

    def call():
        out_d.fill_(123.0)  # stale contents must not leak into the result
        torch.cuda.synchronize()
        r = abi.Report()
        st = lib.pdeb200_jacobi_noalloc(C.byref(cp), max_iter, tol, 0, None, C.c_void_p(out_d.data_ptr()),
                                        C.byref(r))
        assert st == want, r.message
        assert r.iterations == rep.iterations
        return out_d.cpu().numpy().copy()

    results = [call(), call()]
    for got in results:
        assert rel_l2(got, ref) <= 1e-12
    assert np.array_equal(results[0], results[1])
    del keep


def test_noalloc_call_leaves_free_device_memory_unchanged():
    import torch

    lib = abi.load()
    p = _divk_3d()
    dev = torch.device("cuda", 0)
    dp, keep = _device_problem(p, dev)
    out_d = torch.empty(p.n, dtype=torch.float64, device=dev)
    cp = dp.to_c()
    torch.cuda.synchronize()
    free = []
    for _ in range(3):  # the first call loads the kernels; the later ones must allocate nothing
        r = abi.Report()
        st = lib.pdeb200_jacobi_noalloc(C.byref(cp), 500, 1e-10, 0, None, C.c_void_p(out_d.data_ptr()), C.byref(r))
        assert st in (abi.OK, abi.ERR_NOT_CONVERGED), r.message
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info(0)[0])
    assert free[1] == free[2]
    del keep


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch

    lib = abi.load()
    dev = torch.device("cuda", 0)
    out_d = torch.empty(8, dtype=torch.float64, device=dev)  # never written: rejected before any launch
    big = GridProblem(129, 129, 129, a=-1.0, b=-1.0, az=-1.0, mem_space=abi.MEM_DEVICE)
    cp = big.to_c()
    r = abi.Report()
    st = lib.pdeb200_jacobi_noalloc(C.byref(cp), 10, 1e-6, 0, None, C.c_void_p(out_d.data_ptr()), C.byref(r))
    assert st == abi.ERR_UNSUPPORTED
    assert b"1048576" in r.message
    # under the node limit, but ceil(nx/32)*ceil(ny/8) = 8193 blocks
    thin = GridProblem(32 * 8193, 3, a=-1.0, b=-1.0, mem_space=abi.MEM_DEVICE)
    cp = thin.to_c()
    r = abi.Report()
    st = lib.pdeb200_jacobi_noalloc(C.byref(cp), 10, 1e-6, 0, None, C.c_void_p(out_d.data_ptr()), C.byref(r))
    assert st == abi.ERR_UNSUPPORTED
    assert b"8192" in r.message or b"too wide" in r.message
