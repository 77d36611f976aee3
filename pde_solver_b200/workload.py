"""Run the benchmark workloads through the C ABI without timing harness:

    python -m pde_solver_b200.workload --n 257 --solves 2 [--method MG_PCG] [--mixed]
    python -m pde_solver_b200.workload --batch 2048,256 --solves 2

Used as the target of profiler runs (each solve is the step `bench.py` times;
--batch runs the batched workload: n2d 2D grids and n3d 3D grids).
"""
from __future__ import annotations

import argparse
import sys

from . import abi, solver, synthetic
from .problem import default_options


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=257)
    ap.add_argument("--solves", type=int, default=2)
    ap.add_argument("--method", default="MG_PCG", choices=["MG_PCG", "MG_BICGSTAB", "CG", "JACOBI"])
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--workload", default="varcoef3d", choices=["varcoef3d", "convdiff3d"])
    ap.add_argument("--batch", default="", help="n2d,n3d: batched workload instead of one grid")
    ap.add_argument("--bf16", action="store_true")
    ap.add_argument("--tuned", action="store_true", help="batch schedule from pde_solver_b200/batch_tune_cache.txt")
    ap.add_argument("--retune", default="", help="autotune the batch and append the result to this cache file")
    a = ap.parse_args(argv)
    if a.batch:
        from .batch import Batch

        n2d, n3d = (int(v) for v in a.batch.split(","))
        ms = synthetic.batch_members(n2d, n3d)
        import os

        kw = {}
        if a.retune:
            kw = dict(autotune=1, tune_cache=a.retune)
        elif a.tuned:
            kw = dict(autotune=1, tune_cache=os.path.join(os.path.dirname(__file__), "batch_tune_cache.txt"))
        b = Batch(ms, bf16_coefficients=1 if a.bf16 else 0, **kw)
        o = b.options()
        print(f"schedule tile=({o.tile_x},{o.tile_y},{o.tile_z}) pre={o.pre_smooth} post={o.post_smooth} "
              f"inner_tol={o.inner_tol:g}", flush=True)
        for _ in range(a.solves):
            b.solve(1e-10)
            s = b.stats
            print(f"members={s.members} converged={s.converged} cycles={s.cycles} device_ms={s.device_ms:.2f} "
                  f"launches={s.kernel_launches}", flush=True)
        b.close()
        return 0
    if a.workload == "varcoef3d":
        p = synthetic.varcoef_poisson_3d(a.n, seed=1234)
    else:
        p = synthetic.convection_diffusion_3d(a.n, seed=99)
    opt = default_options(method=getattr(abi, a.method), tol=1e-10, tol_mode=abi.TOL_RELATIVE, max_iter=400,
                          precision=abi.MIXED if a.mixed else abi.FP64)
    for _ in range(a.solves):
        _, rep = solver.solve(p, opt)
        print(f"iterations={rep.iterations} outer={rep.outer_iterations} rel_residual={rep.rel_residual:.3e} "
              f"device_ms={rep.device_ms:.2f} launches={rep.kernel_launches}", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
