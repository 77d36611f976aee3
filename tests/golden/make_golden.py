"""Writes tests/golden/reference_cases.npz from the reference's own CPU solver
(oracle/_ref/libpderef.so, built by `make -C oracle` from the reference
sources). Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import cases  # noqa: E402
from oracle import oracle  # noqa: E402


def main():
    oracle.build(ref=True)
    out = {}
    for name, (p, opt, latex) in cases.solve_cases().items():
        st, grid, _, err = oracle.ref_solve(p, opt, rhs_latex=latex)
        assert st == 0, (name, err)
        if latex is not None:
            p.f = oracle.ref_materialize(latex, p)
        out[f"{name}/f"] = p.f
        out[f"{name}/grid"] = grid
    p, t0, dt, frames = cases.heat_case()
    grid, fr = oracle.ref_time_series(p, t0, dt, frames, keep_frames=True)
    out["heat_2d/grid"] = grid
    out["heat_2d/frames"] = fr
    c = cases.projection_case()
    st, u, v, w, pr, rep = oracle.ref_project(c["u"], c["v"], c["w"], c["p"], c["nx"], c["ny"], c["nz"], c["dx"],
                                              c["dy"], c["dz"], c["dt"], c["max_iter"], c["tol"])
    out["projection_2d/u"], out["projection_2d/v"], out["projection_2d/p"] = u, v, pr
    out["projection_2d/report"] = np.asarray(rep, dtype=np.float64)
    p, grid = cases.residual_case()
    l2, linf = oracle.ref_residual_norms(p, grid)
    out["residual_2d/norms"] = np.array([l2, linf])
    p, t0, dt, frames = cases.heat_nl_case()
    grid, fr = oracle.ref_time_series(p, t0, dt, frames, keep_frames=True)
    out["heat_nl_2d/grid"] = grid
    out["heat_nl_2d/frames"] = fr
    p, grid = cases.residual_nl_case()
    l2, linf = oracle.ref_residual_norms(p, grid)
    out["residual_nl_2d/norms"] = np.array([l2, linf])
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_cases.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, len(out), "arrays")


if __name__ == "__main__":
    main()
