"""Writes tests/golden/expression_cases.npz: the reference's ExpressionEvaluator
(oracle/_ref/libpderef.so, built by `make -C oracle` from the reference
sources) evaluated on the grids of cases.expression_cases(), and its error
messages for cases.expression_errors(). Run from the repository root:

    python tests/golden/make_expression_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import cases  # noqa: E402
from oracle import oracle  # noqa: E402
from pde_solver_b200.problem import GridProblem  # noqa: E402


def grid_of(nx, ny, nz, b):
    return GridProblem(nx=nx, ny=ny, nz=nz, bounds=b)


def main():
    oracle.build(ref=True)
    out = {}
    for q, (latex, nx, ny, nz, b, t) in enumerate(cases.expression_cases()):
        out[f"value/{q}"] = oracle.ref_materialize(latex, grid_of(nx, ny, nz, b), t)
    msgs = []
    for latex in cases.expression_errors():
        try:
            oracle.ref_materialize(latex, grid_of(3, 3, 1, (0.0, 1.0, 0.0, 1.0, 0.0, 0.0)))
            msgs.append("")
        except RuntimeError as e:
            msgs.append(str(e))
    out["errors"] = np.array(msgs)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "expression_cases.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, len(out), "arrays")


if __name__ == "__main__":
    main()
