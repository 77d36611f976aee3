"""Writes tests/golden/vtk_cases.npz: the bytes of the reference's own VTK
writers (WriteVtkStructuredPoints and WriteVtkXmlImageData with the CLI's
derived fields, from oracle/_ref/libpderef.so built by `make -C oracle` from
the reference sources) for the fields of cases.vtk_cases(). Run from the
repository root:

    python tests/golden/make_vtk_golden.py
"""
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import cases  # noqa: E402
from oracle import oracle  # noqa: E402


def main():
    oracle.build(ref=True)
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, p, f in cases.vtk_cases():
            path = os.path.join(tmp, name)
            oracle.ref_write_vtk(path + ".vtk", p, f)
            oracle.ref_write_vti(path + ".vti", p, f, derived=True)
            oracle.ref_write_vti(path + "_plain.vti", p, f, derived=False)
            for key, suffix in (("vtk", ".vtk"), ("vti", ".vti"), ("vti_plain", "_plain.vti")):
                with open(path + suffix, "rb") as fh:
                    out[f"{key}/{name}"] = np.frombuffer(fh.read(), dtype=np.uint8)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "vtk_cases.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, len(out), "arrays")


if __name__ == "__main__":
    main()
