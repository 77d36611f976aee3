"""VTK output (include/pdeb200.h: pdeb200_write_vtk / pdeb200_write_vti).

Fixtures: tests/golden/vtk_cases.npz holds the bytes the reference's own
writers produce (WriteVtkStructuredPoints, WriteVtkXmlImageData with the CLI's
derived fields; src/vtk_writer.cpp) for cases.vtk_cases(), made by
tests/golden/make_vtk_golden.py. The bar is byte equality of whole files."""
import base64
import os
import struct
import sys

import numpy as np
import pytest

from pde_solver_b200 import abi, solver
from pde_solver_b200.problem import GridProblem

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import cases  # noqa: E402

FIX = np.load(os.path.join(HERE, "golden", "vtk_cases.npz"))
CASES = cases.vtk_cases()
NAMES = [c[0] for c in CASES]


def _fixture(key, name):
    return bytes(FIX[f"{key}/{name}"])


def _body(vtk: bytes) -> bytes:
    return vtk.split(b"LOOKUP_TABLE default\n", 1)[1]


@pytest.mark.parametrize("q", range(len(CASES)))
def test_host_formatter_matches_reference_fixture(lib, q):
    name, p, f = CASES[q]
    assert solver.vtk_values_host(f, p.nx) == _body(_fixture("vtk", name))


def test_host_formatter_matches_correct_rounding(lib):
    """Every float32 exponent: the text equals the correctly rounded %.6f of
    the float value (ties to even), which the C library also produces."""
    rng = np.random.default_rng(11)
    bits = rng.integers(0, 2**32, 200_000, dtype=np.uint64).astype(np.uint32)
    v = bits.view(np.float32)
    v = v[np.isfinite(v)].astype(np.float64)
    got = solver.vtk_values_host(v, 1 << 30).decode().split(" ")[:-1]
    assert got == ["%.6f" % x for x in v]


def test_host_formatter_matches_live_reference(ref_oracle, lib, tmp_path):
    rng = np.random.default_rng(5)
    p = GridProblem(33, 17, 3, bounds=(0.0, 2.0, -1.0, 1.0, 0.0, 0.5))
    f = rng.standard_normal(p.n) * 10.0 ** rng.integers(-9, 9, p.n)
    ref_oracle.ref_write_vtk(tmp_path / "r.vtk", p, f)
    assert solver.vtk_values_host(f, p.nx) == _body((tmp_path / "r.vtk").read_bytes())


@pytest.mark.gpu
@pytest.mark.parametrize("q", range(len(CASES)))
def test_gpu_writers_match_reference_files(lib, q, tmp_path):
    name, p, f = CASES[q]
    solver.write_vtk(tmp_path / "a.vtk", p, f)
    assert (tmp_path / "a.vtk").read_bytes() == _fixture("vtk", name)
    solver.write_vti(tmp_path / "a.vti", p, f, derived=True)
    assert (tmp_path / "a.vti").read_bytes() == _fixture("vti", name)
    solver.write_vti(tmp_path / "b.vti", p, f, derived=False)
    assert (tmp_path / "b.vti").read_bytes() == _fixture("vti_plain", name)


@pytest.mark.gpu
def test_gpu_writers_device_field_and_errors(lib, tmp_path):
    import torch

    name, p, f = CASES[1]
    dev = torch.from_numpy(f.copy()).to("cuda:0")
    solver.write_vtk(tmp_path / "d.vtk", p, dev.data_ptr())
    assert (tmp_path / "d.vtk").read_bytes() == _fixture("vtk", name)
    fractions = []
    solver.write_vti(tmp_path / "d.vti", p, dev.data_ptr(), progress=fractions.append)
    assert (tmp_path / "d.vti").read_bytes() == _fixture("vti", name)
    assert fractions and fractions[-1] == 1.0
    with pytest.raises(solver.SolveError) as e:
        solver.write_vtk(tmp_path / "missing" / "x.vtk", p, f)
    assert e.value.status == abi.ERR_INVALID and e.value.message == "failed to open output file"


def _decode_arrays(vti: bytes):
    """The float32 arrays of a VTI file (header: uint64 8, uint64 bytes)."""
    out = {}
    parts = vti.split(b'<DataArray type="Float32" Name="')[1:]
    for part in parts:
        name = part.split(b'"', 1)[0].decode()
        data = base64.b64decode(part.split(b">\n", 1)[1].split(b"\n", 1)[0])
        hsize, nbytes = struct.unpack("<QQ", data[:16])
        assert hsize == 8 and nbytes == len(data) - 16
        out[name] = np.frombuffer(data[16:], dtype=np.float32)
    return out


@pytest.mark.gpu
def test_gpu_writers_257_cubed(lib, tmp_path):
    """A 257^3 field (several pipelined chunks): the legacy text equals the
    host formatter's, and the VTI arrays decode to the float32 cast of the
    field and of the derived fields computed in numpy (same operation order)."""
    n = 257
    p = GridProblem(n, n, n, bounds=(0.0, 1.0, 0.0, 2.0, -1.0, 1.0), a=-1.0, b=-2.0, az=-0.5)
    rng = np.random.default_rng(9)
    f = rng.standard_normal(p.n) * 10.0 ** rng.integers(-6, 7, p.n)
    fractions = []
    solver.write_vtk(tmp_path / "big.vtk", p, f, progress=fractions.append)
    text = (tmp_path / "big.vtk").read_bytes()
    assert len(fractions) >= 2 and fractions[-1] == 1.0
    assert _body(text) == solver.vtk_values_host(f, n)
    solver.write_vti(tmp_path / "big.vti", p, f, derived=True)
    arrays = _decode_arrays((tmp_path / "big.vti").read_bytes())
    assert list(arrays) == ["solution", "gradient_x", "gradient_y", "gradient_z", "laplacian", "flux_x", "flux_y",
                            "flux_z", "energy_norm"]
    assert np.array_equal(arrays["solution"].view(np.uint32), f.astype(np.float32).view(np.uint32))
    u = f.reshape(n, n, n)
    dx, dy, dz = 1.0 / (n - 1), 2.0 / (n - 1), 2.0 / (n - 1)
    gx = np.zeros_like(u)
    gx[1:-1, 1:-1, 1:-1] = (u[1:-1, 1:-1, 2:] - u[1:-1, 1:-1, :-2]) * 0.5 * (1.0 / dx)
    lap = np.zeros_like(u)
    c = u[1:-1, 1:-1, 1:-1]
    lap[1:-1, 1:-1, 1:-1] = ((u[1:-1, 1:-1, 2:] - 2.0 * c + u[1:-1, 1:-1, :-2]) * (1.0 / (dx * dx))
                             + (u[1:-1, 2:, 1:-1] - 2.0 * c + u[1:-1, :-2, 1:-1]) * (1.0 / (dy * dy))
                             + (u[2:, 1:-1, 1:-1] - 2.0 * c + u[:-2, 1:-1, 1:-1]) * (1.0 / (dz * dz)))
    en = np.zeros_like(u)
    en[1:-1, 1:-1, 1:-1] = c * c
    for name, ref in (("gradient_x", gx), ("flux_x", -(-1.0) * gx), ("laplacian", lap), ("energy_norm", en)):
        assert np.array_equal(arrays[name].view(np.uint32), ref.reshape(-1).astype(np.float32).view(np.uint32)), name
