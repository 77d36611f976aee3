"""CPU checks of the C-ABI boundary: the library loads, exports every entry
point include/*.h declares, and the ctypes mirror matches the C layout."""
import ctypes as C
import os
import re

import pytest

from pde_solver_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    inc = os.path.join(ROOT, "include")
    text = "".join(open(os.path.join(inc, f)).read() for f in sorted(os.listdir(inc)) if f.endswith(".h"))
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pdeb200_[a-z0-9_]+)\s*\(", text)) - {"pdeb200_frame_cb"})


def test_library_exports_every_declared_symbol(lib):
    syms = declared_symbols()
    assert len(syms) >= 10
    for s in syms:
        assert hasattr(lib, s), s


def test_abi_version(lib):
    assert lib.pdeb200_abi_version() == abi.PDEB200_ABI_VERSION


@pytest.mark.parametrize("which,cls", [(0, abi.Face), (1, abi.Problem), (2, abi.Options), (3, abi.Report),
                                       (4, abi.TimeOptions), (5, abi.ProjectionOptions), (6, abi.ProjectionReport),
                                       (7, abi.BatchOptions), (8, abi.BatchStats), (9, abi.ServerOptions),
                                       (10, abi.Request), (11, abi.Result), (12, abi.ServerStats)])
def test_struct_layout_matches_header(oracle_mod, which, cls):
    assert oracle_mod.restate().rs_sizeof(which) == C.sizeof(cls)


def test_default_options_match_reference_solver_config(lib):
    o = abi.Options()
    lib.pdeb200_default_options(C.byref(o))
    # SolverConfig defaults, include/pde_types.h:282-303
    assert (o.max_iter, o.tol, o.sor_omega, o.gmres_restart) == (10000, 1e-6, 1.5, 30)
    assert (o.mg_pre_smooth, o.mg_post_smooth, o.mg_coarse_iters, o.mg_max_levels) == (2, 2, 50, 10)


def test_status_strings(lib):
    assert lib.pdeb200_status_string(abi.ERR_DEGENERATE) == b"degenerate PDE center coefficient"
    assert lib.pdeb200_status_string(abi.OK) == b""


def test_probe_without_device_reports_reason(lib):
    from tests.conftest import gpu_available

    note = C.create_string_buffer(256)
    ok = lib.pdeb200_probe(note, 256)
    if not gpu_available():
        assert ok == 0 and len(note.value) > 0


def test_solve_rejects_invalid_input(lib):
    # validation happens before any device work; null arguments never reach CUDA
    rep = abi.Report()
    assert lib.pdeb200_solve(None, None, None, C.byref(rep)) == abi.ERR_INVALID
