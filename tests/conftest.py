import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O

    O.build(ref=O.have_reference_sources())
    return O


@pytest.fixture(scope="session")
def ref_oracle(oracle_mod):
    if not oracle_mod.have_reference():
        pytest.skip("oracle/_ref/libpderef.so not built (reference sources absent)")
    return oracle_mod


@pytest.fixture(scope="session")
def lib():
    """libpdeb200.so, built in-tree; no fallback."""
    from pde_solver_b200 import abi

    if not os.path.exists(abi.LIB_PATH):
        import __graft_entry__

        __graft_entry__.build_library()
    return abi.load()
