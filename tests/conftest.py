"""Shared fixtures: the CPU oracle (test infrastructure) and the B200 library."""
import ctypes
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA library)")


def _gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


# Modules that run after the step, adjoint and shape parity suites (the
# selectable-solver rows and the frozen-turbulence gradient), so that those
# suites report first; the allocation-free module stays last.
_LATE = ("test_gpu_block_solvers.py", "test_gpu_adjoint_frozen_sa.py", "test_gpu_tutorial_schemes.py",
         "test_gpu_adjoint_c5.py", "test_gpu_decompose.py", "test_gpu_dual_sa.py")


def _order(item):
    name = Path(str(item.fspath)).name
    return 2 if name.startswith("test_zz") else (1 if name in _LATE else 0)


def pytest_collection_modifyitems(config, items):
    items.sort(key=_order)
    if _gpu_available():
        return
    skip = pytest.mark.skip(reason="no GPU in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    from tests.oracle_lib import load_oracle
    return load_oracle()


@pytest.fixture(scope="session")
def gpulib():
    import rhodst_b200
    return rhodst_b200.load_library()
