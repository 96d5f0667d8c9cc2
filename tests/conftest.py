"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device (B200); the rest
run on the CPU: the oracle against the golden fixtures, the host logic, and
the C ABI library's loading and exports."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run with -m gpu on a B200)")
    config.addinivalue_line("markers", "slow: full-size (n=30000) cases")


def load_build_recipe():
    """pactae_b200/build.py, loaded by path: importing the package would load
    the (possibly stale) library before it is rebuilt."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("pactae_b200_build", ROOT / "pactae_b200" / "build.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def pytest_sessionstart(session):
    # Build the oracle (test infrastructure) and the CUDA library in-tree
    # before any test module imports them.
    import oracle

    if not oracle.ORACLE_LIB.exists():
        oracle.build()
    load_build_recipe().build()


def load_cases() -> list[dict]:
    return json.loads((GOLDEN / "cases.json").read_text())["cases"]


def golden_match(name: str) -> np.ndarray:
    return np.load(GOLDEN / f"match_{name}.npy")


@pytest.fixture(scope="session")
def cases() -> list[dict]:
    return load_cases()


@pytest.fixture(scope="session")
def cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ctx(cuda_available):
    if not cuda_available:
        pytest.skip("no CUDA device")
    import pactae_b200 as pb

    c = pb.Context(device=0)
    yield c
    c.close()
