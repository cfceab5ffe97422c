"""Shared fixtures.  `-m "not gpu"` runs the CPU suite (oracle, host logic, ABI);
`-m gpu` runs the CUDA parity tests through the C ABI."""
import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG_DIR = ROOT / "reservoir-splatting_b200"
sys.path.insert(0, str(ROOT / "oracle"))


def load_package():
    if "reservoir_splatting_b200" in sys.modules:
        return sys.modules["reservoir_splatting_b200"]
    spec = importlib.util.spec_from_file_location("reservoir_splatting_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["reservoir_splatting_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built sm_100a library")
    load_package()


@pytest.fixture(scope="session")
def rs():
    return load_package()


@pytest.fixture(scope="session")
def scenes(rs):
    import reservoir_splatting_b200.scenes as S
    return S


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle as O
    O.build()
    return O
