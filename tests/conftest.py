"""Shared fixtures: the package (loaded as tgh_b200) and the CPU oracle (test infrastructure)."""
import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "treegeneralizedharmonic.jl_b200"


def load_package():
    if "tgh_b200" in sys.modules:
        return sys.modules["tgh_b200"]
    spec = importlib.util.spec_from_file_location("tgh_b200", PKG / "__init__.py",
                                                  submodule_search_locations=[str(PKG)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["tgh_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


sys.path.insert(0, str(Path(__file__).resolve().parent))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built native library")


@pytest.fixture(scope="session")
def tgh():
    return load_package()


@pytest.fixture(scope="session")
def oracle():
    import oracle_binding
    return oracle_binding.Oracle.load()


@pytest.fixture(scope="session")
def bench_module():
    """bench.py as a module: the workloads' definitions (cases, forests) the tests share."""
    spec = importlib.util.spec_from_file_location("bench_workloads", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod
