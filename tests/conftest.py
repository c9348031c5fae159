"""Shared test setup: the `gpu` marker, the package loader and the oracle.

`-m "not gpu"` tests run here on CPU: the oracle against the reference's known answers, the native host layout against
the oracle (bit-exact), the library loading and exporting every symbol include/blsgpu.h declares, and the multi-process
host logic. `-m gpu` tests run the device kernels through the C ABI against the oracle.
"""
import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def load_package():
    name = "blsgpu"
    if name in sys.modules:
        return sys.modules[name]
    pkg = ROOT / "blocklinearsystems.jl_b200"
    spec = importlib.util.spec_from_file_location(name, pkg / "__init__.py", submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")
    # build the native libraries once per session (no-op when up to date)
    import importlib
    b = importlib.util.spec_from_file_location("bls_build", ROOT / "blocklinearsystems.jl_b200" / "build.py")
    m = importlib.util.module_from_spec(b)
    b.loader.exec_module(m)
    m.build()
    import oracle as orc
    orc.build()


@pytest.fixture(scope="session")
def bls():
    return load_package()


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle
