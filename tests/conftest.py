"""Test configuration: the `gpu` marker, and imports of the product package
(p-trans_b200/, loaded as ``ptrans_b200``) and of the oracle (test
infrastructure)."""
import importlib.util
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "p-trans_b200")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def load_pkg():
    if "ptrans_b200" in sys.modules:
        return sys.modules["ptrans_b200"]
    spec = importlib.util.spec_from_file_location(
        "ptrans_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ptrans_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def _ensure_built():
    lib = os.path.join(PKG_DIR, "libptrans_b200.so")
    orc = os.path.join(ROOT, "oracle", "_build", "libptrans_oracle.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", PKG_DIR], check=True)
    if not os.path.exists(orc):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


_ensure_built()
load_pkg()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA sm_100 device (B200)")


def gpu_available() -> bool:
    try:
        import ctypes
        cudart = ctypes.CDLL("libcuda.so.1")
        n = ctypes.c_int(0)
        if cudart.cuInit(0) != 0:
            return False
        return cudart.cuDeviceGetCount(ctypes.byref(n)) == 0 and n.value > 0
    except OSError:
        return False


@pytest.fixture(scope="session")
def pkg():
    return load_pkg()


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as O
    O.lib()
    return O
