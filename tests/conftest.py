"""Test configuration.

Markers: `gpu` tests need a CUDA device and the built libcbf.so; everything else
runs on CPU (oracle pinning, host logic, ABI/export checks, CSV layout, gloo).
"""
import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG_DIR = ROOT / "cudabifurcation3.0_b200"

if str(ROOT / "oracle") not in sys.path:
    sys.path.insert(0, str(ROOT / "oracle"))
if str(ROOT / "tests") not in sys.path:
    sys.path.insert(0, str(ROOT / "tests"))


def load_cbf():
    """Import the package directory (its name is not a Python identifier)."""
    name = "cbf_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libcbf.so")


@pytest.fixture(scope="session")
def cbf():
    mod = load_cbf()
    if not mod.LIB_PATH.exists():
        from importlib import import_module  # noqa: F401
        build_spec = importlib.util.spec_from_file_location("cbf_build", PKG_DIR / "build.py")
        b = importlib.util.module_from_spec(build_spec)
        build_spec.loader.exec_module(b)
        b.build()
    return mod


@pytest.fixture(scope="session")
def orc():
    import oracle as O
    if not O.LIB_PATH.exists():
        O.build(with_ref=False)
    return O


@pytest.fixture(scope="session")
def gpu_ok(cbf):
    try:
        import torch
        if not torch.cuda.is_available():
            pytest.skip("no CUDA device")
    except ImportError:
        pass
    return True
