import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "plenoptic-for-depth_b200")
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def load_pfd():
    """Import the engine package (its directory name is not an identifier)."""
    name = "pfd_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def pfd():
    mod = load_pfd()
    build = importlib.util.spec_from_file_location("pfd_build", os.path.join(PKG_DIR, "build.py"))
    b = importlib.util.module_from_spec(build)
    build.loader.exec_module(b)
    if not all(os.path.exists(p) for p in (mod.LIB_PATH, mod.SYNTH_PATH, b.HOST_LIB, b.SHIM_PROBE, b.TEX_PROBE)):
        b.build_all()
    return mod


@pytest.fixture(scope="session")
def oracle():
    import pfd_oracle
    pfd_oracle.build()
    return pfd_oracle
