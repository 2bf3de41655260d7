import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

PKG_DIR = os.path.join(ROOT, "rustmpeg-next_b200")


def load_pkg():
    """Import the package directory rustmpeg-next_b200/ as `rustmpeg_next_b200`."""
    if "rustmpeg_next_b200" in sys.modules:
        return sys.modules["rustmpeg_next_b200"]
    spec = importlib.util.spec_from_file_location(
        "rustmpeg_next_b200", os.path.join(PKG_DIR, "__init__.py"),
        submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["rustmpeg_next_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def orc():
    import oracle

    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def pkg():
    return load_pkg()


@pytest.fixture(scope="session")
def ctx(pkg):
    """A libvvcg context on cuda:0; GPU tests fail loudly without the native library."""
    import torch

    assert torch.cuda.is_available(), "GPU test run without a CUDA device"
    pkg.build()
    c = pkg.Context(0)
    yield c
    c.close()
