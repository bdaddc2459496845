import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "wavetoysecondorder.jl_b200")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs through libwavetoy_b200.so")
    config.addinivalue_line("markers", "slow: longer CPU test")


def load_package():
    """Import wavetoysecondorder.jl_b200/ as module 'wavetoy_b200'."""
    name = "wavetoy_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def wt():
    return load_package()


@pytest.fixture(scope="session")
def O():
    from oracle import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def ctx(wt):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return wt.Context(0)


@pytest.fixture(autouse=True)
def _bounds_words_clear(request):
    """With the bounds-check library loaded (WAVETOY_B200_LIB=.../libwavetoy_b200_bc.so), every GPU
    test must leave the bounds words clear: no kernel read a table index out of range."""
    checked = None
    if "gpu" in request.keywords and os.environ.get("WAVETOY_B200_LIB"):
        wt = load_package()
        if wt.build_flags() & wt.BUILD_BOUNDS_CHECK:
            checked = request.getfixturevalue("ctx")
    yield
    if checked is not None:
        assert checked.bounds_status() == 0, "a kernel read a table index out of range"
