import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "halo2-gpu_b200")
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_package():
    name = "halo2_gpu_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def h2b():
    return load_package()


@pytest.fixture(scope="session")
def orc():
    import oracle as o
    o.lib()
    return o


@pytest.fixture(scope="session")
def built_lib(h2b):
    if not os.path.exists(h2b.LIB_PATH):
        spec = importlib.util.spec_from_file_location("h2b_build", os.path.join(PKG_DIR, "build.py"))
        m = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(m)
        m.build()
    return h2b.lib()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def rand_fr(orc, n, seed):
    return orc.chacha_fr(seed, n)


def assert_limbs_equal(a, b, what=""):
    a = np.asarray(a, dtype=np.uint64)
    b = np.asarray(b, dtype=np.uint64)
    assert a.shape == b.shape, f"{what}: shape {a.shape} != {b.shape}"
    if not np.array_equal(a, b):
        bad = np.nonzero(np.any(a.reshape(a.shape[0], -1) != b.reshape(b.shape[0], -1), axis=1))[0] \
            if a.ndim > 1 else np.nonzero(a != b)[0]
        raise AssertionError(f"{what}: {len(bad)} mismatching rows, first {bad[:8].tolist()}")
