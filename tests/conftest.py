import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import binding
    binding.lib()  # builds with make when missing
    return binding


@pytest.fixture(scope="session")
def hb():
    from hasteboots_b200 import build
    if not os.path.exists(build.OUT):
        build.build()
    from hasteboots_b200 import tfhe
    return tfhe


_KEYS = {}


@pytest.fixture(scope="session")
def oracle_keys(oracle):
    """Oracle key material per (preset, seed), generated once per session."""
    def get(preset, seed=0):
        k = (preset, seed)
        if k not in _KEYS:
            _KEYS[k] = oracle.keygen(oracle.preset(preset), seed)
        return _KEYS[k]
    return get


def rng(seed):
    return np.random.default_rng(seed)
