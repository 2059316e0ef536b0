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
    """Oracle key material per (key set, seed), generated once per session."""
    def get(preset, seed=0):
        k = (preset, seed)
        if k not in _KEYS:
            _KEYS[k] = oracle.keygen(oracle.params(preset), seed)
        return _KEYS[k]
    return get


def rng(seed):
    return np.random.default_rng(seed)


# Key sets of the tests (oracle SET_NAMES ids): the five presets and, as 100, CUSTOM_TERNARY_128_BITS
# with a ternary LWE key.
ALL_SETS = [0, 1, 2, 3, 4, 100]


def hb_params_of(hb, set_id):
    """The product's parameters of a key set (101: GOLDILOCKS with n = 500, 102: BABYBEAR with
    n = 300, both switching keys in two chunks of 512 words)."""
    if set_id == 100:
        return hb.Parameters.preset(4).with_ternary_lwe_key()
    if set_id in (101, 102):
        from hasteboots_b200._lib import HbParams
        base = hb.Parameters.preset(1 if set_id == 101 else 0)
        raw = HbParams.from_buffer_copy(base.raw)
        raw.lwe_dim = 500 if set_id == 101 else 300
        return hb.Parameters(raw, base.name + f"+n={raw.lwe_dim}")
    return hb.Parameters.preset(set_id)
