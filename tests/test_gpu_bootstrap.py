"""Gate bootstrapping on the GPU, bit-exact against the oracle and the golden fixtures."""

import os

import numpy as np
import pytest

from conftest import ALL_SETS, hb_params_of
from gpu_util import empty_dev, from_dev, to_dev

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden_seed0.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="module")
def ctx(hb):
    c = hb.Context(0)
    yield c
    c.close()


_EV = {}


@pytest.fixture(scope="module")
def evaluator(hb, ctx):
    def get(pid):
        if pid not in _EV:
            sk = hb.KeyGen.generate_secret_key(hb_params_of(hb, pid), 0)
            _EV[pid] = (sk, hb.Evaluator(sk, ctx))
        return _EV[pid]
    yield get
    for sk, ev in _EV.values():
        ev.keys.free()
    _EV.clear()


@pytest.mark.parametrize("pid", ALL_SETS)
def test_nand_golden(oracle, golden, evaluator, pid):
    name = oracle.SET_NAMES[pid]
    sk, ev = evaluator(pid)
    out = ev.nand(golden[f"{name}/c0"], golden[f"{name}/c1"])
    assert (out == golden[f"{name}/nand"]).all()
    m, noise = sk.decrypt_with_noise(out)
    assert (m == [1, 1, 1, 0]).all()


@pytest.mark.parametrize("gate", ["and", "or", "nor", "xor", "xnor", "majority", "mux", "not"])
def test_all_gates_babybear_golden(oracle, golden, evaluator, gate):
    name = oracle.PRESET_NAMES[0]
    sk, ev = evaluator(0)
    c0, c1, c2 = golden[f"{name}/c0"], golden[f"{name}/c1"], golden[f"{name}/c2"]
    if gate == "not":
        out = ev.not_(c0)
    elif gate in ("majority", "mux"):
        out = getattr(ev, gate)(c0, c1, c2)
    else:
        out = getattr(ev, gate + "_" if gate in ("and", "or") else gate)(c0, c1)
    assert (out == golden[f"{name}/{gate}"]).all()


def test_bootstrap_custom_lut(oracle, golden, evaluator):
    name = oracle.PRESET_NAMES[0]
    sk, ev = evaluator(0)
    out = ev.bootstrap(golden[f"{name}/c0"], golden[f"{name}/lut"])
    assert (out == golden[f"{name}/bootstrap_lut"]).all()


@pytest.mark.parametrize("pid,count", [(0, 45), (1, 9), (3, 7), (4, 31), (100, 13), (101, 6),
                                       (102, 19)])
def test_random_batch_vs_oracle_and_plain(hb, oracle, oracle_keys, evaluator, ctx, pid, count):
    """Batched launch (partial last CTA) == oracle == one-gate-per-launch form."""
    from hasteboots_b200._lib import check, lib
    sk, ev = evaluator(pid)
    bits = np.random.default_rng(100 + pid).integers(0, 2, (2, count)).astype(np.uint8)
    c0 = sk.encrypt(bits[0], 1000)
    c1 = sk.encrypt(bits[1], 2000)
    out = ev.nand(c0, c1)
    k = oracle_keys(pid)
    assert (out == oracle.gate(k, "nand", c0, c1)).all()
    assert (sk.decrypt(out) == 1 - (bits[0] & bits[1])).all()
    d0, d1 = to_dev(c0), to_dev(c1)
    dout = empty_dev(c0.shape, c0.dtype)
    check(lib().hb_gate_device_plain(ctx.handle, ev.keys.handle, 0, d0.data_ptr(), d1.data_ptr(),
                                     dout.data_ptr(), count), "plain", ctx.handle)
    ctx.synchronize()
    assert (from_dev(dout, c0.dtype) == out).all()


def test_device_tensors_large_batch(hb, evaluator, ctx):
    """A larger BabyBear batch through device tensors decrypts to the NAND truth table."""
    sk, ev = evaluator(0)
    count = 1500
    bits = np.random.default_rng(7).integers(0, 2, (2, count)).astype(np.uint8)
    c0, c1 = sk.encrypt(bits[0], 10_000), sk.encrypt(bits[1], 20_000)
    out = from_dev(ev.nand(to_dev(c0), to_dev(c1)), c0.dtype)
    m, noise = sk.decrypt_with_noise(out)
    assert (m == 1 - (bits[0] & bits[1])).all()
    assert (noise < sk.params.modulus // 16).all()


@pytest.mark.parametrize("pid", [3, 4, 100])
def test_default_field_gates_vs_oracle(hb, oracle, oracle_keys, evaluator, pid):
    """Every gate kind on the DefaultFieldU32 sets: one key-switching chunk (n = N), two chunks
    (n = 512) and the ternary-LWE-key blind rotation, bit-exact against the oracle."""
    sk, ev = evaluator(pid)
    k = oracle_keys(pid)
    bits = np.random.default_rng(300 + pid).integers(0, 2, (3, 6)).astype(np.uint8)
    c = [sk.encrypt(bits[i], 5000 + 100 * i) for i in range(3)]
    for g in ("and", "or", "nor", "xor", "xnor", "majority", "mux", "not"):
        if g == "not":
            out, ref = ev.not_(c[0]), oracle.gate(k, g, c[0])
        elif g in ("majority", "mux"):
            out, ref = getattr(ev, g)(*c), oracle.gate(k, g, *c)
        else:
            out = getattr(ev, g + "_" if g in ("and", "or") else g)(c[0], c[1])
            ref = oracle.gate(k, g, c[0], c[1])
        assert (out == ref).all(), g
