"""Host-side client code of the product (keygen / encrypt / decrypt) against the oracle."""

import hashlib
import os

import numpy as np
import pytest

from conftest import ALL_SETS, hb_params_of

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden_seed0.npz")


@pytest.mark.parametrize("pid", ALL_SETS)
def test_product_keygen_matches_oracle(hb, oracle, oracle_keys, pid):
    p = hb_params_of(hb, pid)
    sk = hb.KeyGen.generate_secret_key(p, 0)
    bsk, ksk = sk.evaluation_key_material()
    k = oracle_keys(pid)
    assert (sk.lwe_secret_key == k.lwe_sk).all()
    assert (sk.ring_secret_key == k.ring_sk).all()
    assert (bsk == k.bsk).all()
    assert (ksk == k.ksk).all()
    g = np.load(GOLDEN)
    name = oracle.SET_NAMES[pid]
    assert hashlib.sha256(bsk.tobytes()).hexdigest() == str(g[f"{name}/sha_bsk"])


@pytest.mark.parametrize("pid", [101, 102])
def test_chunked_key_switching_key_matches_oracle(hb, oracle_keys, pid):
    sk = hb.KeyGen.generate_secret_key(hb_params_of(hb, pid), 0)
    bsk, ksk = sk.evaluation_key_material()
    k = oracle_keys(pid)
    assert (bsk == k.bsk).all() and (ksk == k.ksk).all()


@pytest.mark.parametrize("pid", [0, 1, 4])
def test_cbd_keygen_matches_oracle(hb, oracle, pid):
    """sigma exactly 3.2 selects the centered binomial sampler for the RGSW and key-switching error
    polynomials (algebra/src/random.rs:91-92); the product's generator and the oracle's agree on
    every field, including the release-build wrap of its a < b branch."""
    from hasteboots_b200._lib import HbParams
    base = hb.Parameters.preset(pid)
    raw = HbParams.from_buffer_copy(base.raw)
    raw.ring_noise_std = 3.2
    raw.ks_noise_std = 3.2
    p = hb.Parameters(raw, base.name + "+cbd")
    bsk, ksk = hb.KeyGen.generate_secret_key(p, 3).evaluation_key_material()
    op = oracle.preset(pid)
    op.ring_noise_std = 3.2
    op.ks_noise_std = 3.2
    k = oracle.keygen(op, 3)
    assert (bsk == k.bsk).all() and (ksk == k.ksk).all()


@pytest.mark.parametrize("pid", ALL_SETS)
def test_encrypt_decrypt_matches_oracle(hb, oracle, oracle_keys, pid):
    p = hb_params_of(hb, pid)
    sk = hb.SecretKeyPack(p, 0)
    bits = np.random.default_rng(pid).integers(0, 2, 64).astype(np.uint8)
    c = sk.encrypt(bits, index0=100)
    k = oracle_keys(pid)
    assert (c == oracle.encrypt(k.p, k.lwe_sk, 0, 100, bits)).all()
    m, noise = sk.decrypt_with_noise(c)
    mo, noiseo = oracle.decrypt(k.p, k.lwe_sk, c)
    assert (m == bits).all() and (mo == bits).all() and (noise == noiseo).all()
    g = np.load(GOLDEN)
    name = oracle.SET_NAMES[pid]
    assert (sk.encrypt([0, 0, 1, 1], 0) == g[f"{name}/c0"]).all()


def test_parameter_validation(hb):
    from hasteboots_b200._lib import HbError, HbParams, lib
    import ctypes
    raw = HbParams()
    assert lib().hb_params_preset(1, ctypes.byref(raw)) == 0
    assert lib().hb_params_validate(ctypes.byref(raw)) == 0
    # n only needs next_pow2(n) <= N (n = 300 switches keys in two chunks of 512 words)
    bad = [("ring_dim", 1000), ("lwe_dim", 2000), ("lwe_dim", 0), ("br_len", 7), ("br_bits", 0),
           ("field_id", 5), ("ring_dim", 8192), ("lwe_ternary", 1), ("lwe_ternary", 2)]
    for field, value in bad:
        r = HbParams()
        lib().hb_params_preset(1, ctypes.byref(r))
        setattr(r, field, value)
        assert lib().hb_params_validate(ctypes.byref(r)) == -1, field
    r = HbParams()
    lib().hb_params_preset(1, ctypes.byref(r))
    r.lwe_dim = 300
    assert lib().hb_params_validate(ctypes.byref(r)) == 0
    # ternary LWE keys: DefaultFieldU32 only (ternary.rs:80 marks the other fields incompatible)
    r = HbParams()
    lib().hb_params_preset(4, ctypes.byref(r))
    r.lwe_ternary = 1
    assert lib().hb_params_validate(ctypes.byref(r)) == 0
    with pytest.raises(HbError):
        hb.Parameters(bad_params())
    with pytest.raises(HbError):
        hb.Parameters.preset(0).with_ternary_lwe_key()
    assert lib().hb_params_preset(9, ctypes.byref(raw)) == -1


def bad_params():
    from hasteboots_b200._lib import HbParams
    return HbParams()


def test_empty_batches(hb):
    # zero ciphertexts in, zero out (host encryption and decryption)
    sk = hb.KeyGen.generate_secret_key(hb.Parameters.preset(0), 0)
    c = sk.encrypt(np.zeros(0, np.uint8))
    assert c.shape == (0, sk.params.raw.lwe_dim + 1)
    bits, noise = sk.decrypt_with_noise(c)
    assert bits.shape == (0,) and noise.shape == (0,)
