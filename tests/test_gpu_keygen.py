"""Key generation and LWE encryption on the device against the host generator (which equals the
oracle's, tests/test_client.py): the device key words must equal hb_keygen + hb_keys_upload's."""

import ctypes

import numpy as np
import pytest

from conftest import ALL_SETS, hb_params_of
from gpu_util import empty_dev, from_dev, ptr, to_dev

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(hb):
    c = hb.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("pid", ALL_SETS + [101, 102])
def test_device_keygen_equals_host_keygen_and_upload(hb, ctx, pid):
    params = hb_params_of(hb, pid)
    sk = hb.KeyGen.generate_secret_key(params, 5)
    bsk, ksk = sk.evaluation_key_material()
    up = hb.DeviceKeys(ctx, params, bsk, ksk)
    gen, lwe, ring = hb.DeviceKeys.generate(ctx, params, 5)
    try:
        assert (lwe == sk.lwe_secret_key).all() and (ring == sk.ring_secret_key).all()
        b_up, k_up = up.download()
        b_gen, k_gen = gen.download()
        assert (b_gen == b_up).all()
        assert (k_gen == k_up).all()
    finally:
        up.free()
        gen.free()


@pytest.mark.parametrize("pid", [0, 1, 4])
def test_device_keygen_cbd_noise_equals_host(hb, ctx, pid):
    """sigma exactly 3.2: the device generator's centered binomial noise equals the host's."""
    from hasteboots_b200._lib import HbParams
    base = hb.Parameters.preset(pid)
    raw = HbParams.from_buffer_copy(base.raw)
    raw.ring_noise_std = 3.2
    raw.ks_noise_std = 3.2
    params = hb.Parameters(raw, base.name + "+cbd")
    sk = hb.KeyGen.generate_secret_key(params, 3)
    bsk, ksk = sk.evaluation_key_material()
    up = hb.DeviceKeys(ctx, params, bsk, ksk)
    gen, _, _ = hb.DeviceKeys.generate(ctx, params, 3)
    try:
        b_up, k_up = up.download()
        b_gen, k_gen = gen.download()
        assert (b_gen == b_up).all() and (k_gen == k_up).all()
    finally:
        up.free()
        gen.free()


@pytest.mark.parametrize("pid", [0, 1, 3, 100])
def test_device_encrypt_equals_host(hb, ctx, pid):
    from hasteboots_b200._lib import check, lib
    params = hb_params_of(hb, pid)
    sk = hb.SecretKeyPack(params, 1)
    count = 300
    bits = np.random.default_rng(pid).integers(0, 2, count).astype(np.uint8)
    host = sk.encrypt(bits, index0=77)
    import torch
    d_bits = torch.from_numpy(bits.copy()).cuda()
    d_sk = to_dev(sk.lwe_secret_key)
    d_out = empty_dev(host.shape, host.dtype)
    check(lib().hb_encrypt_device(ctx.handle, ctypes.byref(params.raw), ptr(d_sk), 1, 77,
                                  ptr(d_bits), count, ptr(d_out)), "encrypt_device", ctx.handle)
    ctx.synchronize()
    assert (from_dev(d_out, host.dtype) == host).all()


def test_evaluator_on_device_keys_matches_golden(hb, oracle, ctx):
    import os
    golden = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_seed0.npz"))
    name = oracle.SET_NAMES[1]
    sk = hb.KeyGen.generate_secret_key(hb.Parameters.preset(1), 0)
    ev = hb.Evaluator(sk, ctx, device_keygen=True)
    try:
        out = ev.nand(golden[f"{name}/c0"], golden[f"{name}/c1"])
        assert (out == golden[f"{name}/nand"]).all()
    finally:
        ev.keys.free()
