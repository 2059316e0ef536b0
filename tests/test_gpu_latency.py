"""Launches of at most one gate per SM take the latency form (bootstrap_dp_kernel: one gate per
CTA, or a cluster of CTAs with a binary LWE key, the gadget digits spread over the thread groups).
Bit-exact against the oracle for every field and both key layouts (T = 64 and 128 threads per
group), including ZAMA's 26 digits over 4 groups, launches at the cluster limit and one gate past
it, a launch of exactly one gate per SM, and ternary LWE keys."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(hb):
    c = hb.Context(0)
    yield c
    c.close()


def variants_for(field_id, T):
    # a compiled gates-per-CTA variant of each (field, T) key layout
    return {(1, 64): 4, (1, 128): 4, (0, 64): 6, (0, 128): 6, (2, 64): 6, (2, 128): 6}[(field_id, T)]


@pytest.mark.parametrize("pid", [0, 1, 2, 3])
@pytest.mark.parametrize("T", [64, 128])
def test_latency_form_vs_oracle(hb, oracle, oracle_keys, ctx, pid, T):
    from hasteboots_b200._lib import check, lib
    params = hb.Parameters.preset(pid)
    sk = hb.KeyGen.generate_secret_key(params, 0)
    ev = hb.Evaluator(sk, ctx)
    try:
        check(lib().hb_keys_set_config(ctx.handle, ev.keys.handle, T, variants_for(params.field_id, T)),
              "set_config", ctx.handle)
        k = oracle_keys(pid)
        bits = np.random.default_rng(40 + pid).integers(0, 2, (3, 5)).astype(np.uint8)
        c = [sk.encrypt(bits[i], 900 + 10 * i) for i in range(3)]
        for g in ("nand", "xor", "majority"):
            if g == "majority":
                out, ref = ev.majority(*c), oracle.gate(k, g, *c)
            else:
                out, ref = getattr(ev, g)(c[0], c[1]), oracle.gate(k, g, c[0], c[1])
            assert (out == ref).all(), g
    finally:
        ev.keys.free()


def test_latency_form_one_gate_per_sm(hb, oracle, oracle_keys, ctx):
    """148 BabyBear gates: one CTA per SM, every output decrypts, sampled outputs match the oracle."""
    sk = hb.KeyGen.generate_secret_key(hb.Parameters.preset(0), 0)
    ev = hb.Evaluator(sk, ctx)
    try:
        count = 148
        bits = np.random.default_rng(11).integers(0, 2, (2, count)).astype(np.uint8)
        c0, c1 = sk.encrypt(bits[0], 3000), sk.encrypt(bits[1], 4000)
        out = ev.nand(c0, c1)
        assert (sk.decrypt(out) == 1 - (bits[0] & bits[1])).all()
        k = oracle_keys(0)
        pick = [0, 77, 147]
        assert (out[pick] == oracle.gate(k, "nand", c0[pick], c1[pick])).all()
    finally:
        ev.keys.free()


@pytest.mark.parametrize("pid,count", [(1, 3), (1, 37), (1, 100), (0, 1), (0, 74), (0, 75), (4, 5), (3, 2)])
def test_latency_form_cluster_and_single_sm(hb, oracle, oracle_keys, ctx, pid, count):
    """Launches small enough for a cluster of CTAs per gate (Goldilocks: 4 CTAs, up to 37 gates on
    148 SMs; 32-bit fields: 2 CTAs, up to 74 gates, CUSTOM_TERNARY with its two key-switching
    chunks) and just beyond (one SM per gate) against the oracle."""
    sk = hb.KeyGen.generate_secret_key(hb.Parameters.preset(pid), 0)
    ev = hb.Evaluator(sk, ctx)
    try:
        bits = np.random.default_rng(70 + count).integers(0, 2, (2, count)).astype(np.uint8)
        c0, c1 = sk.encrypt(bits[0], 7000), sk.encrypt(bits[1], 8000)
        out = ev.nand(c0, c1)
        assert (sk.decrypt(out) == 1 - (bits[0] & bits[1])).all()
        k = oracle_keys(pid)
        pick = sorted({0, count // 2, count - 1})
        assert (out[pick] == oracle.gate(k, "nand", c0[pick], c1[pick])).all()
    finally:
        ev.keys.free()


@pytest.mark.parametrize("base", [3, 4])
@pytest.mark.parametrize("T", [64, 128])
def test_latency_form_ternary_lwe_key(hb, oracle, ctx, base, T):
    """Ternary LWE keys in the latency form (one CTA per gate; the CTA's two halves of groups take
    RGSW(s_i = 1) and RGSW(s_i = -1)) against the oracle's ternary blind rotation, over
    DefaultFieldU32 with n = N (DEFAULT_TERNARY) and with two key-switching chunks
    (CUSTOM_TERNARY), both key layouts; the plain one-group form gives the same words."""
    from hasteboots_b200._lib import check, lib
    from gpu_util import empty_dev, from_dev, to_dev
    params = hb.Parameters.preset(base).with_ternary_lwe_key()
    sk = hb.KeyGen.generate_secret_key(params, 0)
    ev = hb.Evaluator(sk, ctx)
    try:
        check(lib().hb_keys_set_config(ctx.handle, ev.keys.handle, T, 4), "set_config", ctx.handle)
        op = oracle.preset(base)
        op.lwe_ternary = 1
        k = oracle.keygen(op, 0)
        bits = np.random.default_rng(90 + base).integers(0, 2, (3, 6)).astype(np.uint8)
        c = [sk.encrypt(bits[i], 600 + 10 * i) for i in range(3)]
        for g in ("nand", "xnor", "majority"):
            if g == "majority":
                out, ref = ev.majority(*c), oracle.gate(k, g, *c)
            else:
                out, ref = getattr(ev, g)(c[0], c[1]), oracle.gate(k, g, c[0], c[1])
            assert (out == ref).all(), g
        d0, d1 = to_dev(c[0]), to_dev(c[1])
        dp = empty_dev(c[0].shape, c[0].dtype)
        check(lib().hb_gate_device_plain(ctx.handle, ev.keys.handle, 0, d0.data_ptr(), d1.data_ptr(),
                                         dp.data_ptr(), len(c[0])), "plain", ctx.handle)
        ctx.synchronize()
        assert (from_dev(dp, c[0].dtype) == ev.nand(c[0], c[1])).all()
    finally:
        ev.keys.free()
