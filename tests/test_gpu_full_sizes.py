"""Parity at the full sizes of the measured workloads, through properties that do not need the
oracle to redo the whole batch: exact NTT round trips on 4096 polynomials, sampled external
products and sampled gates against the oracle, truth tables and noise bounds on every gate."""

import ctypes

import numpy as np
import pytest

from gpu_util import empty_dev, from_dev, ptr, to_dev

pytestmark = pytest.mark.gpu

GOLDILOCKS = 1


@pytest.fixture(scope="module")
def ctx(hb):
    c = hb.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("log_n", [10, 11])
def test_ntt_and_external_product_4096(hb, oracle, ctx, log_n):
    """Kernel microbench sizes: 4096 polynomials, RGSW with l = 13 rows at B = 2^5."""
    from hasteboots_b200._lib import check, lib
    n, count, bits, length = 1 << log_n, 4096, 5, 13
    q = np.uint64(oracle.MODULUS[GOLDILOCKS])
    rg = np.random.default_rng(100 + log_n)
    x = rg.integers(0, 2**63, (count, n), dtype=np.uint64) % q
    d_in, d_out = to_dev(x), empty_dev(x.shape, x.dtype)
    check(lib().hb_ntt_roundtrip_device(ctx.handle, GOLDILOCKS, log_n, ptr(d_in), ptr(d_out), count),
          "roundtrip", ctx.handle)
    ctx.synchronize()
    assert (from_dev(d_out, x.dtype) == x).all()

    rgsw = rg.integers(0, 2**63, (2 * length * 2 * n,), dtype=np.uint64) % q
    rl = rg.integers(0, 2**63, (count, 2 * n), dtype=np.uint64) % q
    h = ctypes.c_void_p()
    check(lib().hb_rgsw_upload(ctx.handle, GOLDILOCKS, log_n, bits, length,
                               rgsw.ctypes.data_as(ctypes.c_void_p), ctypes.byref(h)), "rgsw", ctx.handle)
    d_rl, d_ext = to_dev(rl), empty_dev(rl.shape, rl.dtype)
    check(lib().hb_external_product_device(ctx.handle, GOLDILOCKS, log_n, bits, length, h, ptr(d_rl),
                                           ptr(d_ext), count), "ext", ctx.handle)
    ctx.synchronize()
    lib().hb_rgsw_free(ctx.handle, h)
    got = from_dev(d_ext, rl.dtype)
    sample = np.sort(rg.choice(count, 24, replace=False))
    sample[0], sample[-1] = 0, count - 1
    expect = oracle.external_product(GOLDILOCKS, log_n, bits, length, rl[sample], rgsw)
    assert (got[sample] == expect).all()


def test_16384_goldilocks_nand(hb, oracle, oracle_keys, ctx):
    """The headline batch: every gate decrypts to NAND with noise below Q/16, sampled gates equal
    the oracle bit for bit."""
    from hasteboots_b200._lib import check, lib
    params = hb.Parameters.preset(GOLDILOCKS)
    sk = hb.KeyGen.generate_secret_key(params, 0)
    ev = hb.Evaluator(sk, ctx)
    count = 16384
    bits = np.random.default_rng(3).integers(0, 2, (2, count)).astype(np.uint8)
    c0, c1 = sk.encrypt(bits[0], 0), sk.encrypt(bits[1], 1 << 20)
    d0, d1, dout = to_dev(c0), to_dev(c1), empty_dev(c0.shape, c0.dtype)
    check(lib().hb_gate_device(ctx.handle, ev.keys.handle, 0, ptr(d0), ptr(d1), None, ptr(dout), count),
          "nand", ctx.handle)
    ctx.synchronize()
    out = from_dev(dout, c0.dtype)
    m, noise = sk.decrypt_with_noise(out)
    assert (m == 1 - (bits[0] & bits[1])).all()
    assert (noise < params.modulus // 16).all()
    keys = oracle_keys(GOLDILOCKS, 0)
    for i in (0, 9001, count - 1):
        ref = oracle.gate(keys, "nand", c0[i:i + 1], c1[i:i + 1])
        assert (out[i:i + 1] == ref).all(), i
    ev.keys.free()


def test_64_mixed_jobs(hb, ctx):
    """The mixed-set workload: 64 jobs, log-uniform 1-4096 gates, sets drawn from the three presets,
    in one graph; every gate decrypts to its truth table."""
    evs = {}
    for pid in (0, 1, 2):
        sk = hb.KeyGen.generate_secret_key(hb.Parameters.preset(pid), 0)
        evs[pid] = (sk, hb.Evaluator(sk, ctx))
    rng = np.random.default_rng(4)
    jobs, expect = [], []
    for i in range(64):
        pid = int(rng.integers(0, 3))
        count = int(np.clip(np.round(np.exp(rng.uniform(0, np.log(4096)))), 1, 4096))
        sk, ev = evs[pid]
        bits = rng.integers(0, 2, (2, count)).astype(np.uint8)
        c0, c1 = sk.encrypt(bits[0], (i << 24) + 1), sk.encrypt(bits[1], (i << 24) + (1 << 20))
        out = empty_dev(c0.shape, c0.dtype)
        jobs.append((ev, "nand", to_dev(c0), to_dev(c1), None, out))
        expect.append((pid, 1 - (bits[0] & bits[1])))
    batch = hb.Batch(ctx, jobs)
    batch.launch()
    ctx.synchronize()
    for job, (pid, exp) in zip(jobs, expect):
        sk = evs[pid][0]
        got = from_dev(job[5], sk.params.dtype)
        m, noise = sk.decrypt_with_noise(got)
        assert (m == exp).all()
        assert (noise < sk.params.modulus // 16).all()
    batch.free()
    for sk, ev in evs.values():
        ev.keys.free()
