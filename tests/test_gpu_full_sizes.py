"""Parity at the full sizes of the measured workloads: exact NTT round trips on 4096 polynomials,
sampled external products against the oracle, and every output ciphertext of the 16384-gate
headline batch and of the 64-job mixed-set batch against the oracle's, through the SHA-256 digests
that tests/golden/gen_digests.py recorded by running the oracle on the same inputs."""

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




def _digests():
    import json
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "digests_full.json")
    return json.load(open(path))


def test_16384_goldilocks_nand_every_output(hb, ctx):
    """The headline batch: every one of the 16384 output ciphertexts equals the oracle's, through the
    SHA-256 of each 1024-gate slice (tests/golden/gen_digests.py ran the oracle on the same inputs,
    whose digests are checked first); every gate decrypts to NAND with noise below Q/16."""
    from hasteboots_b200 import workloads as W
    from hasteboots_b200._lib import check, lib
    ref = _digests()["headline"]
    params = hb.Parameters.preset(W.HEADLINE_PRESET)
    sk = hb.KeyGen.generate_secret_key(params, 0)
    ev = hb.Evaluator(sk, ctx)
    count = W.HEADLINE_GATES
    bits = W.headline_bits(count)
    c0, c1 = sk.encrypt(bits[0], W.HEADLINE_INDEX0[0]), sk.encrypt(bits[1], W.HEADLINE_INDEX0[1])
    assert W.digest(c0) == ref["c0"] and W.digest(c1) == ref["c1"]
    d0, d1, dout = to_dev(c0), to_dev(c1), empty_dev(c0.shape, c0.dtype)
    check(lib().hb_gate_device(ctx.handle, ev.keys.handle, 0, ptr(d0), ptr(d1), None, ptr(dout), count),
          "nand", ctx.handle)
    ctx.synchronize()
    out = from_dev(dout, c0.dtype)
    m, noise = sk.decrypt_with_noise(out)
    assert (m == W.truth("nand", bits[0], bits[1])).all()
    assert (noise < params.modulus // 16).all()
    got = W.slice_digests(out, ref["slice"])
    bad = [i for i, (a, b) in enumerate(zip(got, ref["out_slices"])) if a != b]
    assert len(ref["out_slices"]) == count // ref["slice"] and not bad, f"slices differing: {bad}"
    ev.keys.free()


def test_64_mixed_jobs_every_output(hb, ctx):
    """The mixed-set workload: 64 jobs of seven gate kinds, log-uniform 1-4096 gates, sets drawn from
    the three presets, in one graph; every job's outputs equal the oracle's (SHA-256 per job, inputs
    checked first) and decrypt to the job's truth table."""
    from hasteboots_b200 import workloads as W
    ref = _digests()["mixed"]
    evs = {}
    for pid in (0, 1, 2):
        sk = hb.KeyGen.generate_secret_key(hb.Parameters.preset(pid), 0)
        evs[pid] = (sk, hb.Evaluator(sk, ctx))
    jobs, plan = [], W.mixed_plan()
    assert len(ref) == len(plan)
    for job in plan:
        sk, ev = evs[job.preset]
        cs = [sk.encrypt(job.bits[k], job.index0(k)) for k in range(job.inputs)]
        r = ref[str(job.index)]
        assert (r["preset"], r["gate"], r["count"]) == (job.preset, job.gate, job.count)
        assert [W.digest(c) for c in cs] == r["inputs"], job.index
        d = [to_dev(c) for c in cs]
        out = empty_dev(cs[0].shape, cs[0].dtype)
        jobs.append((ev, job.gate, d[0], d[1], d[2] if job.inputs == 3 else None, out))
    batch = hb.Batch(ctx, jobs)
    batch.launch()
    ctx.synchronize()
    bad = []
    for job, j in zip(plan, jobs):
        sk = evs[job.preset][0]
        got = from_dev(j[5], sk.params.dtype)
        m, noise = sk.decrypt_with_noise(got)
        assert (m == job.expected()).all(), job.index
        assert (noise < sk.params.modulus // 16).all(), job.index
        if W.digest(got) != ref[str(job.index)]["out"]:
            bad.append(job.index)
    assert not bad, f"jobs differing from the oracle: {bad}"
    batch.free()
    for sk, ev in evs.values():
        ev.keys.free()
