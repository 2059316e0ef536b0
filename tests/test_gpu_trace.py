"""Traces for the proof system.

hb_bootstrap_trace: one bootstrap through the latency form that also returns the accumulator after
every blind-rotation step (the AccTrace of vfhe's bootstrap, vfhe/src/bfhe/evaluate.rs:47-141),
checked against the oracle's golden accumulators after 1, 2, 10 and all n steps of the first NAND row
(c0 + c1 under the NAND LUT) and the output against the golden NAND output, on every binary-key
set: BabyBear (one CTA), Goldilocks and ZAMA (a cluster of four CTAs), DEFAULT_TERNARY (n = N) and
CUSTOM_TERNARY (key switching in two chunks).

hb_bootstrap_trace_device: a batch in one persistent launch, every accumulator row and every
gadget digit of every step checked against the oracle."""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden_seed0.npz")


@pytest.fixture(scope="module")
def ctx(hb):
    c = hb.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("pid", [0, 1, 2, 3, 4])
def test_trace_matches_golden_accumulators(hb, oracle, ctx, pid):
    g = np.load(GOLDEN)
    name = oracle.SET_NAMES[pid]
    params = hb.Parameters.preset(pid)
    sk = hb.KeyGen.generate_secret_key(params, 0)
    ev = hb.Evaluator(sk, ctx)
    try:
        n, q = params.lwe_dimension(), params.modulus
        c0, c1 = g[f"{name}/c0"][0], g[f"{name}/c1"][0]
        s = np.array([(int(a) + int(b)) % q for a, b in zip(c0, c1)], params.dtype)
        lut = oracle.lut_poly(params.field_id, "nand", params.ring_dimension())
        out, trace = ev.bootstrap_with_trace(s, lut)
        assert (out == g[f"{name}/nand"][0]).all()
        for steps in (1, 2, 10, n):
            assert (trace[steps - 1] == g[f"{name}/acc{steps}"]).all(), steps
        # a zero rotation leaves the accumulator as it was
        ms = g[f"{name}/ms0"]
        for i in range(1, n):
            if ms[i] == 0:
                assert (trace[i] == trace[i - 1]).all(), i
        # the same ciphertext through the plain bootstrap entry point
        assert (ev.bootstrap(s, lut)[0] == out).all()
    finally:
        ev.keys.free()


def test_trace_other_steps_vs_oracle(hb, oracle, oracle_keys, ctx):
    """BabyBear: steps 3 and n / 2 against fresh oracle runs on another input."""
    params = hb.Parameters.preset(0)
    sk = hb.KeyGen.generate_secret_key(params, 0)
    ev = hb.Evaluator(sk, ctx)
    try:
        k = oracle_keys(0)
        c = sk.encrypt(np.array([1], np.uint8), 77)[0]
        lut = oracle.lut_poly(params.field_id, "and", params.ring_dimension())
        out, trace = ev.bootstrap_with_trace(c, lut)
        n = params.lwe_dimension()
        for steps in (3, n // 2):
            assert (trace[steps - 1] == oracle.blind_rotate(k, c, lut, steps)).all(), steps
        assert (out == oracle.bootstrap_lut(k, c[None, :], lut)[0]).all()
    finally:
        ev.keys.free()


def test_trace_refuses_ternary_lwe_keys(hb, ctx):
    from hasteboots_b200._lib import HbError
    params = hb.Parameters.preset(4).with_ternary_lwe_key()
    sk = hb.KeyGen.generate_secret_key(params, 0)
    ev = hb.Evaluator(sk, ctx)
    try:
        c = sk.encrypt(np.array([1], np.uint8), 5)[0]
        with pytest.raises(HbError):
            ev.bootstrap_with_trace(c, np.zeros(params.ring_dimension(), params.dtype))
    finally:
        ev.keys.free()


@pytest.mark.parametrize("set_id", [0, 1, 2, 3, 4, 101, 102])
def test_batched_trace_rows_and_digits_vs_oracle(hb, oracle, oracle_keys, ctx, set_id):
    """hb_bootstrap_trace_device: three gates in one persistent launch (two gates per CTA, the
    second CTA half full); every accumulator row and every gadget digit of every step of every gate
    equals the oracle's (orc_blind_rotate_trace), and the outputs equal hb_bootstrap_lut's. All
    binary-key sets: both Goldilocks sets, BabyBear, DefaultFieldU32 with n = N and with two
    key-switching chunks, and GOLDILOCKS n = 500 / BABYBEAR n = 300 (chunked key switching)."""
    from conftest import hb_params_of
    params = hb_params_of(hb, set_id)
    sk = hb.KeyGen.generate_secret_key(params, 0)
    ev = hb.Evaluator(sk, ctx)
    try:
        k = oracle_keys(set_id)
        count = 3
        bits = np.random.default_rng(200 + set_id).integers(0, 2, count).astype(np.uint8)
        c = sk.encrypt(bits, 900)
        lut = oracle.lut_poly(params.field_id, "or" if set_id % 2 else "nand", params.ring_dimension())
        out, acc, dig = ev.bootstrap_with_trace_batch(c, lut)
        n, N, L = params.lwe_dimension(), params.ring_dimension(), params.raw.br_len
        assert acc.shape == (count, n, 2 * N) and dig.shape == (count, n, 2, L, N)
        for g in range(count):
            rows, digits = oracle.blind_rotate_trace(k, c[g], lut, digits=True)
            bad = [i for i in range(n) if not (acc[g, i] == rows[i]).all()]
            assert not bad, (g, bad[:5])
            bad = [i for i in range(n) if not (dig[g, i] == digits[i]).all()]
            assert not bad, (g, bad[:5])
        assert (out == ev.bootstrap(c, lut)).all()
    finally:
        ev.keys.free()


def test_batched_trace_without_digits_and_refusals(hb, ctx):
    """The digit buffer is optional; ternary LWE keys are refused."""
    from hasteboots_b200._lib import HbError
    params = hb.Parameters.preset(0)
    sk = hb.KeyGen.generate_secret_key(params, 0)
    ev = hb.Evaluator(sk, ctx)
    try:
        c = sk.encrypt(np.array([1, 0], np.uint8), 11)
        lut = np.zeros(params.ring_dimension(), params.dtype)
        out, acc, dig = ev.bootstrap_with_trace_batch(c, lut, digits=False)
        assert dig is None and (out == ev.bootstrap(c, lut)).all()
        _, full, _ = ev.bootstrap_with_trace_batch(c, lut)
        assert (acc == full).all()
    finally:
        ev.keys.free()
    tp = hb.Parameters.preset(4).with_ternary_lwe_key()
    tsk = hb.KeyGen.generate_secret_key(tp, 0)
    tev = hb.Evaluator(tsk, ctx)
    try:
        with pytest.raises(HbError):
            tev.bootstrap_with_trace_batch(tsk.encrypt(np.array([1], np.uint8), 5),
                                           np.zeros(tp.ring_dimension(), tp.dtype))
    finally:
        tev.keys.free()
