"""hb_bootstrap_trace: one bootstrap through the latency form that also returns the accumulator after
every blind-rotation step (the AccTrace of vfhe's bootstrap, vfhe/src/bfhe/evaluate.rs:47-141).
The trace is checked against the oracle's golden accumulators after 1, 2, 10 and all n steps of the
first NAND row (c0 + c1 under the NAND LUT) and the output against the golden NAND output, on every
binary-key set: BabyBear (one CTA), Goldilocks and ZAMA (a cluster of four CTAs), DEFAULT_TERNARY
(n = N) and CUSTOM_TERNARY (key switching in two chunks)."""

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
