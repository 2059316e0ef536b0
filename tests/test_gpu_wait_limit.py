"""Failure detection on the GPU without a fault: every wait of the bootstrapping kernel for a key
chunk is bounded. With the key copies withheld (a flag that nothing sets) and a short wait limit,
the call must return HB_ERR_TIMEOUT within the limit, and the same context must then bootstrap
correctly again."""

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_withheld_keys_time_out_and_context_recovers(hb):
    from hasteboots_b200._lib import HbError, lib
    ctx = hb.Context(0)
    sk = hb.KeyGen.generate_secret_key(hb.Parameters.preset(0), 0)
    ev = hb.Evaluator(sk, ctx)
    bits = np.random.default_rng(31).integers(0, 2, (2, 300)).astype(np.uint8)
    c0, c1 = sk.encrypt(bits[0], 5 << 20), sk.encrypt(bits[1], 6 << 20)
    ref = ev.nand(c0, c1)
    try:
        assert lib().hb_ctx_set_wait_limit(ctx.handle, 200000) == 0  # ~0.1 ms of SM clocks
        assert lib().hb_ctx_test_withhold_keys(ctx.handle, 1) == 0
        t0 = time.perf_counter()
        with pytest.raises(HbError) as err:
            ev.nand(c0, c1)
        assert err.value.code == -4  # HB_ERR_TIMEOUT
        assert time.perf_counter() - t0 < 30
    finally:
        lib().hb_ctx_test_withhold_keys(ctx.handle, 0)
        lib().hb_ctx_set_wait_limit(ctx.handle, 0)
    out = ev.nand(c0, c1)
    assert (out == ref).all()
    assert (sk.decrypt(out) == 1 - (bits[0] & bits[1])).all()
    ev.keys.free()
    ctx.close()
