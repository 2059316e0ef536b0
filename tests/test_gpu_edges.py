"""Edge cases of the gate entry points: empty inputs, a batch that does not fit the context's HBM
budget (refused with HB_ERR_NOMEM, context still usable), and invalid arguments."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bb(hb):
    ctx = hb.Context(0)
    sk = hb.KeyGen.generate_secret_key(hb.Parameters.preset(0), 0)
    ev = hb.Evaluator(sk, ctx)
    yield ctx, sk, ev
    ev.keys.free()
    ctx.close()


def test_empty_inputs_launch_nothing(hb, bb):
    from hasteboots_b200._lib import lib
    ctx, sk, ev = bb
    w = sk.params.lwe_dimension() + 1
    empty = np.zeros((0, w), sk.params.dtype)
    before = lib().hb_ctx_launches(ctx.handle)
    for name in ("nand", "xor", "majority", "mux"):
        args = (empty, empty, empty) if name in ("majority", "mux") else (empty, empty)
        out = getattr(ev, name)(*args)
        assert out.shape == (0, w)
    assert ev.bootstrap(empty, np.zeros(sk.params.raw.ring_dim, sk.params.dtype)).shape == (0, w)
    assert lib().hb_ctx_launches(ctx.handle) == before


def test_batch_beyond_budget_is_refused_and_context_recovers(hb, bb):
    from hasteboots_b200._lib import HbError
    _, sk, _ = bb
    small = hb.Context(0, hbm_budget=256 << 20)  # the BabyBear keys (48 MB) fit, 30k gates do not
    ev = hb.Evaluator(sk, small)
    bits = np.random.default_rng(41).integers(0, 2, (2, 30000)).astype(np.uint8)
    c0, c1 = sk.encrypt(bits[0], 9 << 20), sk.encrypt(bits[1], 10 << 20)
    with pytest.raises(HbError) as err:
        ev.nand(c0, c1)
    assert err.value.code == -3  # HB_ERR_NOMEM
    out = ev.nand(c0[:64], c1[:64])
    assert (sk.decrypt(out) == 1 - (bits[0, :64] & bits[1, :64])).all()
    ev.keys.free()
    small.close()


def test_invalid_arguments_are_rejected(hb, bb):
    from hasteboots_b200._lib import lib
    ctx, sk, ev = bb
    c = sk.encrypt(np.array([1], np.uint8), 0)
    out = np.zeros_like(c)
    # gate id out of range, null input
    assert lib().hb_gate(ctx.handle, ev.keys.handle, 99, c.ctypes.data, c.ctypes.data, None,
                         out.ctypes.data, 1) == -1
    assert lib().hb_gate(ctx.handle, ev.keys.handle, 0, None, c.ctypes.data, None, out.ctypes.data, 1) == -1
