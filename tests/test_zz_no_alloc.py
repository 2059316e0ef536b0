"""The allocation-free MUX entry point (hb_gate_mux_device_noalloc) against the allocating one.

It serves callers that cannot call cudaMalloc during a request (a serving process that reserves
its HBM budget at start-up, or a host that owns all device memory through its own pool): its
scratch is a fixed 16 MiB array inside the library. The result must equal hb_gate_device's MUX
bit for bit (the tolerance of every integer test here), on two calls in a row, since every call
reuses the same array. This file is collected last on purpose.
"""

import numpy as np
import pytest

from conftest import hb_params_of
from gpu_util import empty_dev, from_dev, to_dev

pytestmark = pytest.mark.gpu

SCRATCH = 16 << 20
HEADER = 1024  # status word and job table ahead of the intermediate ciphertexts
HB_ERR_INVALID, HB_ERR_TIMEOUT = -1, -4


def max_gates(params, word_bytes):
    return (SCRATCH - HEADER) // (2 * (params.lwe_dimension() + 1) * word_bytes)


def _setup(hb, set_id, count, seed):
    params = hb_params_of(hb, set_id)
    sk = hb.KeyGen.generate_secret_key(params, 0)
    ctx = hb.Context(0)
    ev = hb.Evaluator(sk, ctx)
    bits = np.random.default_rng(seed).integers(0, 2, (3, count)).astype(np.uint8)
    cs = [sk.encrypt(bits[i], 7000 * (i + 1)) for i in range(3)]
    return params, sk, ctx, ev, bits, cs


def _reference(ctx, ev, d, count, like):
    from hasteboots_b200._lib import check, lib
    ref = empty_dev(like.shape, like.dtype)
    check(lib().hb_gate_device(ctx.handle, ev.keys.handle, 8, d[0].data_ptr(), d[1].data_ptr(),
                               d[2].data_ptr(), ref.data_ptr(), count), "mux", ctx.handle)
    ctx.synchronize()
    return from_dev(ref, like.dtype)


def _noalloc(ctx, ev, d, out, count):
    from hasteboots_b200._lib import lib
    return lib().hb_gate_mux_device_noalloc(ctx.handle, ev.keys.handle, d[0].data_ptr(), d[1].data_ptr(),
                                            d[2].data_ptr(), out.data_ptr(), count)


@pytest.mark.parametrize("set_id,count", [(0, 37), (1, 7), (2, 5), (3, 9), (4, 21), (100, 11)])
def test_noalloc_mux_matches_allocating_mux(hb, set_id, count):
    from hasteboots_b200._lib import check
    params, sk, ctx, ev, bits, cs = _setup(hb, set_id, count, 50 + set_id)
    try:
        d = [to_dev(c) for c in cs]
        ref_h = _reference(ctx, ev, d, count, cs[0])
        assert (sk.decrypt(ref_h) == np.where(bits[0] == 1, bits[1], bits[2])).all()
        for _ in range(2):  # the second call sees the first call's leftovers in the array
            out = empty_dev(cs[0].shape, cs[0].dtype)
            check(_noalloc(ctx, ev, d, out, count), "mux_noalloc", ctx.handle)
            assert (from_dev(out, cs[0].dtype) == ref_h).all()
    finally:
        ev.keys.free()
        ctx.close()


@pytest.mark.parametrize("pid", [0, 1])
def test_noalloc_mux_size_limit(hb, pid):
    """Exactly the largest count fits and matches; one more gate is refused before any device work."""
    from hasteboots_b200._lib import check
    params = hb.Parameters.preset(pid)
    word = np.dtype(params.dtype).itemsize
    top = max_gates(params, word)
    params, sk, ctx, ev, bits, cs = _setup(hb, pid, top, 60 + pid)
    try:
        d = [to_dev(c) for c in cs]
        ref_h = _reference(ctx, ev, d, top, cs[0])
        out = empty_dev(cs[0].shape, cs[0].dtype)
        check(_noalloc(ctx, ev, d, out, top), "mux_noalloc", ctx.handle)
        assert (from_dev(out, cs[0].dtype) == ref_h).all()
        assert _noalloc(ctx, ev, d, out, top + 1) == HB_ERR_INVALID
    finally:
        ev.keys.free()
        ctx.close()


def test_noalloc_mux_timeout_then_recovers(hb):
    """A withheld key stream makes the call return HB_ERR_TIMEOUT (a wait that nothing ends,
    bounded), and the next call on the same context matches the allocating MUX again."""
    from hasteboots_b200._lib import check, lib
    params, sk, ctx, ev, bits, cs = _setup(hb, 0, 13, 77)
    try:
        d = [to_dev(c) for c in cs]
        ref_h = _reference(ctx, ev, d, 13, cs[0])
        out = empty_dev(cs[0].shape, cs[0].dtype)
        assert lib().hb_ctx_set_wait_limit(ctx.handle, 200000) == 0  # ~0.1 ms of SM clocks
        assert lib().hb_ctx_test_withhold_keys(ctx.handle, 1) == 0
        try:
            assert _noalloc(ctx, ev, d, out, 13) == HB_ERR_TIMEOUT
        finally:
            lib().hb_ctx_test_withhold_keys(ctx.handle, 0)
            lib().hb_ctx_set_wait_limit(ctx.handle, 0)
        out2 = empty_dev(cs[0].shape, cs[0].dtype)
        check(_noalloc(ctx, ev, d, out2, 13), "mux_noalloc", ctx.handle)
        assert (from_dev(out2, cs[0].dtype) == ref_h).all()
    finally:
        ev.keys.free()
        ctx.close()
