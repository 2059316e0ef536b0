"""The allocation-free MUX entry point (hb_gate_mux_device_noalloc) against the allocating one.

It serves callers that cannot call cudaMalloc during a request (a serving process that reserves
its HBM budget at start-up, or a host that owns all device memory through its own pool): its
scratch is a fixed 16 MiB array inside the library. The result must equal hb_gate_device's MUX
bit for bit (the tolerance of every integer test here), on two calls in a row, since every call
reuses the same array. This file is collected last on purpose.
"""

import ctypes

import numpy as np
import pytest

from gpu_util import empty_dev, from_dev, to_dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pid,count", [(0, 37), (1, 7)])
def test_noalloc_mux_matches_allocating_mux(hb, pid, count):
    from hasteboots_b200._lib import HbError, check, lib
    params = hb.Parameters.preset(pid)
    sk = hb.KeyGen.generate_secret_key(params, 0)
    ctx = hb.Context(0)
    ev = hb.Evaluator(sk, ctx)
    try:
        bits = np.random.default_rng(50 + pid).integers(0, 2, (3, count)).astype(np.uint8)
        cs = [sk.encrypt(bits[i], 7000 * (i + 1)) for i in range(3)]
        d = [to_dev(c) for c in cs]
        ref = empty_dev(cs[0].shape, cs[0].dtype)
        check(lib().hb_gate_device(ctx.handle, ev.keys.handle, 8, d[0].data_ptr(), d[1].data_ptr(),
                                   d[2].data_ptr(), ref.data_ptr(), count), "mux", ctx.handle)
        ctx.synchronize()
        ref_h = from_dev(ref, cs[0].dtype)
        expect = np.where(bits[0] == 1, bits[1], bits[2])
        assert (sk.decrypt(ref_h) == expect).all()
        for _ in range(2):  # the second call sees the first call's leftovers in the array
            out = empty_dev(cs[0].shape, cs[0].dtype)
            check(lib().hb_gate_mux_device_noalloc(ctx.handle, ev.keys.handle, d[0].data_ptr(),
                                                   d[1].data_ptr(), d[2].data_ptr(), out.data_ptr(),
                                                   count), "mux_noalloc", ctx.handle)
            assert (from_dev(out, cs[0].dtype) == ref_h).all()
        # sizes beyond the fixed scratch are refused before any device work
        too_many = (16 << 20) // (2 * (params.lwe_dimension() + 1) * cs[0].itemsize) + 1
        rc = lib().hb_gate_mux_device_noalloc(ctx.handle, ev.keys.handle, d[0].data_ptr(),
                                              d[1].data_ptr(), d[2].data_ptr(), ref.data_ptr(),
                                              too_many)
        assert rc == -1
    finally:
        ev.keys.free()
        ctx.close()
