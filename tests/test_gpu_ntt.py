"""Device NTT and external product against the oracle (bit-exact)."""

import ctypes

import numpy as np
import pytest

from conftest import rng
from gpu_util import empty_dev, from_dev, ptr, to_dev

pytestmark = pytest.mark.gpu

CASES = [(1, 10), (1, 11), (0, 10), (0, 11), (2, 10), (2, 11)]


def rand(oracle, field, shape, seed):
    q = oracle.MODULUS[field]
    return (rng(seed).integers(0, 2**63, shape, dtype=np.uint64) % np.uint64(q)).astype(
        oracle.dtype_of(field))


@pytest.fixture(scope="module")
def ctx(hb):
    c = hb.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("field,log_n", CASES)
def test_ntt_roundtrip(hb, oracle, ctx, field, log_n):
    from hasteboots_b200._lib import check, lib
    n = 1 << log_n
    x = rand(oracle, field, (37, n), 10 + log_n)
    # edge values: zero, Q-1, non-trivial
    x[0] = 0
    x[1] = oracle.MODULUS[field] - 1
    d_in = to_dev(x)
    d_out = empty_dev(x.shape, x.dtype)
    check(lib().hb_ntt_roundtrip_device(ctx.handle, field, log_n, ptr(d_in), ptr(d_out), len(x)),
          "roundtrip", ctx.handle)
    ctx.synchronize()
    assert (from_dev(d_out, x.dtype) == x).all()


def _pointwise(a, b, q):
    return np.array([(int(u) * int(v)) % q for u, v in zip(a, b)], dtype=a.dtype)


@pytest.mark.parametrize("field,log_n", [(1, 10), (0, 10), (1, 11), (2, 10)])
def test_ntt_forward_inverse_product(hb, oracle, ctx, field, log_n):
    from hasteboots_b200._lib import check, lib
    n = 1 << log_n
    q = oracle.MODULUS[field]
    x = rand(oracle, field, (2, n), 20 + log_n)
    d = to_dev(x)
    check(lib().hb_ntt_forward_device(ctx.handle, field, log_n, ptr(d), 2), "fwd", ctx.handle)
    ctx.synchronize()
    f = from_dev(d, x.dtype)
    prod = _pointwise(f[0], f[1], q)
    d2 = to_dev(prod[None, :])
    check(lib().hb_ntt_inverse_device(ctx.handle, field, log_n, ptr(d2), 1), "inv", ctx.handle)
    ctx.synchronize()
    got = from_dev(d2, x.dtype)[0]
    assert (got == oracle.negacyclic_mul(field, log_n, x[0], x[1])).all()


@pytest.mark.parametrize("field,log_n,bits,length", [(1, 10, 5, 13), (1, 11, 5, 13),
                                                     (1, 10, 8, 8), (0, 10, 8, 4), (0, 11, 5, 7),
                                                     (2, 10, 3, 9), (2, 10, 1, 27), (2, 11, 7, 4)])
def test_external_product(hb, oracle, ctx, field, log_n, bits, length):
    from hasteboots_b200._lib import check, lib
    n = 1 << log_n
    count = 9
    rgsw = rand(oracle, field, (2 * length * 2 * n,), 30 + bits)
    rl = rand(oracle, field, (count, 2 * n), 40 + bits)
    expect = oracle.external_product(field, log_n, bits, length, rl, rgsw)
    h = ctypes.c_void_p()
    check(lib().hb_rgsw_upload(ctx.handle, field, log_n, bits, length,
                               rgsw.ctypes.data_as(ctypes.c_void_p), ctypes.byref(h)),
          "rgsw_upload", ctx.handle)
    d_in = to_dev(rl)
    d_out = empty_dev(rl.shape, rl.dtype)
    check(lib().hb_external_product_device(ctx.handle, field, log_n, bits, length, h, ptr(d_in),
                                           ptr(d_out), count), "ext", ctx.handle)
    ctx.synchronize()
    lib().hb_rgsw_free(ctx.handle, h)
    assert (from_dev(d_out, rl.dtype) == expect).all()
