"""The first blind-rotation steps restated without any NTT, checked against the oracle's golden
accumulators (tests/golden/gen_golden.py) on every key set.

The oracle transforms keys and digits with its own negacyclic NTT; the NTT-domain words are not
pinned by the reference (concrete-ntt's slot order is unspecified), but the coefficient-domain
accumulator is: the negacyclic product mod Q is unique. This file recomputes, in numpy with exact
integer schoolbook convolutions, the modulus switch (fhe_core/src/modulus_switch.rs:12-38), the
accumulator LUT * X^-b (fhe_core/src/blind_rotation/rlwe/binary.rs:40-64), E = (X^a - 1) * ACC
(lattice/src/rlwe.rs:437-487), the unsigned LSB-first gadget digits of canonical values
(algebra/src/polynomial/univariate/native_polynomial.rs:340-348), the RLWE x RGSW product
(lattice/src/rlwe.rs:573-596) and ACC += E (:287-290); for a ternary LWE key the evaluation key
RGSW(s = 1) + RGSW(s = -1) * (-X^-a) (fhe_core/src/blind_rotation/rlwe/ternary.rs:78-89).

The arithmetic here is plain arithmetic mod Q. The reference's Goldilocks words may sit in
[Q, 2^64), where its negation is not the true one (algebra/src/modulus/goldilocks/ops.rs:69-73) and
the oracle follows it; the two part only where such a word occurs, which these inputs never produce.
"""

import os

import numpy as np
import pytest

from conftest import ALL_SETS

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden_seed0.npz")


def modswitch(v, q, two_n):
    """round(f64(v) * 2N / f64(Q)) with f64::round (half away from zero), 2N mapped to 0."""
    x = v.astype(np.float64) * float(two_n) / float(q)
    r = np.trunc(x)
    r = r + (x - r >= 0.5)
    return (r.astype(np.int64) % two_n).astype(np.uint32)


def mono_mul(y, e, q):
    """X^e * y mod (X^N + 1, Q) for e in [0, 2N); y holds canonical Python ints."""
    n = len(y)
    idx = (np.arange(n) - e) % (2 * n)
    out = np.empty(n, dtype=object)
    for k in range(n):
        j = idx[k]
        out[k] = y[j] if j < n else (q - y[j - n]) % q
    return out


def negacyclic_sum(pairs, q, n):
    """sum of x * y mod (X^N + 1, Q) over (digit polynomial, key polynomial) pairs: digits are
    below 2^8, keys are canonical words split into 16-bit limbs, so every int64 convolution and
    their sums are exact (N * 2^8 * 2^16 * pairs < 2^63)."""
    limbs = 4 if q > 2**32 else 2
    tot = np.zeros((limbs, n), np.int64)
    for d, key in pairs:
        key = key.astype(np.uint64)
        for lb in range(limbs):
            kl = ((key >> np.uint64(16 * lb)) & np.uint64(0xFFFF)).astype(np.int64)
            c = np.convolve(d, kl)
            tot[lb] += c[:n]
            tot[lb, :n - 1] -= c[n:]
    words = [sum(int(tot[lb, k]) << (16 * lb) for lb in range(limbs)) % q for k in range(n)]
    return np.array(words, dtype=object)


def digits(e, bits, length):
    v = np.array([int(x) for x in e], dtype=np.uint64)
    mask = np.uint64((1 << bits) - 1)
    return [((v >> np.uint64(j * bits)) & mask).astype(np.int64) for j in range(length)]


def external_product(ea, eb, rgsw, bits, length, q):
    """rgsw[part][j][a|b][N] coefficient domain; part 0 multiplies the digits of E.a, part 1 those
    of E.b."""
    n = len(ea)
    da, db = digits(ea, bits, length), digits(eb, bits, length)
    out = []
    for ab in range(2):
        pairs = [(da[j], rgsw[0, j, ab]) for j in range(length)]
        pairs += [(db[j], rgsw[1, j, ab]) for j in range(length)]
        out.append(negacyclic_sum(pairs, q, n))
    return out


def blind_rotate(p, bsk, lwe_sk_ternary, ms, lut, steps, q):
    n_ring, n, length, bits = p.ring_dim, p.lwe_dim, p.br_len, p.br_bits
    pairs = 2 if lwe_sk_ternary else 1
    bsk = bsk.reshape(n, pairs, 2, length, 2, n_ring)
    acc_a = np.array([0] * n_ring, dtype=object)
    acc_b = mono_mul(np.array([int(x) for x in lut], dtype=object),
                     (2 * n_ring - int(ms[n])) % (2 * n_ring), q)
    for i in range(steps):
        a = int(ms[i])
        if a == 0:  # binary.rs:70, ternary.rs:73
            continue
        ea = (mono_mul(acc_a, a, q) - acc_a) % q
        eb = (mono_mul(acc_b, a, q) - acc_b) % q
        if pairs == 1:
            rgsw = bsk[i, 0]
        else:
            k0, k1 = bsk[i, 0].astype(object), bsk[i, 1]
            rgsw = np.empty(k0.shape, dtype=object)
            for part in range(2):
                for j in range(length):
                    for ab in range(2):
                        m = mono_mul(np.array([int(x) for x in k1[part, j, ab]], dtype=object),
                                     2 * n_ring - a, q)
                        rgsw[part, j, ab] = (k0[part, j, ab] - m) % q
            rgsw = np.array([[[[int(x) for x in rgsw[pt, j, ab]] for ab in range(2)]
                              for j in range(length)] for pt in range(2)], dtype=np.uint64)
        oa, ob = external_product(ea, eb, rgsw, bits, length, q)
        acc_a, acc_b = (acc_a + oa) % q, (acc_b + ob) % q
    return np.concatenate([acc_a, acc_b])


@pytest.mark.parametrize("set_id", ALL_SETS)
def test_first_steps_without_ntt(oracle, oracle_keys, set_id):
    g = np.load(GOLDEN)
    name = oracle.SET_NAMES[set_id]
    k = oracle_keys(set_id)
    p = k.p
    q = oracle.MODULUS[p.field_id]
    c0, c1 = g[f"{name}/c0"][0], g[f"{name}/c1"][0]
    s = np.array([(int(a) + int(b)) % q for a, b in zip(c0, c1)], dtype=np.uint64)
    ms = modswitch(s, q, 2 * p.ring_dim)
    assert (ms == g[f"{name}/ms0"]).all()
    lut = oracle.lut_poly(p.field_id, "nand", p.ring_dim)
    ternary = bool(getattr(p, "lwe_ternary", 0))
    for steps in (1, 2):
        acc = blind_rotate(p, k.bsk, ternary, ms, lut, steps, q)
        assert (acc.astype(np.uint64) == g[f"{name}/acc{steps}"].astype(np.uint64)).all(), steps


def test_modswitch_rounding_edges():
    q, two_n = 2**31 - 2**27 + 1, 2048
    # v * 2N / Q just below one half rounds down, just above rounds up
    assert modswitch(np.array([q // 4096], dtype=np.uint64), q, two_n)[0] == 0
    assert modswitch(np.array([q // 4096 + 1], dtype=np.uint64), q, two_n)[0] == 1
    # the largest words map to 2N, which wraps to 0
    assert modswitch(np.array([q - 1], dtype=np.uint64), q, two_n)[0] == 0
    # (Q + 1) / 2 lands on N
    assert modswitch(np.array([(q + 1) // 2], dtype=np.uint64), q, two_n)[0] == two_n // 2
