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
From the accumulator after all n steps it also recomputes b[0] += Q/8 (tfhe/src/bfhe/evaluate.rs:52),
the RLWE key switch in n'-word chunks (fhe_core/src/key_switch/rlwe.rs:115-137,250-286) and the
sample extraction (lattice/src/rlwe.rs:393-402), and gets the committed NAND output.

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


def key_switch(p, ksk, acc, q):
    """LWE of dimension n from the accumulator [a | b] (canonical) under the key-switching key
    ksk[c][j][a|b][n'], n' = next_pow2(n), one gadget RLWE per n'-word chunk of the ring key."""
    n_ring, n = p.ring_dim, p.lwe_dim
    m = 1 << (n - 1).bit_length()
    chunks = n_ring // m
    a = [int(x) for x in acc[:n_ring]]
    b0 = (int(acc[n_ring]) + (q >> 3)) % q  # evaluate.rs:52
    if m != n_ring:  # rlwe.rs:123-131: negate a[0], reverse the rest; then the same per chunk
        a = [(q - a[0]) % q] + a[1:][::-1]
        for c in range(chunks):
            ch = a[c * m:(c + 1) * m]
            a[c * m:(c + 1) * m] = [(q - ch[0]) % q] + ch[1:][::-1]
    ksk = ksk.reshape(chunks, p.ks_len, 2, m)
    pairs_a, pairs_b = [], []
    for c in range(chunks):
        # sub_assign_gadget_rlwe_mul_polynomial_inplace_fast (lattice/src/rlwe.rs:1147-1166):
        # the digits of -a, products added
        ds = digits([(q - x) % q for x in a[c * m:(c + 1) * m]], p.ks_bits, p.ks_len)
        pairs_a += [(ds[j], ksk[c, j, 0]) for j in range(p.ks_len)]
        pairs_b += [(ds[j], ksk[c, j, 1]) for j in range(p.ks_len)]
    ia, ib = negacyclic_sum(pairs_a, q, m), negacyclic_sum(pairs_b, q, m)
    # extract_partial_lwe_locally: a' = [A0, -A(n'-1), ..., -A(n'-n+1)], b' = B0 + b0
    out = [ia[0]] + [(q - ia[m - k]) % q for k in range(1, n)] + [(ib[0] + b0) % q]
    return np.array(out, dtype=np.uint64)


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
    # init_nand_lut (tfhe/src/bfhe/evaluate.rs:267-330): Q/8 on [0, 3N/4), -Q/8 on [3N/4, N)
    mid = 3 * p.ring_dim // 4
    assert (lut[:mid] == q >> 3).all() and (lut[mid:] == q - (q >> 3)).all()
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


@pytest.mark.parametrize("set_id", ALL_SETS)
def test_key_switch_and_extraction_without_ntt(oracle, oracle_keys, set_id):
    g = np.load(GOLDEN)
    name = oracle.SET_NAMES[set_id]
    k = oracle_keys(set_id)
    p = k.p
    q = oracle.MODULUS[p.field_id]
    acc = g[f"{name}/acc{p.lwe_dim}"]
    out = key_switch(p, k.ksk, acc, q)
    assert (out == g[f"{name}/nand"][0].astype(np.uint64)).all()
