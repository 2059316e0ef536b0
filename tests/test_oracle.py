"""The CPU oracle against the reference's own known-answer tests and properties, and against the
committed golden fixtures (tests/golden/gen_golden.py)."""

import os

import numpy as np
import pytest

from conftest import rng

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden_seed0.npz")
FIELDS = [0, 1, 2]


def rand_poly(oracle, field, n, seed):
    q = oracle.MODULUS[field]
    return (rng(seed).integers(0, 2**63, n, dtype=np.uint64) % np.uint64(q)).astype(
        oracle.dtype_of(field))


@pytest.mark.parametrize("field", FIELDS)
def test_monomial_products_kat(oracle, field):
    # algebra/src/baby_bear/babybear_ntt.rs:185-213: 37 X^50 * 67 X^70 = 2479 X^120,
    # and * 55 X^90 = 136345 X^210
    dt = oracle.dtype_of(field)
    p1, p2, p3 = (np.zeros(1024, dt) for _ in range(3))
    p1[50], p2[70], p3[90] = 37, 67, 55
    prod = oracle.negacyclic_mul(field, 10, p1, p2)
    expect = np.zeros(1024, dt)
    expect[120] = 37 * 67
    assert (prod == expect).all()
    prod3 = oracle.negacyclic_mul(field, 10, prod, p3)
    expect3 = np.zeros(1024, dt)
    expect3[210] = 37 * 67 * 55
    assert (prod3 == expect3).all()
    # wrap-around is negacyclic: X^600 * X^600 = -X^176
    a = np.zeros(1024, dt)
    a[600] = 1
    w = oracle.negacyclic_mul(field, 10, a, a)
    assert w[176] == oracle.MODULUS[field] - 1 and np.count_nonzero(w) == 1


@pytest.mark.parametrize("field", FIELDS)
@pytest.mark.parametrize("log_n", [5, 10, 11])
def test_ntt_roundtrip_and_schoolbook(oracle, field, log_n):
    # goldilocks_ntt.rs:173-183 / babybear_ntt.rs:169-182 round trips; polynomial_test.rs:110-154
    n = 1 << log_n
    x = rand_poly(oracle, field, n, 1 + log_n)
    y = rand_poly(oracle, field, n, 2 + log_n)
    assert (oracle.ntt_roundtrip(field, log_n, x) == x).all()
    if log_n <= 10:
        assert (oracle.negacyclic_mul(field, log_n, x, y) ==
                oracle.negacyclic_mul(field, log_n, x, y, schoolbook=True)).all()


@pytest.mark.parametrize("field,bits,length", [(1, 5, 13), (1, 8, 8), (0, 8, 4), (0, 5, 7),
                                               (2, 3, 9), (2, 7, 4), (2, 1, 27)])
def test_external_product_vs_plaintext(oracle, field, bits, length):
    # lattice/tests/lattice_test.rs:352-406: RGSW(m) x RLWE(p) decrypts to m*p. With a noiseless
    # "RGSW" of message 1 under key 0 (c_m rows = (0, B^j), c_neg_s_m rows = (B^j, 0)) the external
    # product must reproduce the input exactly (gadget recomposition).
    n = 64
    dt = oracle.dtype_of(field)
    rgsw = np.zeros((2, length, 2, n), dt)
    for j in range(length):
        rgsw[0, j, 0, 0] = 1 << (bits * j)
        rgsw[1, j, 1, 0] = 1 << (bits * j)
    rl = np.stack([rand_poly(oracle, field, 2 * n, 5)]).reshape(1, 2 * n)
    out = oracle.external_product(field, 6, bits, length, rl, rgsw.reshape(-1))
    assert (out == rl).all()


def test_keygen_deterministic_and_truth_tables(oracle, oracle_keys):
    p = oracle.preset(0)
    k = oracle_keys(0)
    k2 = oracle.keygen(p, 0, threads=3)
    assert (k.bsk == k2.bsk).all() and (k.ksk == k2.ksk).all()
    assert set(np.unique(k.lwe_sk)) <= {0, 1}
    assert set(np.unique(k.ring_sk)) <= {0, 1, oracle.MODULUS[0] - 1}
    bits = np.array([0, 0, 1, 1], np.uint8), np.array([0, 1, 0, 1], np.uint8)
    c0 = oracle.encrypt(p, k.lwe_sk, 3, 0, bits[0])
    c1 = oracle.encrypt(p, k.lwe_sk, 3, 4, bits[1])
    tables = {"nand": lambda a, b: 1 - (a & b), "and": lambda a, b: a & b, "or": lambda a, b: a | b,
              "nor": lambda a, b: 1 - (a | b), "xor": lambda a, b: a ^ b,
              "xnor": lambda a, b: 1 - (a ^ b)}
    q = oracle.MODULUS[0]
    for g, f in tables.items():
        m, noise = oracle.decrypt(p, k.lwe_sk, oracle.gate(k, g, c0, c1))
        assert (m == f(*bits)).all(), g
        assert (noise < q // 16).all(), g  # tfhe/examples/nand_babybear.rs:16-24


def test_golden_fixtures_reproduce(oracle, oracle_keys):
    import hashlib
    g = np.load(GOLDEN)
    for pid, name in oracle.SET_NAMES.items():
        k = oracle_keys(pid)
        assert hashlib.sha256(k.bsk.tobytes()).hexdigest() == str(g[f"{name}/sha_bsk"])
        assert hashlib.sha256(k.ksk.tobytes()).hexdigest() == str(g[f"{name}/sha_ksk"])
        if pid == 0:  # full bootstrap re-run on the fast set; the others are checked on the GPU
            out = oracle.gate(k, "nand", g[f"{name}/c0"], g[f"{name}/c1"])
            assert (out == g[f"{name}/nand"]).all()
        m, noise = oracle.decrypt(k.p, k.lwe_sk, g[f"{name}/nand"])
        assert (m == [1, 1, 1, 0]).all()
        assert (noise == g[f"{name}/nand_noise"]).all()
        assert (noise < oracle.MODULUS[k.p.field_id] // 16).all()
        # the first row's combined input through the modulus switch and the blind rotation
        q = oracle.MODULUS[k.p.field_id]
        c0, c1 = g[f"{name}/c0"][0], g[f"{name}/c1"][0]
        s = np.array([(int(a) + int(b)) % q for a, b in zip(c0, c1)], c0.dtype)
        assert (oracle.modswitch(k.p, s) == g[f"{name}/ms0"]).all()
        lut = oracle.lut_poly(k.p.field_id, "nand", k.p.ring_dim)
        for steps in (1, 2, 10, k.p.lwe_dim):
            assert (oracle.blind_rotate(k, s, lut, steps) == g[f"{name}/acc{steps}"]).all(), steps


@pytest.mark.parametrize("set_id", [3, 4, 100])
def test_default_field_sets_truth_tables(oracle, oracle_keys, set_id):
    # DEFAULT_TERNARY_128_BITS (n = N: one key-switching chunk), CUSTOM_TERNARY_128_BITS (n = 512:
    # two chunks of 512) and the ternary-LWE-key blind rotation on the CUSTOM set.
    k = oracle_keys(set_id)
    p = k.p
    if set_id == 100:
        assert set(np.unique(k.lwe_sk)) == {0, 1, oracle.MODULUS[2] - 1}
    else:
        assert set(np.unique(k.lwe_sk)) <= {0, 1} and set(np.unique(k.ring_sk)) <= {0, 1}
    bits = np.array([0, 0, 1, 1], np.uint8), np.array([0, 1, 0, 1], np.uint8)
    c0 = oracle.encrypt(p, k.lwe_sk, 9, 0, bits[0])
    c1 = oracle.encrypt(p, k.lwe_sk, 9, 4, bits[1])
    for g, f in (("nand", lambda a, b: 1 - (a & b)), ("xor", lambda a, b: a ^ b)):
        m, noise = oracle.decrypt(p, k.lwe_sk, oracle.gate(k, g, c0, c1))
        assert (m == f(*bits)).all(), g
        assert (noise < oracle.MODULUS[2] // 16).all(), g


def test_cbd_error_polynomials(oracle):
    # sigma exactly 3.2 selects sample_cbd_field_vec for RLWE error polynomials
    # (algebra/src/random.rs:91-92); in a release build its a < b branch yields b - a for a
    # 32-bit field, so every error coefficient lies in [0, 13].
    p = oracle.preset(4)
    p.ks_noise_std = 3.2
    k = oracle.keygen(p, 2)
    M, L = 512, p.ks_len
    s = np.zeros(M, np.uint32)
    s[:p.lwe_dim] = k.lwe_sk
    q = oracle.MODULUS[2]
    ksk = k.ksk.reshape(2, L, 2, M)
    errs = []
    for c in range(2):
        z = k.ring_sk[c * M:(c + 1) * M].astype(np.uint64)
        for j in range(L):
            a_s = oracle.negacyclic_mul(2, 9, ksk[c, j, 0], s).astype(np.uint64)
            zb = (z * pow(2, 7 * j, q)) % q
            e = (ksk[c, j, 1].astype(np.uint64) + 2 * q - a_s - zb) % q
            errs.append(e)
    e = np.concatenate(errs)
    assert e.max() <= 13 and e.min() == 0 and np.count_nonzero(e) > len(e) // 2


def test_blind_rotation_trace_rows(oracle, oracle_keys):
    # one pass over all n steps gives the per-step probes' accumulators (golden rows 1, 2, 10, n),
    # and a step whose rotation is zero repeats the previous row; binary and ternary LWE keys
    g = np.load(GOLDEN)
    for pid in (0, 100):
        name = oracle.SET_NAMES[pid]
        k = oracle_keys(pid)
        q = oracle.MODULUS[k.p.field_id]
        c0, c1 = g[f"{name}/c0"][0], g[f"{name}/c1"][0]
        s = np.array([(int(a) + int(b)) % q for a, b in zip(c0, c1)], c0.dtype)
        lut = oracle.lut_poly(k.p.field_id, "nand", k.p.ring_dim)
        rows = oracle.blind_rotate_trace(k, s, lut)
        n = k.p.lwe_dim
        assert rows.shape == (n, 2 * k.p.ring_dim)
        for steps in (1, 2, 10, n):
            assert (rows[steps - 1] == g[f"{name}/acc{steps}"]).all(), (pid, steps)
        ms = g[f"{name}/ms0"]
        for i in range(1, n):
            if ms[i] == 0:
                assert (rows[i] == rows[i - 1]).all(), (pid, i)


def _rot_sub(y, r, q):
    """(X^r - 1) y in Z_q[X]/(X^N + 1), canonical (numpy object arithmetic)."""
    N = len(y)
    y = [int(v) for v in y]
    x = [0] * N
    for k in range(N):
        s = k - r
        x[k] = y[s] if s >= 0 else (q - y[s + N]) % q if s >= -N else y[s + 2 * N]
    return [(x[k] - y[k]) % q for k in range(N)]


def test_blind_rotation_trace_digits(oracle, oracle_keys):
    """The trace's gadget digits of every step are below B, recombine (sum d_j B^j) to
    E = (X^a_i - 1) ACC computed without any NTT from the previous accumulator row, and are zero on
    steps whose rotation a_i is zero (binary LWE keys; the unsigned LSB-first decomposition of
    native_polynomial.rs:340-348)."""
    g = np.load(GOLDEN)
    for pid in (0, 1):
        name = oracle.SET_NAMES[pid]
        k = oracle_keys(pid)
        q, N, L, b = oracle.MODULUS[k.p.field_id], k.p.ring_dim, k.p.br_len, k.p.br_bits
        c0, c1 = g[f"{name}/c0"][0], g[f"{name}/c1"][0]
        s = np.array([(int(a) + int(x)) % q for a, x in zip(c0, c1)], c0.dtype)
        lut = oracle.lut_poly(k.p.field_id, "nand", N)
        rows, dig = oracle.blind_rotate_trace(k, s, lut, digits=True)
        assert dig.shape == (k.p.lwe_dim, 2, L, N) and int(dig.max()) < (1 << b)
        ms = oracle.modswitch(k.p, s)
        weights = [1 << (b * j) for j in range(L)]
        for i in (1, 2, 57, k.p.lwe_dim - 1):
            if ms[i] == 0:
                assert not dig[i].any()
                continue
            prev = rows[i - 1]
            for part in (0, 1):
                e = _rot_sub(prev[part * N:(part + 1) * N], int(ms[i]), q)
                got = [sum(int(dig[i, part, j, c]) * weights[j] for j in range(L)) for c in range(N)]
                assert got == e, (pid, i, part)
        zero = [i for i in range(k.p.lwe_dim) if ms[i] == 0]
        assert all(not dig[i].any() for i in zero)
