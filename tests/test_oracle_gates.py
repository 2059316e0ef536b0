"""The gate front-ends and LUT polynomials restated in numpy from the reference's Evaluator
(tfhe/src/bfhe/evaluate.rs:95-262, LUT builders :265-465), checked against the oracle's committed
BabyBear gate outputs through the oracle's plain LUT bootstrap: this pins the oracle's gate
composition independently of its own gate code.

  NOT            -c, then b += Q/4 (no bootstrap)
  NAND/AND/OR/NOR c0 + c1          XOR/XNOR 2 (c0 - c1)          MAJORITY c0 + c1 + c2
  MUX            bootstrap_or(and(c0, c1) + and(not(c0), c2))
  LUTs (lut_step 1, +-Q/8 with Q/8 = Q >> 3):
    NAND +Q/8 on [0, 3N/4), -Q/8 after; AND/MAJORITY the negation
    OR   -Q/8 on [0, N/4), +Q/8 after;  NOR the negation
    XOR  -Q/8 on [0, N/2), +Q/8 after;  XNOR the negation
"""

import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden_seed0.npz")


def lut(q, n, gate):
    q8, nq8 = q >> 3, q - (q >> 3)
    mid, lo = {"nand": (3 * n // 4, q8), "and": (3 * n // 4, nq8), "majority": (3 * n // 4, nq8),
               "or": (n // 4, nq8), "nor": (n // 4, q8), "xor": (n // 2, nq8),
               "xnor": (n // 2, q8)}[gate]
    hi = nq8 if lo == q8 else q8
    out = np.full(n, hi, dtype=object)
    out[:mid] = lo
    return out


def combine(q, terms):
    """sum of s * c over (s, c) pairs, component-wise mod Q."""
    acc = np.zeros(terms[0][1].shape, dtype=object)
    for s, c in terms:
        acc = (acc + s * c.astype(object)) % q
    return acc


def lwe_not(q, c):
    out = (-c.astype(object)) % q
    out[..., -1] = (out[..., -1] + (q >> 2)) % q
    return out


def test_gate_front_ends_and_luts(oracle, oracle_keys):
    g = np.load(GOLDEN)
    name = oracle.SET_NAMES[0]
    k = oracle_keys(0)
    p = k.p
    q, n_ring = oracle.MODULUS[p.field_id], p.ring_dim
    dt = oracle.dtype_of(p.field_id)
    c0, c1, c2 = (g[f"{name}/{x}"] for x in ("c0", "c1", "c2"))
    as_words = lambda x: np.array(x, dtype=np.uint64).astype(dt)  # noqa: E731

    def boot(c, gate):
        return oracle.bootstrap_lut(k, as_words(c), as_words(lut(q, n_ring, gate)))

    assert (as_words(lwe_not(q, c0)) == g[f"{name}/not"]).all()
    for gate in ("nand", "and", "or", "nor"):
        assert (boot(combine(q, [(1, c0), (1, c1)]), gate) == g[f"{name}/{gate}"]).all(), gate
    for gate in ("xor", "xnor"):
        assert (boot(combine(q, [(2, c0), (-2, c1)]), gate) == g[f"{name}/{gate}"]).all(), gate
    maj = combine(q, [(1, c0), (1, c1), (1, c2)])
    assert (boot(maj, "majority") == g[f"{name}/majority"]).all()
    t0 = boot(combine(q, [(1, c0), (1, c1)]), "and")
    t1 = boot(combine(q, [(1, lwe_not(q, c0)), (1, c2)]), "and")
    assert (boot(combine(q, [(1, t0), (1, t1)]), "or") == g[f"{name}/mux"]).all()
    # and the oracle's own LUT builder agrees with the restated one for every gate
    for gate in ("nand", "and", "or", "nor", "xor", "xnor", "majority"):
        assert (oracle.lut_poly(p.field_id, gate, n_ring) == as_words(lut(q, n_ring, gate))).all()
