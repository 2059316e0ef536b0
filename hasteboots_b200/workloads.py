"""Seeded definitions of the measured workloads, shared by bench.py, the GPU tests and the script
that records the oracle's digests of their outputs (tests/golden/gen_digests.py), so that all three
encrypt the same bits at the same encryption indices.

* headline: NAND over GOLDILOCKS_BINARY_128_BITS, 16384 gates, input bits from seed 3 + rank,
  c0 encrypted at indices 0.., c1 at 2^20.. (seed-0 keys).
* mixed: 64 jobs; per job a parameter set drawn uniformly from {BABYBEAR, GOLDILOCKS, ZAMA}
  (presets 0, 1, 2), a gate count log-uniform in [1, 4096], the gate kinds cycling NAND, AND, OR,
  NOR, XOR, XNOR, MAJORITY, and three input-bit rows (the third feeds MAJORITY only), all from
  seed 4; input k of job i is encrypted at indices (i << 24) + (k << 20).
"""

from dataclasses import dataclass

import numpy as np

HEADLINE_PRESET = 1  # GOLDILOCKS_BINARY_128_BITS
HEADLINE_GATES = 16384
HEADLINE_INDEX0 = (0, 1 << 20)

MIXED_GATES = ("nand", "and", "or", "nor", "xor", "xnor", "majority")


def headline_bits(gates=HEADLINE_GATES, rank=0):
    """Input bits of the headline batch, shape (2, gates)."""
    return np.random.default_rng(3 + rank).integers(0, 2, (2, gates)).astype(np.uint8)


def truth(gate, a, b, c=None):
    """Plaintext result of a gate on bit arrays."""
    return {"nand": lambda: 1 - (a & b), "and": lambda: a & b, "or": lambda: a | b,
            "nor": lambda: 1 - (a | b), "xor": lambda: a ^ b, "xnor": lambda: 1 - (a ^ b),
            "majority": lambda: (a & b) | (b & c) | (a & c)}[gate]().astype(np.uint8)


@dataclass
class MixedJob:
    index: int
    preset: int
    count: int
    gate: str
    bits: np.ndarray  # (3, count) uint8

    def index0(self, k):
        """Encryption index of the first ciphertext of input k."""
        return (self.index << 24) + (k << 20)

    @property
    def inputs(self):
        return 3 if self.gate == "majority" else 2

    def expected(self):
        a, b, c = self.bits
        return truth(self.gate, a, b, c)


def mixed_plan(seed=4, jobs=64):
    rng = np.random.default_rng(seed)
    plan = []
    for i in range(jobs):
        pid = int(rng.integers(0, 3))
        count = int(np.clip(np.round(np.exp(rng.uniform(0, np.log(4096)))), 1, 4096))
        bits = rng.integers(0, 2, (3, count)).astype(np.uint8)
        plan.append(MixedJob(i, pid, count, MIXED_GATES[i % len(MIXED_GATES)], bits))
    return plan


def slice_digests(words, rows_per_slice):
    """SHA-256 (hex) of consecutive slices of `rows_per_slice` ciphertexts, little-endian words."""
    import hashlib
    words = np.ascontiguousarray(words)
    return [hashlib.sha256(words[i:i + rows_per_slice].astype(words.dtype.newbyteorder("<")).tobytes()).hexdigest()
            for i in range(0, len(words), rows_per_slice)]


def digest(words):
    import hashlib
    words = np.ascontiguousarray(words)
    return hashlib.sha256(words.astype(words.dtype.newbyteorder("<")).tobytes()).hexdigest()
