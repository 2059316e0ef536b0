"""Generate the golden fixtures of tests/golden/ with the CPU oracle.

    python tests/golden/gen_golden.py

For each key set (the BABYBEAR / GOLDILOCKS / ZAMA _BINARY_128_BITS and DEFAULT / CUSTOM
_TERNARY_128_BITS presets, and CUSTOM_TERNARY_128_BITS with a ternary LWE key) with key seed 0 it
records:
SHA-256 digests of the secret keys, BSK and KSK (the project's seeded key convention); the input
ciphertexts of the four NAND truth-table rows (encryption seed 0, sample indices 0..7); the oracle's
NAND outputs and their decryption noise; the modulus switch of the first row's combined input
c0 + c1 (ms0) and the NAND blind-rotation accumulator of that input, [a | b] canonical, after 1, 2
and 10 steps and after all n steps (acc<n>: the RLWE that enters b[0] += Q/8 and the key switch).
The BabyBear set also records every other gate and a caller-LUT bootstrap.
The reference ships no golden vectors (its tests draw from OS entropy), so these files pin the
oracle and the GPU path against each other and against regressions.
"""

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import binding as O  # noqa: E402

ROWS = np.array([[0, 0], [0, 1], [1, 0], [1, 1]], np.uint8)


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    out = {}
    for pid, name in O.SET_NAMES.items():
        p = O.params(pid)
        k = O.keygen(p, 0)
        out[f"{name}/sha_lwe_sk"] = np.array(digest(k.lwe_sk))
        out[f"{name}/sha_ring_sk"] = np.array(digest(k.ring_sk))
        out[f"{name}/sha_bsk"] = np.array(digest(k.bsk))
        out[f"{name}/sha_ksk"] = np.array(digest(k.ksk))
        c0 = O.encrypt(p, k.lwe_sk, 0, 0, ROWS[:, 0])
        c1 = O.encrypt(p, k.lwe_sk, 0, 4, ROWS[:, 1])
        out[f"{name}/c0"] = c0
        out[f"{name}/c1"] = c1
        out[f"{name}/nand"] = O.gate(k, "nand", c0, c1)
        out[f"{name}/nand_noise"] = O.decrypt(p, k.lwe_sk, out[f"{name}/nand"])[1]
        q = O.MODULUS[p.field_id]
        s = np.array([(int(a) + int(b)) % q for a, b in zip(c0[0], c1[0])], O.dtype_of(p.field_id))
        out[f"{name}/ms0"] = O.modswitch(p, s)
        nl = O.lut_poly(p.field_id, "nand", p.ring_dim)
        for steps in (1, 2, 10, p.lwe_dim):
            out[f"{name}/acc{steps}"] = O.blind_rotate(k, s, nl, steps)
        if pid == O.PRESET_BABYBEAR:
            c2 = O.encrypt(p, k.lwe_sk, 0, 8, np.array([1, 0, 1, 0], np.uint8))
            out[f"{name}/c2"] = c2
            for g in ("and", "or", "nor", "xor", "xnor"):
                out[f"{name}/{g}"] = O.gate(k, g, c0, c1)
            out[f"{name}/majority"] = O.gate(k, "majority", c0, c1, c2)
            out[f"{name}/mux"] = O.gate(k, "mux", c0, c1, c2)
            out[f"{name}/not"] = O.gate(k, "not", c0)
            lut = (np.random.default_rng(11).integers(0, O.MODULUS[p.field_id], p.ring_dim,
                                                       dtype=np.uint64)).astype(np.uint32)
            out[f"{name}/lut"] = lut
            out[f"{name}/bootstrap_lut"] = O.bootstrap_lut(k, c0, lut)
    np.savez_compressed(os.path.join(HERE, "golden_seed0.npz"), **out)
    print("wrote", os.path.join(HERE, "golden_seed0.npz"), len(out), "arrays")


if __name__ == "__main__":
    main()
