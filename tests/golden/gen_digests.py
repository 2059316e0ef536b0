"""Records SHA-256 digests of the oracle's outputs for the full-size workloads (CPU only).

    python tests/golden/gen_digests.py [--threads K]

Writes tests/golden/digests_full.json:
  * headline: the 16384 GOLDILOCKS NAND gates of the bench (hasteboots_b200/workloads.py), one
    digest per 1024-gate slice of the output ciphertexts, plus digests of the two input batches;
  * mixed: the 64 jobs of the mixed-set plan, one digest of each job's inputs and of its outputs.
The GPU tests and bench.py hash their own outputs of the same inputs and compare every digest, so
every output ciphertext is checked against the oracle without the oracle running on the GPU host.
The file is rewritten after every slice or job, and a rerun resumes where it stopped. The oracle
needs about 90 CPU-minutes on 8 threads for all of it.
"""

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hasteboots_b200 import workloads as W  # noqa: E402
from oracle import binding as O  # noqa: E402

OUT = os.path.join(HERE, "digests_full.json")
SLICE = 1024


def load():
    if os.path.exists(OUT):
        return json.load(open(OUT))
    return {"format": "sha256 of little-endian words, [count][n + 1] per ciphertext batch",
            "keys_seed": 0, "headline": {}, "mixed": {}}


def save(d):
    tmp = OUT + ".tmp"
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, OUT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    ap.add_argument("--skip-mixed", action="store_true")
    args = ap.parse_args()
    d = load()
    keys = {}

    def keys_of(pid):
        if pid not in keys:
            keys[pid] = O.keygen(O.preset(pid), 0, args.threads)
            keys[pid].evaluator(args.threads)
        return keys[pid]

    # headline
    h = d["headline"]
    p = O.preset(W.HEADLINE_PRESET)
    k = keys_of(W.HEADLINE_PRESET)
    bits = W.headline_bits()
    c0 = O.encrypt(p, k.lwe_sk, 0, W.HEADLINE_INDEX0[0], bits[0])
    c1 = O.encrypt(p, k.lwe_sk, 0, W.HEADLINE_INDEX0[1], bits[1])
    h.update({"preset": W.HEADLINE_PRESET, "gates": W.HEADLINE_GATES, "slice": SLICE,
              "c0": W.digest(c0), "c1": W.digest(c1)})
    outs = h.setdefault("out_slices", [])
    for s in range(len(outs), W.HEADLINE_GATES // SLICE):
        t = time.time()
        out = O.gate(k, "nand", c0[s * SLICE:(s + 1) * SLICE], c1[s * SLICE:(s + 1) * SLICE],
                     threads=args.threads)
        m, _ = O.decrypt(p, k.lwe_sk, out)
        assert (m == W.truth("nand", bits[0], bits[1])[s * SLICE:(s + 1) * SLICE]).all()
        outs.append(W.digest(out))
        save(d)
        print(f"headline slice {s}: {time.time() - t:.0f} s", flush=True)
    if args.skip_mixed:
        return
    for job in W.mixed_plan():
        key = str(job.index)
        if key in d["mixed"]:
            continue
        t = time.time()
        p = O.preset(job.preset)
        k = keys_of(job.preset)
        cs = [O.encrypt(p, k.lwe_sk, 0, job.index0(i), job.bits[i]) for i in range(job.inputs)]
        out = O.gate(k, job.gate, *cs, threads=args.threads)
        m, _ = O.decrypt(p, k.lwe_sk, out)
        assert (m == job.expected()).all()
        d["mixed"][key] = {"preset": job.preset, "gate": job.gate, "count": job.count,
                           "inputs": [W.digest(c) for c in cs], "out": W.digest(out)}
        save(d)
        print(f"mixed job {job.index} ({job.count} gates, preset {job.preset}): {time.time() - t:.0f} s",
              flush=True)


if __name__ == "__main__":
    main()
