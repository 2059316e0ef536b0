"""Host logic of the measured workloads (CPU): the seeded plans that bench.py, the GPU tests and the
digest generator share, the digest helpers, the committed digest file's shape, and the algorithmic
modular-multiply counts behind bench.py's roofline."""

import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from hasteboots_b200 import workloads as W  # noqa: E402


def test_headline_bits_are_seeded():
    a, b = W.headline_bits(), W.headline_bits()
    assert a.shape == (2, W.HEADLINE_GATES) and a.dtype == np.uint8
    assert (a == b).all() and set(np.unique(a)) <= {0, 1}
    assert not (W.headline_bits(rank=1) == a).all()


def test_mixed_plan_is_seeded_and_covers_the_three_sets():
    plan, again = W.mixed_plan(), W.mixed_plan()
    assert len(plan) == 64
    assert [(j.preset, j.count, j.gate) for j in plan] == [(j.preset, j.count, j.gate) for j in again]
    assert all((j.bits == k.bits).all() for j, k in zip(plan, again))
    assert {j.preset for j in plan} == {0, 1, 2}
    assert all(1 <= j.count <= 4096 for j in plan)
    assert sum(j.count for j in plan) == 32847
    assert {j.gate for j in plan} == set(W.MIXED_GATES)
    # encryption indices of different inputs and jobs never overlap (counts stay below 2^20)
    starts = sorted(j.index0(k) for j in plan for k in range(j.inputs))
    assert len(set(starts)) == len(starts)
    assert max(j.count for j in plan) < (1 << 20)


def test_truth_tables():
    a = np.array([0, 0, 1, 1], np.uint8)
    b = np.array([0, 1, 0, 1], np.uint8)
    c = np.array([1, 0, 1, 0], np.uint8)
    assert list(W.truth("nand", a, b)) == [1, 1, 1, 0]
    assert list(W.truth("xor", a, b)) == [0, 1, 1, 0]
    assert list(W.truth("majority", a, b, c)) == [0, 0, 1, 1]


def test_digests_are_little_endian_sha256_of_slices():
    x = np.arange(6 * 3, dtype=np.uint64).reshape(6, 3)
    d = W.slice_digests(x, 4)
    assert len(d) == 2
    assert d[0] == hashlib.sha256(x[:4].astype("<u8").tobytes()).hexdigest()
    assert W.digest(x) == hashlib.sha256(x.astype("<u8").tobytes()).hexdigest()


def test_committed_digests_cover_every_output():
    d = json.load(open(os.path.join(ROOT, "tests", "golden", "digests_full.json")))
    h = d["headline"]
    assert h["preset"] == W.HEADLINE_PRESET and h["gates"] == W.HEADLINE_GATES
    assert len(h["out_slices"]) * h["slice"] == W.HEADLINE_GATES
    plan = W.mixed_plan()
    assert sorted(int(k) for k in d["mixed"]) == list(range(len(plan)))
    for job in plan:
        r = d["mixed"][str(job.index)]
        assert (r["preset"], r["gate"], r["count"]) == (job.preset, job.gate, job.count)
        assert len(r["inputs"]) == job.inputs


def test_modmul_counts():
    import bench
    # GOLDILOCKS: 728 steps of 18 transforms and 32 N products, key switch 15 transforms + 26 N
    assert bench.modmuls_per_gate(1024, 728, 8, 13) == 728 * (18 * 5120 + 32 * 1024) + 15 * 5120 + 26 * 1024
    # ZAMA and BABYBEAR as in the published per-gate figures
    assert abs(bench.modmuls_per_gate(1024, 728, 13, 13) - 1.432e8) / 1.432e8 < 1e-3
    assert abs(bench.modmuls_per_gate(1024, 728, 4, 7) - 4.926e7) / 4.926e7 < 1e-3
    # CUSTOM_TERNARY (n = 512): the key switch in two chunks of 512-point transforms
    kn = 512
    ks = (2 * 4 + 2) * (kn // 2) * 9 + 2 * 2 * 4 * kn
    assert bench.modmuls_per_gate(1024, 512, 4, 4) == 512 * (10 * 5120 + 16 * 1024) + ks
