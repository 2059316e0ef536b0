"""Autotuner and mixed-parameter-set batches (one graph launch) against single-set launches."""

import numpy as np
import pytest

from conftest import hb_params_of
from gpu_util import empty_dev, from_dev, to_dev

SETS = [0, 1, 2, 3, 4, 100]  # the five presets and the ternary-LWE-key set

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(hb):
    c = hb.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def evaluators(hb, ctx):
    evs = {}
    for pid in SETS:
        sk = hb.KeyGen.generate_secret_key(hb_params_of(hb, pid), 0)
        evs[pid] = (sk, hb.Evaluator(sk, ctx))
    yield evs
    for sk, ev in evs.values():
        ev.keys.free()


def test_autotune_picks_a_compiled_variant(hb, evaluators, ctx):
    import ctypes
    from hasteboots_b200._lib import lib
    sk, ev = evaluators[0]
    (t, g), rate, cached = hb.autotune(ev, sample_gates=148 * 24, use_cache=False)
    assert t in (64, 128) and g in (4, 6, 8) and rate > 0 and not cached
    tt, gg = ctypes.c_int(), ctypes.c_int()
    lib().hb_keys_config(ev.keys.handle, ctypes.byref(tt), ctypes.byref(gg))
    assert (tt.value, gg.value) == (t, g)
    assert lib().hb_keys_set_config(ctx.handle, ev.keys.handle, 64, 5) != 0  # not compiled


def test_key_relayout_keeps_results(hb, evaluators, ctx):
    """Switching the NTT tile (threads per gate) re-lays the device keys out; outputs stay identical."""
    from hasteboots_b200._lib import check, lib
    for pid in (0, 1):
        sk, ev = evaluators[pid]
        bits = np.random.default_rng(9).integers(0, 2, (2, 40)).astype(np.uint8)
        c0, c1 = sk.encrypt(bits[0], 3000), sk.encrypt(bits[1], 4000)
        outs = []
        for t in (64, 128, 64):
            check(lib().hb_keys_set_config(ctx.handle, ev.keys.handle, t, 4), "set_config", ctx.handle)
            outs.append(ev.nand(c0, c1))
        assert (outs[0] == outs[1]).all() and (outs[0] == outs[2]).all()
        assert (sk.decrypt(outs[1]) == 1 - (bits[0] & bits[1])).all()


def test_mixed_batch_equals_alone(hb, evaluators, ctx):
    """Every job's outputs are identical alone (single-set launch) and inside the mixed graph."""
    rng = np.random.default_rng(4)
    gates = ["nand", "and", "or", "xor", "xnor", "nor", "majority"]
    plan = []
    for i in range(12):
        pid = SETS[int(rng.integers(0, len(SETS)))]
        count = int(np.exp(rng.uniform(0, np.log(300))))
        gate = gates[i % len(gates)]
        plan.append((pid, gate, max(1, count)))
    jobs, alone, expect = [], [], []
    for i, (pid, gate, count) in enumerate(plan):
        sk, ev = evaluators[pid]
        bits = rng.integers(0, 2, (3, count)).astype(np.uint8)
        cs = [sk.encrypt(bits[k], 100000 * (i + 1) + 1000 * k) for k in range(3)]
        ds = [to_dev(c) for c in cs]
        out = empty_dev(cs[0].shape, cs[0].dtype)
        jobs.append((ev, gate, ds[0], ds[1], ds[2] if gate == "majority" else None, out))
        fn = {"and": ev.and_, "or": ev.or_}.get(gate, getattr(ev, gate, None))
        args = (cs[0], cs[1], cs[2]) if gate == "majority" else (cs[0], cs[1])
        alone.append(fn(*args))
        a, b, c = bits
        expect.append({"nand": 1 - (a & b), "and": a & b, "or": a | b, "xor": a ^ b,
                       "xnor": 1 - (a ^ b), "nor": 1 - (a | b),
                       "majority": (a & b) | (b & c) | (a & c)}[gate])
    batch = hb.Batch(ctx, jobs)
    info = batch.info()
    assert info["launches"] == len({p for p, _, _ in plan})
    assert all(1 <= g <= 148 for g in info["sm_split"])  # full grids, SMs backfilled across sets
    for rep in range(2):
        batch.launch()
        ctx.synchronize()
        for (pid, gate, count), job, ref, exp in zip(plan, jobs, alone, expect):
            sk = evaluators[pid][0]
            got = from_dev(job[5], ref.dtype)
            assert (got == ref).all(), (pid, gate, count)
            assert (sk.decrypt(got) == exp).all()
    batch.free()
