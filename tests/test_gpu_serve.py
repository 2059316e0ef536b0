"""The serving loop: every request's outputs are identical alone and inside the continuous batch,
across parameter sets, with admission against an HBM budget."""

import numpy as np
import pytest

from conftest import hb_params_of

pytestmark = pytest.mark.gpu

SETS = [0, 1, 2, 3, 4, 100]  # the five presets and the ternary-LWE-key set


@pytest.fixture(scope="module")
def setup(hb):
    ctx = hb.Context(0)
    evs = {}
    for pid in SETS:
        sk = hb.KeyGen.generate_secret_key(hb_params_of(hb, pid), 0)
        evs[pid] = (sk, hb.Evaluator(sk, ctx))
    yield ctx, evs
    for sk, ev in evs.values():
        ev.keys.free()
    ctx.close()


def _plan(evs, n, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        pid = SETS[int(rng.integers(0, len(SETS)))]
        count = int(np.exp(rng.uniform(0, np.log(200))))
        gate = ["nand", "and", "xor", "majority"][i % 4]
        sk, ev = evs[pid]
        bits = rng.integers(0, 2, (3, count)).astype(np.uint8)
        cs = [sk.encrypt(bits[k], (seed << 28) + (i << 16) + (k << 12)) for k in range(3)]
        reqs.append((pid, gate, cs, bits))
    return reqs


def _alone(evs, pid, gate, cs):
    sk, ev = evs[pid]
    if gate == "majority":
        return ev.majority(cs[0], cs[1], cs[2])
    return {"nand": ev.nand, "and": ev.and_, "xor": ev.xor}[gate](cs[0], cs[1])


def test_serve_results_equal_alone(hb, setup):
    ctx, evs = setup
    srv = hb.Server(ctx, max_wave_gates=600)
    reqs = _plan(evs, 24, 11)
    ids = {}
    # first burst, then more requests while the first ones are on the GPU
    for r in reqs[:12]:
        ids[srv.submit(evs[r[0]][1], r[1], r[2][0], r[2][1], r[2][2] if r[1] == "majority" else None)] = r
    first = srv.next_done(60.0)
    assert first is not None
    for r in reqs[12:]:
        ids[srv.submit(evs[r[0]][1], r[1], r[2][0], r[2][1], r[2][2] if r[1] == "majority" else None)] = r
    got = {}
    got[first] = srv.fetch(first)
    while len(got) < len(ids):
        rid = srv.next_done(60.0)
        assert rid is not None
        got[rid] = srv.fetch(rid)
    st = srv.stats()
    assert srv.stop() == 0
    assert st["completed"] == len(reqs) and st["failed"] == 0 and st["waves"] >= 2
    assert 0 < st["p50_latency_s"] <= st["p99_latency_s"]
    for rid, (pid, gate, cs, bits) in ids.items():
        out, lat = got[rid]
        assert lat > 0
        assert (out == _alone(evs, pid, gate, cs)).all(), (rid, pid, gate)


def test_serve_budget_admits_one_at_a_time(hb, setup):
    ctx, evs = setup
    reqs = _plan(evs, 6, 12)
    largest = max(len(r[2][0]) * r[2][0].shape[1] * r[2][0].itemsize * 4 for r in reqs)
    srv = hb.Server(ctx, hbm_budget=largest)
    ids = {srv.submit(evs[p][1], g, cs[0], cs[1], cs[2] if g == "majority" else None): (p, g, cs)
           for p, g, cs, _ in reqs}
    done = 0
    while done < len(ids):
        rid = srv.next_done(60.0)
        assert rid is not None
        out, _ = srv.fetch(rid)  # fetching returns memory, which admits the next request
        p, g, cs = ids[rid]
        assert (out == _alone(evs, p, g, cs)).all()
        done += 1
    st = srv.stats()
    assert st["hbm_peak"] <= largest and st["completed"] == len(reqs)
    assert srv.stop() == 0


def test_serve_sheds_load_beyond_queue_bound(hb, setup):
    """With max_queue_s, a submission whose predicted completion (work ahead of it over the key
    set's calibrated rate) lies beyond the bound is refused; the admitted ones complete unchanged."""
    from hasteboots_b200._lib import lib
    ctx, evs = setup
    sk, ev = evs[0]
    assert lib().hb_keys_set_rate(ev.keys.handle, 1000.0) == 0  # 1000 gates/s: 0.2 s per request
    try:
        srv = hb.Server(ctx, max_queue_s=0.5)
        bits = np.random.default_rng(21).integers(0, 2, (2, 200)).astype(np.uint8)
        c0, c1 = sk.encrypt(bits[0], 77 << 20), sk.encrypt(bits[1], 78 << 20)
        ids = [srv.submit(ev, "nand", c0, c1) for _ in range(8)]
        accepted = [i for i in ids if i is not None]
        assert ids[0] is not None and ids[1] is not None  # 0.4 s of predicted work fits
        assert len(accepted) < len(ids)
        ref = ev.nand(c0, c1)
        for _ in accepted:
            rid = srv.next_done(60.0)
            assert rid in accepted
            out, _ = srv.fetch(rid)
            assert (out == ref).all()
        st = srv.stats()
        assert srv.stop() == 0
        assert st["rejected"] == len(ids) - len(accepted) and st["completed"] == len(accepted)
    finally:
        lib().hb_keys_set_rate(ev.keys.handle, 0.0)
