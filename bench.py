#!/usr/bin/env python
"""Batched NAND gate bootstrapping throughput on B200.

Workload (the largest single-GPU configuration): 16384 independent NAND gates under
GOLDILOCKS_BINARY_128_BITS_PARAMETERS (N=1024, n=728, B=2^8, l=8, KS base 2^5 x 13) in one
persistent-kernel launch sharing one device-resident BSK/KSK; seed-0 keys, uniformly random input
bit pairs (seed 3; hasteboots_b200/workloads.py). One step = one launch over all gates. Inputs
(191 MB) and the BSK (191 MB) exceed the 126 MB L2, so no flush is needed between steps. Every
output is checked against the NAND truth table and against the oracle's SHA-256 digests of the
same batch (tests/golden/digests_full.json).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--no-extras]

Prints one JSON line (rank 0). At N = 1 the line also carries the other configurations, measured
after the headline: `single` (one BABYBEAR NAND: latency and plain forms), `ntt_microbench` (NTT
round trip and external product, N = 1024/2048, 4096 polynomials), `mixed` (64 jobs over three
sets in one graph, beside the same jobs set by set) and `serve` (Poisson 200 req/s with load
shedding). Multi-GPU runs are replicas (every rank bootstraps its own 16384 gates with its own key
copy; no collective on the data path; weak scaling).
"""

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "bootstraps/s on 1 B200, batched vs 1-gate launches; p50/p99 latency"
PRESET = 1  # GOLDILOCKS_BINARY_128_BITS
GATE_NAND = 0


def modmuls_per_gate(N, n, length, ks_len, ternary=False):
    """Algorithmic modular multiplications of one bootstrap: n steps of (2l+2) size-N NTTs plus the
    4lN-term multiply-accumulate (a ternary LWE key: two RGSWs, so 8lN terms and 2 more inverse
    NTTs), and key switching over N/n' chunks of n' = next_pow2(n) words: l_ks NTTs per chunk, 2
    inverse NTTs and 2 l_ks n' products per chunk, all of size n'."""
    logn = N.bit_length() - 1
    ntt = (N // 2) * logn
    kn = 1 << max(0, (n - 1).bit_length())
    chunks = N // kn
    ks_ntt = (kn // 2) * (kn.bit_length() - 1)
    if ternary:
        step = (2 * length + 4) * ntt + 8 * length * N
    else:
        step = (2 * length + 2) * ntt + 4 * length * N
    return n * step + (chunks * ks_len + 2) * ks_ntt + 2 * chunks * ks_len * kn


def reduce_max(x, world):
    """Max of a per-rank float over all ranks (the step time every replica must wait for)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate(ms_per_step_local, gates_per_rank, world):
    """Whole-job throughput of `world` replicas: all ranks' gates over the slowest rank's step."""
    ms = reduce_max(ms_per_step_local, world)
    return ms, gates_per_rank * world / (ms / 1e3)


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu_index = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.gpu_index), "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except ValueError:
                continue
            for nm, val in zip(names, r[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


def physical_gpu_index(local_rank):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    ids = [v for v in vis.split(",") if v.strip()]
    if ids and all(v.strip().isdigit() for v in ids) and local_rank < len(ids):
        return int(ids[local_rank])
    return local_rank


# Published single-thread NAND PBS times of the reference (Apple M4 Pro), ms per gate:
# statistics/HasteBoots_Performance.xlsx, sheet "Table 2", cells H5 (BABYBEAR), H6 (GOLDILOCKS), H4 (ZAMA).
PUBLISHED_MS = {0: 28.497, 1: 107.96, 2: 160.18}
PARITY_NOTE = ("bit-exact against the oracle (oracle/hb_oracle.cpp, a C++ restatement of the reference "
               "path); unpinned against the Rust reference itself, which cannot be built here")


def load_json(*parts):
    try:
        return json.load(open(os.path.join(ROOT, *parts)))
    except (OSError, ValueError):
        return None


def cpu_reference(params_id, gates_per_step, steps, warmup, threads):
    """The CPU restatement of the reference path (oracle port) built for this host, one gate per
    host thread. Returns (bootstraps/s, mean step seconds, build description)."""
    from oracle import binding as O
    build = O.use_native_build()
    p = O.preset(params_id)
    keys = O.keygen(p, 0, threads)
    bits = np.random.default_rng(3).integers(0, 2, (2, gates_per_step)).astype(np.uint8)
    c0 = O.encrypt(p, keys.lwe_sk, 0, 0, bits[0])
    c1 = O.encrypt(p, keys.lwe_sk, 0, 1 << 20, bits[1])
    # transform the keys once (Evaluator::new), outside the timed steps
    keys.evaluator(threads)
    times = []
    for s in range(warmup + steps):
        t0 = time.perf_counter()
        out = O.gate(keys, "nand", c0, c1, threads=threads)
        dt = time.perf_counter() - t0
        if s >= warmup:
            times.append(dt)
    m, _ = O.decrypt(p, keys.lwe_sk, out)
    assert (m == 1 - (bits[0] & bits[1])).all()
    return gates_per_step / statistics.mean(times), statistics.mean(times), build


def cpu_figures(preset, value, threads, build):
    """Per-thread cost of the CPU port beside the reference's published single-thread figure."""
    d = {"ms_per_gate_per_thread": threads / value * 1e3, "build": build}
    if preset in PUBLISHED_MS:
        d["published_reference_ms_per_gate"] = PUBLISHED_MS[preset]
        d["published_reference_source"] = ("the reference's single-thread NAND PBS on an Apple M4 Pro, "
                                           "statistics/HasteBoots_Performance.xlsx, Table 2")
    return d


def gates_workload(gates, set_name, p):
    """The workload both arms name: `gates` NAND bootstraps under one parameter set."""
    return (f"{gates} NAND gate bootstraps, {set_name} (N={p.ring_dim}, n={p.lwe_dim}, "
            f"B=2^{p.br_bits}, l={p.br_len}, KS 2^{p.ks_bits} x {p.ks_len})")


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    from oracle import binding as O
    threads = os.cpu_count() or 1
    gates = 4 * threads  # about a second of work per step on the host's cores
    steps, warmup = args.steps, args.warmup
    value, step_s, build = cpu_reference(args.preset, gates, steps, warmup, threads)
    p = O.preset(args.preset)
    line = {
        "metric": METRIC, "value": value, "unit": "bootstraps/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": steps, "warmup": warmup, "ms_per_step": step_s * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64" if p.field_id == O.FIELD_GOLDILOCKS else "u32",
        "data": "synthetic (seed-0 keys, seed-3 uniform input bits)",
        "config": {"workload": gates_workload(args.gates, O.PRESET_NAMES[args.preset], p),
                   "execution": f"a {gates}-gate sample per step, one gate per host thread",
                   "gates_per_step": gates, "parallelism": "one gate per host thread"},
        "cpu_baseline": dict({"value": value, "unit": "bootstraps/s", "cores": threads, "kind": "port",
                              "sample": f"{gates} NAND gates per step over {threads} threads (C++ oracle: "
                                        "the reference's Rust path cannot be built here)"},
                             **cpu_figures(args.preset, value, threads, build)),
        "e2e": {"value": value, "unit": "bootstraps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _timed(stream, fn, reps):
    """Device time of `reps` calls of fn() enqueued on `stream` (CUDA events), in ms."""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def _ivt(params):
    return np.int64 if params.dtype == np.uint64 else np.int32


class KeySets:
    """One context holding seed-0 device keys of BABYBEAR, GOLDILOCKS and ZAMA (presets 0, 1, 2),
    each autotuned: the parameter sets of the mixed-set and serving workloads."""

    def __init__(self):
        from hasteboots_b200 import tfhe
        self.ctx = tfhe.Context(0)
        self.evs, self.tuned = {}, {}
        for pid in (0, 1, 2):
            sk = tfhe.KeyGen.generate_secret_key(tfhe.Parameters.preset(pid), 0)
            ev = tfhe.Evaluator(sk, self.ctx)
            self.evs[pid] = (sk, ev)
            self.tuned[pid] = tfhe.autotune(ev)[:2]

    def close(self):
        for sk, ev in self.evs.values():
            ev.keys.free()
        self.ctx.close()


def leg_mixed(sets, steps, warmup, digests):
    """Config 4: the 64 jobs of the mixed-set plan (hasteboots_b200/workloads.py) in one CUDA graph
    holding one persistent launch per set, beside the same jobs run set by set (one set's graph
    after the other: the back-to-back time the mixed graph must beat or meet)."""
    import torch
    from hasteboots_b200 import tfhe
    from hasteboots_b200 import workloads as W
    from hasteboots_b200._lib import lib
    ctx = sets.ctx
    plan = W.mixed_plan()
    jobs = []
    for job in plan:
        sk, ev = sets.evs[job.preset]
        cs = [torch.from_numpy(sk.encrypt(job.bits[k], job.index0(k)).view(_ivt(sk.params))).cuda()
              for k in range(job.inputs)]
        out = torch.zeros_like(cs[0])
        jobs.append((ev, job.gate, cs[0], cs[1], cs[2] if job.inputs == 3 else None, out))
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream_ptr())
    batch = tfhe.Batch(ctx, jobs)
    info = batch.info()
    for _ in range(warmup):
        batch.launch()
    ctx.synchronize()
    l0 = lib().hb_ctx_launches(ctx.handle)
    with ClockSampler(physical_gpu_index(0)) as clk:
        ms = _timed(stream, batch.launch, steps) / steps
    ctx.synchronize()
    launches = lib().hb_ctx_launches(ctx.handle) - l0
    # digests of every job's outputs, when the committed file holds the whole plan
    ref = digests.get("mixed", {}) if digests else {}
    if not all(str(job.index) in ref for job in plan):
        ref = None
    ok, dig = True, (True if ref else None)
    for job, j in zip(plan, jobs):
        sk = sets.evs[job.preset][0]
        got = j[5].cpu().numpy().view(sk.params.dtype)
        ok = ok and bool((sk.decrypt(got) == job.expected()).all())
        if ref:
            dig = dig and W.digest(got) == ref[str(job.index)]["out"]
    batch.free()
    per_set = {}
    for pid in (0, 1, 2):
        sel = [j for job, j in zip(plan, jobs) if job.preset == pid]
        b = tfhe.Batch(ctx, sel)
        b.launch()
        ctx.synchronize()
        per_set[pid] = {"gates": b.info()["gates"], "ms": _timed(stream, b.launch, steps) / steps}
        b.free()
    b2b = sum(v["ms"] for v in per_set.values())
    names = {0: "BABYBEAR", 1: "GOLDILOCKS", 2: "ZAMA"}
    return {"metric": "mixed-set batched bootstraps/s (one graph launch per step)",
            "value": info["gates"] / (ms / 1e3), "unit": "bootstraps/s", "ms_per_step": ms,
            "steps": steps, "warmup": warmup, "gates": info["gates"], "kernels_per_graph": info["launches"],
            "back_to_back": {"ms": b2b, "value": info["gates"] / (b2b / 1e3),
                             "per_set": {names[k]: v for k, v in per_set.items()},
                             "graph_over_back_to_back": b2b / ms},
            "autotuned_variant": {names[k]: {"threads_per_gate": v[0][0], "gates_per_cta": v[0][1],
                                             "gates_per_s": v[1]} for k, v in sets.tuned.items()},
            "gpu_launches": int(launches), "clocks": clk.summary(),
            "checks": {"truth_tables": ok, "oracle_digest_match": dig, "parity": PARITY_NOTE}}


def leg_ntt(ctx, steps, warmup):
    """Config 2: batched negacyclic NTT->INTT round trip and RLWE x RGSW external product over
    Goldilocks, N in {1024, 2048}, 4096 polynomials (round trip) / 4096 RLWEs (product),
    coefficients uniform in [0, Q) (seed 1), RGSW l = 13 rows at B = 2^5 uniform (seed 2)."""
    import torch
    from hasteboots_b200._lib import check, lib
    stream = torch.cuda.ExternalStream(ctx.stream_ptr())
    Q = 0xFFFFFFFF00000001
    res = {}
    probe = ctypes.c_double()
    check(lib().hb_probe_modmul(ctx.handle, 1, ctypes.byref(probe)), "probe", ctx.handle)
    with ClockSampler(physical_gpu_index(0)) as clk:
        for log_n in (10, 11):
            n = 1 << log_n
            x = (np.random.default_rng(1).integers(0, 2**63, (4096, n), dtype=np.uint64) * 2) % np.uint64(Q)
            dx = torch.from_numpy(x.view(np.int64)).cuda()
            dy = torch.zeros_like(dx)
            torch.cuda.synchronize()
            rt = lambda: check(lib().hb_ntt_roundtrip_device(ctx.handle, 1, log_n, dx.data_ptr(), dy.data_ptr(),
                                                             4096), "rt")
            for _ in range(warmup):
                rt()
            ms = _timed(stream, rt, steps) / steps
            ok = bool((dy.cpu().numpy().view(np.uint64) == x).all())
            mm = 2 * 4096 * (n // 2) * log_n
            res[f"roundtrip_N{n}"] = {"ms": ms, "polys_per_s": 4096 / (ms / 1e3),
                                     "gmodmul_per_s": mm / (ms / 1e3) / 1e9,
                                     "frac_of_modmul_probe": mm / (ms / 1e3) / probe.value,
                                     "hbm_gbs": 2 * 4096 * n * 8 / (ms / 1e3) / 1e9, "exact": ok}
            length, bits = 13, 5
            rgsw = np.random.default_rng(2).integers(0, 2**63, 2 * length * 2 * n, dtype=np.uint64) % np.uint64(Q)
            h = ctypes.c_void_p()
            check(lib().hb_rgsw_upload(ctx.handle, 1, log_n, bits, length, rgsw.ctypes.data_as(ctypes.c_void_p),
                                       ctypes.byref(h)), "rgsw", ctx.handle)
            rl = torch.from_numpy((np.random.default_rng(1).integers(0, 2**63, (4096, 2 * n), dtype=np.uint64)
                                   % np.uint64(Q)).view(np.int64)).cuda()
            ro = torch.zeros_like(rl)
            torch.cuda.synchronize()
            ep = lambda: check(lib().hb_external_product_device(ctx.handle, 1, log_n, bits, length, h,
                                                                rl.data_ptr(), ro.data_ptr(), 4096), "ext")
            for _ in range(warmup):
                ep()
            ms = _timed(stream, ep, steps) / steps
            mm = 4096 * ((2 * length + 2) * (n // 2) * log_n + 4 * length * n)
            res[f"ext_product_N{n}"] = {"ms": ms, "products_per_s": 4096 / (ms / 1e3),
                                       "gmodmul_per_s": mm / (ms / 1e3) / 1e9,
                                       "frac_of_modmul_probe": mm / (ms / 1e3) / probe.value}
            lib().hb_rgsw_free(ctx.handle, h)
    return {"metric": "NTT round trip and RLWE x RGSW external product throughput (Goldilocks)",
            "value": res["ext_product_N1024"]["products_per_s"], "unit": "external products/s (N=1024)",
            "steps": steps, "warmup": warmup, "modmul_probe_g_per_s": probe.value / 1e9,
            "config": {"workload": "4096 polynomials / 4096 RLWEs per launch, N in {1024, 2048}, RGSW l=13 B=2^5"},
            "results": res, "clocks": clk.summary(),
            "checks": {"roundtrips_exact": all(v.get("exact", True) for v in res.values())}}


def leg_serve(sets, duration, rate, drain, max_queue_s):
    """Config 5: Poisson arrivals (seed 5) at `rate` requests/s for `duration` s, each request
    log-uniform 1-4096 NAND gates of a parameter set drawn uniformly from {BABYBEAR, GOLDILOCKS,
    ZAMA}; keys resident; admission against a 120 GB HBM budget; continuous batching. Inputs are
    slices of a pinned per-set pool whose NAND outputs were computed alone beforehand, so every
    served result is checked bit-exact against its alone result."""
    import threading
    import torch
    from hasteboots_b200 import tfhe
    ctx, evs, pools = sets.ctx, sets.evs, {}
    for pid, (sk, ev) in evs.items():
        bits = np.random.default_rng(50 + pid).integers(0, 2, (2, 4096)).astype(np.uint8)
        c0, c1 = sk.encrypt(bits[0], 0), sk.encrypt(bits[1], 1 << 20)
        ivt = _ivt(sk.params)
        p0 = torch.from_numpy(c0.view(ivt).copy()).pin_memory().numpy().view(sk.params.dtype)
        p1 = torch.from_numpy(c1.view(ivt).copy()).pin_memory().numpy().view(sk.params.dtype)
        ref = ev.nand(p0, p1)
        assert (sk.decrypt(ref) == 1 - (bits[0] & bits[1])).all()
        pools[pid] = (p0, p1, ref)
    srv = tfhe.Server(ctx, hbm_budget=120 << 30, max_wave_gates=16384, max_inflight_waves=2,
                      max_queue_s=max_queue_s)
    rng = np.random.default_rng(5)
    arrivals, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        pid = int(rng.integers(0, 3))
        count = int(np.clip(np.round(np.exp(rng.uniform(0, np.log(4096)))), 1, 4096))
        off = int(rng.integers(0, 4096 - count + 1))
        arrivals.append((t, pid, count, off))
    meta, lock = {}, threading.Lock()
    mismatches, fetched, shed = [0], [0], [0]
    stop_fetch = threading.Event()

    def fetcher():
        while not stop_fetch.is_set():
            rid = srv.next_done(0.5)
            if rid is None:
                continue
            with lock:
                pid, off, count = meta[rid]
            out, _ = srv.fetch(rid)
            if not (out == pools[pid][2][off:off + count]).all():
                mismatches[0] += 1
            fetched[0] += 1

    th = threading.Thread(target=fetcher, daemon=True)
    th.start()
    with ClockSampler(physical_gpu_index(0)) as clk:
        t0 = time.perf_counter()
        for (ta, pid, count, off) in arrivals:
            delay = ta - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            p0, p1, _ = pools[pid]
            with lock:  # the fetcher may see the id before submit returns
                rid = srv.submit(evs[pid][1], "nand", p0[off:off + count], p1[off:off + count])
                if rid is None:
                    shed[0] += 1
                    continue
                meta[rid] = (pid, off, count)
        submitted_s = time.perf_counter() - t0
        deadline = time.perf_counter() + drain
        while fetched[0] < len(arrivals) - shed[0] and time.perf_counter() < deadline:
            time.sleep(0.2)
        st = srv.stats()
    stop_fetch.set()
    th.join()
    srv.stop()
    return {"metric": "served bootstraps/s with p50/p99 request latency", "value": st["gates_per_s"],
            "unit": "bootstraps/s", "higher_is_better": True,
            "latency_ms": {"p50": st["p50_latency_s"] * 1e3, "p99": st["p99_latency_s"] * 1e3,
                           "mean": st["mean_latency_s"] * 1e3, "max": st["max_latency_s"] * 1e3},
            "config": {"workload": f"Poisson {rate} req/s for {duration} s, log-uniform 1-4096 NAND "
                                   "gates per request, set uniform over BABYBEAR/GOLDILOCKS/ZAMA",
                       "hbm_budget_gb": 120, "max_wave_gates": 16384, "max_inflight_waves": 2,
                       "drain_s": drain, "max_queue_s": max_queue_s},
            "requests": {"submitted": len(arrivals), "completed": int(st["completed"]),
                         "shed": int(st["rejected"]),
                         "cancelled_at_stop": len(arrivals) - int(st["rejected"]) - int(st["completed"]),
                         "gates_offered": int(sum(a[2] for a in arrivals)),
                         "gates_completed": int(st["gates_completed"]), "waves": int(st["waves"]),
                         "submit_span_s": submitted_s},
            "hbm_peak_gb": st["hbm_peak"] / 2**30, "clocks": clk.summary(),
            "checks": {"served_equals_alone": mismatches[0] == 0, "mismatches": mismatches[0]}}


def leg_single(ctx, sk, ev, steps, warmup):
    """Config 1: latency of one NAND gate through hb_gate_device (the latency form: a cluster of
    CTAs -- 4 for the Goldilocks sets, 2 for the 32-bit fields; one CTA with a ternary LWE key --
    whose thread groups share the gate's digits), with the plain form (one kernel launch of a single
    thread group) beside it."""
    import torch
    from hasteboots_b200._lib import check, lib
    params = sk.params
    c0, c1 = sk.encrypt([1], 0), sk.encrypt([1], 1)  # NAND(1, 1) = 0
    ivt = _ivt(params)
    d0 = torch.from_numpy(c0.view(ivt).copy()).cuda()
    d1 = torch.from_numpy(c1.view(ivt).copy()).cuda()
    do, dp = torch.zeros_like(d0), torch.zeros_like(d0)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream_ptr())
    gate = lambda: check(lib().hb_gate_device(ctx.handle, ev.keys.handle, 0, d0.data_ptr(), d1.data_ptr(), None,
                                              do.data_ptr(), 1), "gate", ctx.handle)
    plain = lambda: check(lib().hb_gate_device_plain(ctx.handle, ev.keys.handle, 0, d0.data_ptr(), d1.data_ptr(),
                                                     dp.data_ptr(), 1), "plain", ctx.handle)
    for _ in range(warmup):
        gate()
        plain()
    with ClockSampler(physical_gpu_index(0)) as clk:
        times = [_timed(stream, gate, 1) for _ in range(steps)]
        ptimes = [_timed(stream, plain, 1) for _ in range(steps)]
    out = do.cpu().numpy().view(params.dtype)
    bit = sk.decrypt(out)[0]
    same = bool((out == dp.cpu().numpy().view(params.dtype)).all())
    return {"metric": "single NAND bootstrap latency, " + params.name.replace("_PARAMETERS", ""),
            "value": float(np.median(times)), "unit": "ms", "higher_is_better": False, "steps": steps,
            "warmup": warmup, "dtype": "u64" if params.dtype == np.uint64 else "u32",
            "latency_ms": {"p50": float(np.percentile(times, 50)), "p99": float(np.percentile(times, 99))},
            "plain_form_ms": {"p50": float(np.percentile(ptimes, 50)), "p99": float(np.percentile(ptimes, 99))},
            "config": {"workload": "1 NAND gate through hb_gate_device (the latency form: the gate's digits "
                                   "over the thread groups of a 4-CTA cluster for the Goldilocks sets, a "
                                   "2-CTA cluster for the 32-bit fields, one CTA with a ternary LWE key); "
                                   "plain form: one launch of one thread group"},
            "clocks": clk.summary(),
            "checks": {"nand(1,1)=0": bool(bit == 0), "equals_plain_form": same}}


def run_workload(args):
    """--workload mixed|ntt|single|serve: one of the other configurations on its own line."""
    from hasteboots_b200 import tfhe
    base = {"n_gpus": 1, "data": "synthetic (seed-0 keys)"}
    if args.workload == "single":
        params = tfhe.Parameters.preset(args.single_preset)
        if args.ternary_lwe_key:
            params = params.with_ternary_lwe_key()
        sk = tfhe.KeyGen.generate_secret_key(params, 0)
        ctx = tfhe.Context(0)
        ev = tfhe.Evaluator(sk, ctx)
        line = leg_single(ctx, sk, ev, args.steps, args.warmup)
        ok = all(line["checks"].values())
        ev.keys.free()
        ctx.close()
    elif args.workload == "ntt":
        ctx = tfhe.Context(0)
        line = leg_ntt(ctx, args.steps, args.warmup)
        ok = line["checks"]["roundtrips_exact"]
        ctx.close()
    else:
        sets = KeySets()
        if args.workload == "mixed":
            line = leg_mixed(sets, args.steps, args.warmup, load_json("tests", "golden", "digests_full.json"))
            ok = line["checks"]["truth_tables"] and line["checks"]["oracle_digest_match"] is not False
        else:
            line = leg_serve(sets, args.duration, args.rate, args.drain, args.max_queue_s)
            ok = line["checks"]["served_equals_alone"]
        sets.close()
    print(json.dumps(dict(base, **line)), flush=True)
    return 0 if ok else 1


def extra_legs(args):
    """The other configurations, measured after the headline in the default run (about a minute):
    config 1 (single BABYBEAR NAND), 2 (NTT / external-product microbench), 4 (the mixed-set graph
    against the same jobs back to back) and 5 (a shortened serving run with load shedding)."""
    legs = {
        "single": lambda: leg_single(sets.ctx, sets.evs[0][0], sets.evs[0][1], 20, 3),
        "ntt_microbench": lambda: leg_ntt(sets.ctx, 5, 2),
        "mixed": lambda: leg_mixed(sets, 2, 1, load_json("tests", "golden", "digests_full.json")),
        "serve": lambda: leg_serve(sets, args.extra_serve_s, 200.0, 10.0, 2.0),
    }
    passed = {
        "single": lambda r: all(r["checks"].values()),
        "ntt_microbench": lambda r: r["checks"]["roundtrips_exact"],
        "mixed": lambda r: r["checks"]["truth_tables"] and r["checks"]["oracle_digest_match"] is not False,
        "serve": lambda r: r["checks"]["served_equals_alone"],
    }
    out, ok = {}, True
    try:
        sets = KeySets()
    except Exception as e:  # the headline line is printed with the error in place of the legs
        return {"extras_error": repr(e)}, False
    for name, leg in legs.items():
        try:
            out[name] = leg()
            ok = ok and bool(passed[name](out[name]))
        except Exception as e:
            out[name] = {"error": repr(e)}
            ok = False
    sets.close()
    return out, ok


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--gates", type=int, default=16384)
    ap.add_argument("--plain-sample", type=int, default=48)
    ap.add_argument("--latency-sample", type=int, default=8)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the other configurations after the headline (single gate, NTT "
                         "microbench, mixed sets, serving)")
    ap.add_argument("--extra-serve-s", type=float, default=15.0, help="seconds of arrivals of the serving leg")
    ap.add_argument("--preset", type=int, default=PRESET,
                    help="0 BABYBEAR, 1 GOLDILOCKS (default, the headline workload), 2 ZAMA, "
                         "3 DEFAULT_TERNARY, 4 CUSTOM_TERNARY")
    ap.add_argument("--single-preset", type=int, default=0,
                    help="single: the parameter set of the one gate (default 0, BABYBEAR)")
    ap.add_argument("--ternary-lwe-key", action="store_true",
                    help="single: a ternary LWE key (DefaultFieldU32 presets 3 and 4 only)")
    ap.add_argument("--workload", default="gates", choices=["gates", "mixed", "ntt", "single", "serve"],
                    help="gates: 16384 NAND gates (default, the contract line); mixed: 64 jobs across "
                         "the three sets in one graph; ntt: NTT/external-product microbench; single: "
                         "one BabyBear NAND; serve: the request loop")
    ap.add_argument("--duration", type=float, default=60.0, help="serve: seconds of arrivals")
    ap.add_argument("--rate", type=float, default=200.0, help="serve: mean requests per second")
    ap.add_argument("--drain", type=float, default=30.0, help="serve: seconds to finish after arrivals")
    ap.add_argument("--max-queue-s", type=float, default=0.0,
                    help="serve: shed requests predicted to complete later than this (0 = FIFO, admit all)")
    ap.add_argument("--variant", default="", help="T,G: use this kernel variant instead of autotuning "
                                                  "(profiling and sweeps)")
    args = ap.parse_args()
    rank, world, local_rank = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload != "gates":
        import torch
        torch.cuda.set_device(local_rank)
        return run_workload(args) if rank == 0 else 0

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local_rank))

    from hasteboots_b200 import tfhe
    from hasteboots_b200 import workloads as W
    from hasteboots_b200._lib import check, lib

    L = lib()
    params = tfhe.Parameters.preset(args.preset)
    raw = params.raw
    G = args.gates
    sk = tfhe.KeyGen.generate_secret_key(params, 0)
    ctx = tfhe.Context(local_rank)
    t0 = time.perf_counter()
    ev = tfhe.Evaluator(sk, ctx)
    setup_s = time.perf_counter() - t0
    bits = W.headline_bits(G, rank)
    c0 = sk.encrypt(bits[0], W.HEADLINE_INDEX0[0])
    c1 = sk.encrypt(bits[1], W.HEADLINE_INDEX0[1])
    width = raw.lwe_dim + 1
    ivt = _ivt(params)
    d0 = torch.from_numpy(c0.view(ivt).copy()).cuda()
    d1 = torch.from_numpy(c1.view(ivt).copy()).cuda()
    dout = torch.zeros_like(d0)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream_ptr())

    def step():
        check(L.hb_gate_device(ctx.handle, ev.keys.handle, GATE_NAND, d0.data_ptr(), d1.data_ptr(),
                               None, dout.data_ptr(), G), "hb_gate_device", ctx.handle)

    if args.variant:
        tuned_t, tuned_g = (int(x) for x in args.variant.split(","))
        check(L.hb_keys_set_config(ctx.handle, ev.keys.handle, tuned_t, tuned_g), "set_config", ctx.handle)
        tuned_rate, tuned_cached = None, None
    else:  # setup, outside the timed region
        (tuned_t, tuned_g), tuned_rate, tuned_cached = tfhe.autotune(ev)
    # roofline denominator: measured field-multiplication throughput of this GPU
    probe = ctypes.c_double()
    check(L.hb_probe_modmul(ctx.handle, raw.field_id, ctypes.byref(probe)), "probe", ctx.handle)

    for _ in range(args.warmup):
        step()
    ctx.synchronize()
    if world > 1:
        dist.barrier()
    launches0 = L.hb_ctx_launches(ctx.handle)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(physical_gpu_index(local_rank)) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        ev1.synchronize()
        ctx.synchronize()
    launches = L.hb_ctx_launches(ctx.handle) - launches0
    ms_per_step, value = aggregate(ev0.elapsed_time(ev1) / args.steps, G, world)

    # correctness of the timed outputs: NAND truth table on every gate, and every output against
    # the oracle's digests where they exist (the default 16384-gate batch of rank 0)
    out = dout.cpu().numpy().view(params.dtype).reshape(G, width)
    m, noise = sk.decrypt_with_noise(out)
    ok = bool((m == W.truth("nand", bits[0], bits[1])).all() and (noise < params.modulus // 16).all())
    digest_ok = None
    digests = load_json("tests", "golden", "digests_full.json")
    ref = digests.get("headline") if digests else None
    if (ref and len(ref.get("out_slices", [])) * ref["slice"] == G and rank == 0
            and args.preset == W.HEADLINE_PRESET and G == W.HEADLINE_GATES):
        digest_ok = bool(W.digest(c0) == ref["c0"] and W.digest(c1) == ref["c1"]
                         and W.slice_digests(out, ref["slice"]) == ref["out_slices"])

    # end to end through the public host API (pinned buffers, copies in the timed region)
    pin0 = torch.from_numpy(c0.view(ivt).copy()).pin_memory()
    pin1 = torch.from_numpy(c1.view(ivt).copy()).pin_memory()
    pout = torch.zeros_like(pin0).pin_memory()
    e2e_times = []
    for s in range(args.e2e_steps + 1 if args.e2e_steps > 0 else 0):
        a0 = time.perf_counter()
        check(L.hb_gate(ctx.handle, ev.keys.handle, GATE_NAND, pin0.data_ptr(), pin1.data_ptr(), None,
                        pout.data_ptr(), G), "hb_gate", ctx.handle)
        if s > 0:
            e2e_times.append(time.perf_counter() - a0)
    if not e2e_times:  # e2e leg disabled (profiling runs): reuse the device outputs
        pout.copy_(torch.from_numpy(out.view(ivt)))
        e2e_times = [float("nan")]
    e2e_s = reduce_max(max(e2e_times), world)
    e2e_ok = bool((pout.numpy().view(params.dtype).reshape(G, width) == out).all())

    # plain one-gate-per-launch form on a sample of the same gates
    P = min(args.plain_sample, G)
    pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pd = torch.zeros_like(d0[:P])
    check(L.hb_gate_device_plain(ctx.handle, ev.keys.handle, GATE_NAND, d0.data_ptr(), d1.data_ptr(),
                                 pd.data_ptr(), 2), "plain warmup", ctx.handle)
    ctx.synchronize()
    pe0.record(stream)
    check(L.hb_gate_device_plain(ctx.handle, ev.keys.handle, GATE_NAND, d0.data_ptr(), d1.data_ptr(),
                                 pd.data_ptr(), P), "plain", ctx.handle)
    pe1.record(stream)
    pe1.synchronize()
    ctx.synchronize()
    plain_rate = P / (pe0.elapsed_time(pe1) / 1e3)
    plain_ok = bool((pd.cpu().numpy().view(params.dtype).reshape(P, width) == out[:P]).all())

    # the latency form, one gate per hb_gate_device call, on a sample of the same gates
    Lg = min(args.latency_sample, G)
    ld = torch.zeros_like(d0[:Lg])
    row = width
    one = lambda i: check(L.hb_gate_device(ctx.handle, ev.keys.handle, GATE_NAND, d0[i:i + 1].data_ptr(),
                                           d1[i:i + 1].data_ptr(), None, ld[i:i + 1].data_ptr(), 1),
                          "latency form", ctx.handle)
    one(0)
    ctx.synchronize()
    lat_ms = [_timed(stream, lambda: one(i), 1) for i in range(Lg)]
    lat_ok = bool((ld.cpu().numpy().view(params.dtype).reshape(Lg, row) == out[:Lg]).all())
    lat_rate = 1e3 / statistics.mean(lat_ms)

    # roofline: integer-pipe bound (modular multiplies), HBM shown alongside
    mm = modmuls_per_gate(raw.ring_dim, raw.lwe_dim, raw.br_len, raw.ks_len, bool(raw.lwe_ternary))
    modmul_launch = mm * G
    achieved = modmul_launch / (ms_per_step / 1e3)
    ws = np.dtype(params.dtype).itemsize
    bsk_bytes = raw.lwe_dim * (2 if raw.lwe_ternary else 1) * 2 * raw.br_len * 2 * raw.ring_dim * ws
    ksk_bytes = raw.ks_len * 2 * raw.ring_dim * ws
    io_bytes = G * 3 * width * ws
    alg_bytes = bsk_bytes + ksk_bytes + io_bytes
    peaks = load_json("MEASURED_PEAKS.json") or {}
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    counters = (load_json("profiles", "bootstrap_goldilocks_nand_counters.json")
                if args.preset == PRESET and G == 16384 else None)
    traffic = counters.get("full_launch") if counters else None
    issue = counters.get("small_case") if counters else None
    set_name = params.name.replace("_PARAMETERS", "")
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "bootstraps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u64" if ws == 8 else "u32",
        "data": "synthetic (seed-0 keys, seed-3 uniform input bits)",
        "config": {
            "workload": gates_workload(G, set_name, raw),
            "execution": "one persistent launch per step",
            "gates_per_gpu": G,
            "parallelism": f"replicas x{world}",
            "l2": f"inputs ({2 * G * width * ws / 1e6:.0f} MB) and BSK ({bsk_bytes / 1e6:.0f} MB) "
                  + ("exceed L2; no flush" if min(2 * G * width * ws, bsk_bytes) > 126e6
                     else "vs 126 MB L2; no flush"),
            "kernel_variant": {"threads_per_gate": tuned_t, "gates_per_cta": tuned_g},
            "autotune": {"gates_per_s_sample": tuned_rate, "from_cache": tuned_cached},
        },
        "latency_ms": {"p50": ms_per_step, "p99": ms_per_step,
                       "note": "every gate of a batched launch completes with the launch"},
        "plain_one_gate_per_launch": {"value": plain_rate, "unit": "bootstraps/s", "sample_gates": P,
                                      "batched_over_plain": value / world / plain_rate,
                                      "latency_form": {"value": lat_rate, "unit": "bootstraps/s",
                                                       "ms_per_gate": statistics.mean(lat_ms),
                                                       "sample_gates": Lg,
                                                       "batched_over_latency_form": value / world / lat_rate}},
        "roofline": {
            "bound": "int",
            "achieved": achieved / 1e9,
            "peak": probe.value / 1e9,
            "unit": "Gmodmul/s",
            "frac": achieved / probe.value,
            "traffic": traffic.get("dram_bytes") if traffic else None,
            "traffic_source": ({k: traffic.get(k) for k in ("kernel", "gpu_time_ms", "command", "source")}
                               if traffic else None),
            "issue": issue,
            "peak_source": "hb_probe_modmul on this GPU, this run (field multiply throughput)",
            "modmul_per_launch": modmul_launch,
            "hbm": {"achieved_gbs": alg_bytes / (ms_per_step / 1e3) / 1e9, "peak_gbs": hbm_peak,
                    "frac": alg_bytes / (ms_per_step / 1e3) / 1e9 / hbm_peak,
                    "algorithmic_bytes_per_launch": alg_bytes,
                    "peak_source": "MEASURED_PEAKS.json" if "hbm_gbs" in peaks else "fallback 6650 GB/s"},
        },
        "e2e": {"value": None if math.isnan(e2e_s) else G * world / e2e_s, "unit": "bootstraps/s",
                "h2d_bytes_per_step": 2 * G * width * ws, "d2h_bytes_per_step": G * width * ws},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "checks": {"nand_truth_table_and_noise": ok, "oracle_digest_match": digest_ok,
                   "e2e_equals_device": e2e_ok, "plain_equals_batched": plain_ok,
                   "latency_form_equals_batched": lat_ok, "parity": PARITY_NOTE},
        "setup_s": setup_s,
    }
    extras_ok = True
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sample = 24 * threads  # several seconds of work on the host's cores
        v, step_s, build = cpu_reference(args.preset, sample, 1, 0, threads)
        line["cpu_baseline"] = dict({"value": v, "unit": "bootstraps/s", "cores": threads, "kind": "port",
                                     "sample": f"{sample} NAND gates over {threads} host threads in {step_s:.1f} s "
                                               "(C++ oracle, keys transformed beforehand as Evaluator::new does)"},
                                    **cpu_figures(args.preset, v, threads, build))
    ev.keys.free()
    ctx.close()
    if rank == 0 and world == 1 and not args.no_extras:
        extra, extras_ok = extra_legs(args)
        line.update(extra)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0 if (ok and digest_ok is not False and e2e_ok and plain_ok and lat_ok and extras_ok) else 1


if __name__ == "__main__":
    sys.exit(main())
