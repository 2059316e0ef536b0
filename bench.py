#!/usr/bin/env python
"""Batched NAND gate bootstrapping throughput on B200.

Workload (the largest single-GPU configuration): 16384 independent NAND gates under
GOLDILOCKS_BINARY_128_BITS_PARAMETERS (N=1024, n=728, B=2^8, l=8, KS base 2^5 x 13) in one
persistent-kernel launch sharing one device-resident BSK/KSK; seed-0 keys, uniformly random input
bit pairs (seed 3). One step = one launch over all gates. Inputs (191 MB) and the BSK (191 MB)
exceed the 126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Prints one JSON line (rank 0). Multi-GPU runs are replicas (every rank bootstraps its own 16384
gates with its own key copy; no collective on the data path; weak scaling).
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


def load_traffic(name):
    path = os.path.join(ROOT, "profiles", name)
    if os.path.exists(path):
        try:
            return json.load(open(path))
        except ValueError:
            return None
    return None


def cpu_reference(params_id, gates_per_step, steps, warmup, threads):
    """The CPU restatement of the reference path (oracle port), one gate per host thread."""
    from oracle import binding as O
    p = O.preset(params_id)
    keys = O.keygen(p, 0, threads)
    bits = np.random.default_rng(3).integers(0, 2, (2, gates_per_step)).astype(np.uint8)
    c0 = O.encrypt(p, keys.lwe_sk, 0, 0, bits[0])
    c1 = O.encrypt(p, keys.lwe_sk, 0, 1 << 20, bits[1])
    # transform the keys once (Evaluator::new), outside the timed steps
    keys.evaluator(threads)
    lib = O.lib()
    times = []
    for s in range(warmup + steps):
        t0 = time.perf_counter()
        out = O.gate(keys, "nand", c0, c1, threads=threads)
        dt = time.perf_counter() - t0
        if s >= warmup:
            times.append(dt)
    m, _ = O.decrypt(p, keys.lwe_sk, out)
    assert (m == 1 - (bits[0] & bits[1])).all()
    return gates_per_step / statistics.mean(times), statistics.mean(times), lib


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
    value, step_s, _ = cpu_reference(args.preset, gates, steps, warmup, threads)
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
        "cpu_baseline": {"value": value, "unit": "bootstraps/s", "cores": threads, "kind": "port",
                         "sample": f"{gates} NAND gates per step over {threads} threads (C++ oracle: the "
                                   "reference's Rust path cannot be built here)"},
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


def workload_mixed(args):
    """64 jobs, gate counts log-uniform in [1, 4096] (seed 4), parameter set drawn uniformly from
    {ZAMA, GOLDILOCKS, BABYBEAR}, random input bits, gate kinds cycling NAND..MAJORITY; one CUDA graph
    per step holding one persistent launch per set, SMs split by autotuned per-set throughput."""
    import torch
    from hasteboots_b200 import tfhe
    from hasteboots_b200._lib import lib
    ctx = tfhe.Context(0)
    evs = {}
    for pid in (0, 1, 2):
        sk = tfhe.KeyGen.generate_secret_key(tfhe.Parameters.preset(pid), 0)
        evs[pid] = (sk, tfhe.Evaluator(sk, ctx))
    tuned = {pid: tfhe.autotune(ev)[:2] for pid, (sk, ev) in evs.items()}
    rng = np.random.default_rng(4)
    names = ["nand", "and", "or", "nor", "xor", "xnor", "majority"]
    jobs, checks = [], []
    for i in range(64):
        pid = int(rng.integers(0, 3))
        count = int(np.clip(np.round(np.exp(rng.uniform(0, np.log(4096)))), 1, 4096))
        gate = names[i % len(names)]
        sk, ev = evs[pid]
        bits = rng.integers(0, 2, (3, count)).astype(np.uint8)
        ivt = np.int64 if sk.params.dtype == np.uint64 else np.int32
        cs = [torch.from_numpy(sk.encrypt(bits[k], (i << 24) + (k << 20)).view(ivt)).cuda() for k in range(3)]
        out = torch.zeros_like(cs[0])
        jobs.append((ev, gate, cs[0], cs[1], cs[2] if gate == "majority" else None, out))
        a, b, c = bits
        checks.append((sk, out, {"nand": 1 - (a & b), "and": a & b, "or": a | b, "nor": 1 - (a | b),
                                 "xor": a ^ b, "xnor": 1 - (a ^ b),
                                 "majority": (a & b) | (b & c) | (a & c)}[gate]))
    torch.cuda.synchronize()
    batch = tfhe.Batch(ctx, jobs)
    info = batch.info()
    stream = torch.cuda.ExternalStream(ctx.stream_ptr())
    for _ in range(args.warmup):
        batch.launch()
    ctx.synchronize()
    l0 = lib().hb_ctx_launches(ctx.handle)
    with ClockSampler(physical_gpu_index(0)) as clk:
        ms = _timed(stream, batch.launch, args.steps)
    ctx.synchronize()
    launches = lib().hb_ctx_launches(ctx.handle) - l0
    ok = all((sk.decrypt(out.cpu().numpy().view(sk.params.dtype)) == exp).all() for sk, out, exp in checks)
    per = ms / args.steps
    line = {"metric": "mixed-set batched bootstraps/s (one graph launch per step)",
            "value": info["gates"] / (per / 1e3), "unit": "bootstraps/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per, "higher_is_better": True,
            "dtype": "u64+u32", "data": "synthetic (seed-0 keys, seed-4 job plan and bits)",
            "config": {"workload": "64 jobs, log-uniform 1-4096 gates, sets uniform over ZAMA/GOLDILOCKS/BABYBEAR",
                       "gates": info["gates"], "kernels_per_graph": info["launches"],
                       "sm_split": info["sm_split"],
                       "autotuned_variant": {str(k): {"threads_per_gate": v[0][0], "gates_per_cta": v[0][1]}
                                             for k, v in tuned.items()},
                       "autotuned_gates_per_s": {str(k): v[1] for k, v in tuned.items()}},
            "gpu_launches": int(launches), "clocks": clk.summary(),
            "checks": {"truth_tables": bool(ok)}}
    print(json.dumps(line), flush=True)
    batch.free()
    for sk, ev in evs.values():
        ev.keys.free()
    ctx.close()
    return 0 if ok else 1


def workload_ntt(args):
    """Kernel microbench: batched negacyclic NTT->INTT round trip and one RLWE x RGSW external
    product over Goldilocks, N in {1024, 2048}, 4096 polynomials (round trip) / 4096 RLWEs (product),
    coefficients uniform in [0, Q) (seed 1), RGSW l = 13 rows at B = 2^5 uniform (seed 2)."""
    import torch
    from hasteboots_b200 import tfhe
    from hasteboots_b200._lib import check, lib
    ctx = tfhe.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr())
    Q = 0xFFFFFFFF00000001
    res = {}
    probe = ctypes.c_double()
    check(lib().hb_probe_modmul(ctx.handle, 1, ctypes.byref(probe)), "probe", ctx.handle)
    for log_n in (10, 11):
        n = 1 << log_n
        x = (np.random.default_rng(1).integers(0, 2**63, (4096, n), dtype=np.uint64) * 2) % np.uint64(Q)
        dx = torch.from_numpy(x.view(np.int64)).cuda()
        dy = torch.zeros_like(dx)
        torch.cuda.synchronize()
        rt = lambda: check(lib().hb_ntt_roundtrip_device(ctx.handle, 1, log_n, dx.data_ptr(), dy.data_ptr(), 4096), "rt")
        for _ in range(args.warmup):
            rt()
        ms = _timed(stream, rt, args.steps) / args.steps
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
        ep = lambda: check(lib().hb_external_product_device(ctx.handle, 1, log_n, bits, length, h, rl.data_ptr(),
                                                            ro.data_ptr(), 4096), "ext")
        for _ in range(args.warmup):
            ep()
        ms = _timed(stream, ep, args.steps) / args.steps
        mm = 4096 * ((2 * length + 2) * (n // 2) * log_n + 4 * length * n)
        res[f"ext_product_N{n}"] = {"ms": ms, "products_per_s": 4096 / (ms / 1e3),
                                   "gmodmul_per_s": mm / (ms / 1e3) / 1e9,
                                   "frac_of_modmul_probe": mm / (ms / 1e3) / probe.value}
        lib().hb_rgsw_free(ctx.handle, h)
    line = {"metric": "NTT round trip and RLWE x RGSW external product throughput (Goldilocks)",
            "value": res["ext_product_N1024"]["products_per_s"], "unit": "external products/s (N=1024)",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "dtype": "u64", "data": "synthetic (seeds 1, 2)", "modmul_probe_g_per_s": probe.value / 1e9,
            "config": {"workload": "4096 polynomials / 4096 RLWEs per launch, N in {1024, 2048}, RGSW l=13 B=2^5"},
            "results": res}
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0 if all(v.get("exact", True) for v in res.values()) else 1


def workload_serve(args):
    """Serving (config 5): Poisson arrivals (seed 5) at --rate requests/s for --duration s, each request
    log-uniform 1-4096 NAND gates of a parameter set drawn uniformly from {ZAMA, GOLDILOCKS, BABYBEAR};
    keys resident; admission against a 120 GB HBM budget; continuous batching. Inputs are slices of a
    pinned per-set pool whose NAND outputs were computed alone beforehand, so every served result is
    checked bit-exact against its alone result."""
    import threading
    import torch
    from hasteboots_b200 import tfhe
    ctx = tfhe.Context(0)
    evs, pools = {}, {}
    for pid in (0, 1, 2):
        sk = tfhe.KeyGen.generate_secret_key(tfhe.Parameters.preset(pid), 0)
        ev = tfhe.Evaluator(sk, ctx)
        tfhe.autotune(ev)
        bits = np.random.default_rng(50 + pid).integers(0, 2, (2, 4096)).astype(np.uint8)
        c0, c1 = sk.encrypt(bits[0], 0), sk.encrypt(bits[1], 1 << 20)
        ivt = np.int64 if sk.params.dtype == np.uint64 else np.int32
        p0 = torch.from_numpy(c0.view(ivt).copy()).pin_memory().numpy().view(sk.params.dtype)
        p1 = torch.from_numpy(c1.view(ivt).copy()).pin_memory().numpy().view(sk.params.dtype)
        ref = ev.nand(p0, p1)
        assert (sk.decrypt(ref) == 1 - (bits[0] & bits[1])).all()
        evs[pid], pools[pid] = (sk, ev), (p0, p1, ref)
    srv = tfhe.Server(ctx, hbm_budget=120 << 30, max_wave_gates=16384, max_inflight_waves=2,
                      max_queue_s=args.max_queue_s)
    rng = np.random.default_rng(5)
    arrivals, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / args.rate)
        if t > args.duration:
            break
        pid = int(rng.integers(0, 3))
        count = int(np.clip(np.round(np.exp(rng.uniform(0, np.log(4096)))), 1, 4096))
        off = int(rng.integers(0, 4096 - count + 1))
        arrivals.append((t, pid, count, off))
    meta, lock = {}, threading.Lock()
    mismatches = [0]
    fetched = [0]
    shed = [0]
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
        deadline = time.perf_counter() + args.drain
        while fetched[0] < len(arrivals) - shed[0] and time.perf_counter() < deadline:
            time.sleep(0.2)
        st = srv.stats()
    stop_fetch.set()
    th.join()
    srv.stop()
    line = {"metric": "served bootstraps/s with p50/p99 request latency", "value": st["gates_per_s"],
            "unit": "bootstraps/s", "higher_is_better": True, "n_gpus": 1, "dtype": "u64+u32",
            "data": "synthetic (seed-0 keys, seed-5 Poisson arrivals)",
            "latency_ms": {"p50": st["p50_latency_s"] * 1e3, "p99": st["p99_latency_s"] * 1e3,
                           "mean": st["mean_latency_s"] * 1e3, "max": st["max_latency_s"] * 1e3},
            "config": {"workload": f"Poisson {args.rate} req/s for {args.duration} s, log-uniform 1-4096 NAND "
                                   "gates per request, set uniform over ZAMA/GOLDILOCKS/BABYBEAR",
                       "hbm_budget_gb": 120, "max_wave_gates": 16384, "max_inflight_waves": 2,
                       "drain_s": args.drain, "max_queue_s": args.max_queue_s},
            "requests": {"submitted": len(arrivals), "completed": int(st["completed"]),
                         "shed": int(st["rejected"]),
                         "cancelled_at_stop": len(arrivals) - int(st["rejected"]) - int(st["completed"]),
                         "gates_offered": int(sum(a[2] for a in arrivals)),
                         "gates_completed": int(st["gates_completed"]), "waves": int(st["waves"]),
                         "submit_span_s": submitted_s},
            "hbm_peak_gb": st["hbm_peak"] / 2**30, "clocks": clk.summary(),
            "checks": {"served_equals_alone": mismatches[0] == 0, "mismatches": mismatches[0]}}
    print(json.dumps(line), flush=True)
    for sk, ev in evs.values():
        ev.keys.free()
    ctx.close()
    return 0 if mismatches[0] == 0 else 1


def workload_single(args):
    """One NAND gate (config 1: BABYBEAR_BINARY_128_BITS; --single-preset picks another set):
    latency of one hb_gate_device call (the latency form: one CTA -- for the Goldilocks sets a
    cluster of CTAs -- whose thread groups share the gate's digits), with the plain form (one kernel
    launch of a single thread group) beside it."""
    import torch
    from hasteboots_b200 import tfhe
    from hasteboots_b200._lib import check, lib
    params = tfhe.Parameters.preset(args.single_preset)
    sk = tfhe.KeyGen.generate_secret_key(params, 0)
    ctx = tfhe.Context(0)
    ev = tfhe.Evaluator(sk, ctx)
    c0, c1 = sk.encrypt([1], 0), sk.encrypt([1], 1)
    ivt = np.int64 if params.dtype == np.uint64 else np.int32
    d0 = torch.from_numpy(c0.view(ivt).copy()).cuda()
    d1 = torch.from_numpy(c1.view(ivt).copy()).cuda()
    do = torch.zeros_like(d0)
    dp = torch.zeros_like(d0)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream_ptr())
    gate = lambda: check(lib().hb_gate_device(ctx.handle, ev.keys.handle, 0, d0.data_ptr(), d1.data_ptr(), None,
                                              do.data_ptr(), 1), "gate", ctx.handle)
    plain = lambda: check(lib().hb_gate_device_plain(ctx.handle, ev.keys.handle, 0, d0.data_ptr(), d1.data_ptr(),
                                                     dp.data_ptr(), 1), "plain", ctx.handle)
    for _ in range(args.warmup):
        gate()
        plain()
    times = [_timed(stream, gate, 1) for _ in range(args.steps)]
    ptimes = [_timed(stream, plain, 1) for _ in range(args.steps)]
    out = do.cpu().numpy().view(params.dtype)
    bit = sk.decrypt(out)[0]
    same = bool((out == dp.cpu().numpy().view(params.dtype)).all())
    line = {"metric": "single NAND bootstrap latency, " + params.name.replace("_PARAMETERS", ""),
            "value": float(np.median(times)),
            "unit": "ms", "higher_is_better": False, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "dtype": "u64" if params.dtype == np.uint64 else "u32",
            "data": "synthetic (seed-0 keys)",
            "latency_ms": {"p50": float(np.percentile(times, 50)), "p99": float(np.percentile(times, 99))},
            "plain_form_ms": {"p50": float(np.percentile(ptimes, 50)), "p99": float(np.percentile(ptimes, 99))},
            "config": {"workload": "1 NAND gate through hb_gate_device (the latency form: the gate's digits "
                                   "over the thread groups of one CTA, or of a 4-CTA cluster for the "
                                   "Goldilocks sets); plain form: one launch of one thread group"},
            "checks": {"nand(1,1)=0": bool(bit == 0), "equals_plain_form": same}}
    print(json.dumps(line), flush=True)
    ev.keys.free()
    ctx.close()
    return 0 if (bit == 0 and same) else 1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--gates", type=int, default=16384)
    ap.add_argument("--plain-sample", type=int, default=48)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--preset", type=int, default=PRESET,
                    help="0 BABYBEAR, 1 GOLDILOCKS (default, the headline workload), 2 ZAMA, "
                         "3 DEFAULT_TERNARY, 4 CUSTOM_TERNARY")
    ap.add_argument("--single-preset", type=int, default=0,
                    help="single: the parameter set of the one gate (default 0, BABYBEAR)")
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
        fn = {"mixed": workload_mixed, "ntt": workload_ntt, "single": workload_single,
              "serve": workload_serve}[args.workload]
        return fn(args) if rank == 0 else 0

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local_rank))

    from hasteboots_b200 import tfhe
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
    bits = np.random.default_rng(3 + rank).integers(0, 2, (2, G)).astype(np.uint8)
    c0 = sk.encrypt(bits[0], 0)
    c1 = sk.encrypt(bits[1], 1 << 20)
    width = raw.lwe_dim + 1
    ivt = np.int64 if params.dtype == np.uint64 else np.int32
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

    # correctness of the timed outputs: NAND truth table on every gate
    out = dout.cpu().numpy().view(params.dtype).reshape(G, width)
    m, noise = sk.decrypt_with_noise(out)
    ok = bool((m == 1 - (bits[0] & bits[1])).all() and (noise < params.modulus // 16).all())

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

    # roofline: integer-pipe bound (modular multiplies), HBM shown alongside
    mm = modmuls_per_gate(raw.ring_dim, raw.lwe_dim, raw.br_len, raw.ks_len, bool(raw.lwe_ternary))
    modmul_launch = mm * G
    achieved = modmul_launch / (ms_per_step / 1e3)
    ws = np.dtype(params.dtype).itemsize
    bsk_bytes = raw.lwe_dim * (2 if raw.lwe_ternary else 1) * 2 * raw.br_len * 2 * raw.ring_dim * ws
    ksk_bytes = raw.ks_len * 2 * raw.ring_dim * ws
    io_bytes = G * 3 * width * ws
    alg_bytes = bsk_bytes + ksk_bytes + io_bytes
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    traffic = load_traffic("bootstrap_goldilocks_nand_traffic.json") if args.preset == PRESET else None
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
                                      "batched_over_plain": value / world / plain_rate},
        "roofline": {
            "bound": "int",
            "achieved": achieved / 1e9,
            "peak": probe.value / 1e9,
            "unit": "Gmodmul/s",
            "frac": achieved / probe.value,
            "traffic": traffic.get("dram_bytes_per_launch") if traffic else None,
            "peak_source": "hb_probe_modmul on this GPU, this run (field multiply throughput)",
            "modmul_per_launch": modmul_launch,
            "hbm": {"achieved_gbs": alg_bytes / (ms_per_step / 1e3) / 1e9, "peak_gbs": hbm_peak,
                    "frac": alg_bytes / (ms_per_step / 1e3) / 1e9 / hbm_peak,
                    "algorithmic_bytes_per_launch": alg_bytes, "peak_source": "MEASURED_PEAKS.json"},
        },
        "e2e": {"value": None if math.isnan(e2e_s) else G * world / e2e_s, "unit": "bootstraps/s",
                "h2d_bytes_per_step": 2 * G * width * ws, "d2h_bytes_per_step": G * width * ws},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "checks": {"nand_truth_table_and_noise": ok, "e2e_equals_device": e2e_ok,
                   "plain_equals_batched": plain_ok},
        "setup_s": setup_s,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sample = 24 * threads  # several seconds of work on the host's cores
        v, step_s, _ = cpu_reference(args.preset, sample, 1, 0, threads)
        line["cpu_baseline"] = {"value": v, "unit": "bootstraps/s", "cores": threads, "kind": "port",
                                "sample": f"{sample} NAND gates over {threads} host threads in {step_s:.1f} s "
                                          "(C++ oracle, keys transformed beforehand as Evaluator::new does)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ev.keys.free()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0 if (ok and e2e_ok and plain_ok) else 1


if __name__ == "__main__":
    sys.exit(main())
