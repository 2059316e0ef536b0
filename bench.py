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


def modmuls_per_gate(N, n, length, ks_len):
    """Algorithmic modular multiplications of one bootstrap: n steps of (2l+2) size-N NTTs plus the
    4lN-term multiply-accumulate, and key switching's (l_ks+2) NTTs plus 2 l_ks N products."""
    logn = N.bit_length() - 1
    ntt = (N // 2) * logn
    return n * ((2 * length + 2) * ntt + 4 * length * N) + ((ks_len + 2) * ntt + 2 * ks_len * N)


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


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    gates = threads
    steps, warmup = args.steps, max(1, min(args.warmup, 1))
    value, step_s, _ = cpu_reference(PRESET, gates, steps, warmup, threads)
    line = {
        "metric": METRIC, "value": value, "unit": "bootstraps/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": steps, "warmup": warmup, "ms_per_step": step_s * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (seed-0 keys, seed-3 uniform input bits)",
        "config": {"workload": "NAND bootstrap, GOLDILOCKS_BINARY_128_BITS (N=1024, n=728, B=2^8, l=8)",
                   "gates_per_step": gates, "parallelism": "one gate per host thread"},
        "cpu_baseline": {"value": value, "unit": "bootstraps/s", "cores": threads, "kind": "port",
                         "sample": f"{gates} NAND gates per step over {threads} threads (C++ oracle: the "
                                   "reference's Rust path cannot be built here)"},
        "e2e": {"value": value, "unit": "bootstraps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


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
                    help="0 BABYBEAR, 1 GOLDILOCKS (default, the headline workload), 2 ZAMA")
    args = ap.parse_args()
    rank, world, local_rank = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)

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
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / args.steps
    value = G * world / (ms_per_step / 1e3)

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
    e2e_s = max(e2e_times)
    if world > 1:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
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
    mm = modmuls_per_gate(raw.ring_dim, raw.lwe_dim, raw.br_len, raw.ks_len)
    modmul_launch = mm * G
    achieved = modmul_launch / (ms_per_step / 1e3)
    ws = np.dtype(params.dtype).itemsize
    bsk_bytes = raw.lwe_dim * 2 * raw.br_len * 2 * raw.ring_dim * ws
    ksk_bytes = raw.ks_len * 2 * raw.ring_dim * ws
    io_bytes = G * 3 * width * ws
    alg_bytes = bsk_bytes + ksk_bytes + io_bytes
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    traffic = load_traffic("bootstrap_goldilocks_nand_traffic.json")
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
        "dtype": "u64",
        "data": "synthetic (seed-0 keys, seed-3 uniform input bits)",
        "config": {
            "workload": f"{G} NAND gate bootstraps, GOLDILOCKS_BINARY_128_BITS (N=1024, n=728, B=2^8, l=8, "
                        "KS 2^5 x 13), one persistent launch per step",
            "gates_per_gpu": G,
            "parallelism": f"replicas x{world}",
            "l2": "inputs (191 MB) and BSK (191 MB) exceed L2; no flush",
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
        "e2e": {"value": G * world / e2e_s, "unit": "bootstraps/s",
                "h2d_bytes_per_step": 2 * G * width * ws, "d2h_bytes_per_step": G * width * ws},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "checks": {"nand_truth_table_and_noise": ok, "e2e_equals_device": e2e_ok,
                   "plain_equals_batched": plain_ok},
        "setup_s": setup_s,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, step_s, _ = cpu_reference(PRESET, threads, 1, 0, threads)
        line["cpu_baseline"] = {"value": v, "unit": "bootstraps/s", "cores": threads, "kind": "port",
                                "sample": f"{threads} NAND gates, one per host thread (C++ oracle)"}
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
