#!/usr/bin/env python3
"""Benchmark of the Swendsen-Wang sweep engine (one JSON line on rank 0).

Workload (default ``c4_L256``): the L = 256 slice of the uneven-size
finite-size-scaling configuration -- p in {0.02, 0.05, 0.08, 0.10}, 64
disorder realizations per p (4096 * (32/L)^2 rounded up to 8), 32
temperatures in linspace(1.2, 2.4) -- i.e. 8192 chains of 65,536 sites,
seeded synthetic disorder drawn with the reference's generator.  A step is
``--sweeps-per-step`` measured Swendsen-Wang sweeps of every chain on the
resident (batched) engine; ``value`` is lattice-sweeps per second over all
ranks, device-timed with CUDA events (L2 flushed between steps, outside the
timed region).

Also reported: ``e2e`` (the same metric through the public
``run_temperature_scan``, host disorder generation, copies and the jackknife
included), the plain one-lattice-per-launch engine on the same lattice size,
the roofline of the resident kernel against the measured HBM bandwidth,
clocks sampled during the timed region, and the CPU baseline (the oracle's
C restatement of the reference sweep on the host cores).

``--impl reference`` times only that CPU implementation (rank 0), on the same
metric, with all host threads.
"""

from __future__ import annotations

import argparse
import importlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_SITE_UPDATE = 8.5  # packed spins r+w, packed couplings r, one int32 cluster id w+r
PROFILES = os.path.join(ROOT, "profiles")


def workload(name: str):
    if name == "c4_L256":
        L = 256
        ps = [0.02, 0.05, 0.08, 0.10]
        n_real = int(np.ceil(4096 * (32 / L) ** 2 / 8) * 8)
        temps = np.linspace(1.2, 2.4, 32)
    elif name == "c3_L64":
        L = 64
        ps = [0.05]
        n_real = 256
        temps = np.linspace(1.0, 3.0, 64)
    elif name == "c4_L512":
        L = 512
        ps = [0.02, 0.05, 0.08, 0.10]
        n_real = int(np.ceil(4096 * (32 / L) ** 2 / 8) * 8)
        temps = np.linspace(1.2, 2.4, 32)
    elif name == "c2_L1024":
        L = 1024
        ps = [0.10]
        n_real = 4
        temps = np.linspace(1.5, 1.7, 32)
    else:
        raise SystemExit(f"unknown workload {name}")
    return L, ps, n_real, temps


def build_chains(rb, L, ps, n_real, temps, seed, n_total):
    """Chains (T-major per p, as the reference orders tasks) and packed couplings."""
    specs, couplings = [], []
    for pi, p in enumerate(ps):
        ss = np.random.SeedSequence([seed, pi])
        dseed, rseed = ss.spawn(2)
        drng = np.random.default_rng(dseed)
        base = len(couplings)
        for _ in range(n_real):
            J_h, J_v = rb.generate_disorder(L, p, drng)
            couplings.append(rb.packing.pack_couplings(rb.couplings_from_disorder(J_h, J_v), L))
        kids = rseed.spawn(len(temps) * n_real)
        for k, child in enumerate(kids):
            t_index, r = divmod(k, n_real)
            specs.append(rb.ChainSpec(L=L, realization=base + r, key=rb.chain_key(child), beta=1.0 / temps[t_index],
                                      n_therm=0, n_bins=1, sweeps_per_bin=n_total))
    return specs, couplings


class ClockSampler:
    """nvidia-smi samples (200 ms) of the SM clock and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        mhz, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                mhz.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        if not mhz:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(mhz)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(mhz)}


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(path):
    """DRAM bytes per launch of the workload's kernel from the committed ncu summary, or None."""
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_launch_scaled:"):
                    return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


def profiled_sm_throughput(path):
    """sm__throughput (percent of peak) of the workload's kernel from the committed ncu summary, or None.

    The on-chip engines keep every sweep's state in shared memory, so their
    limit is SM issue and shared-memory latency rather than HBM; this is the
    figure that shows how close the kernel runs to that limit.
    """
    try:
        with open(path) as f:
            for line in f:
                if line.strip().startswith("sm__throughput (pct of peak)"):
                    return float(line.split(")", 1)[1].split("%")[0])
    except (OSError, ValueError):
        pass
    return None


def cpu_baseline(L, temps, ps, seconds=10.0, threads=0):
    """The oracle's restatement of the reference sweep on the host cores: lattice-sweeps/s."""
    import oracle

    n_threads = threads or os.cpu_count() or 1
    rng = np.random.default_rng(0)
    J = np.stack([np.where(rng.random(2 * L * L) < ps[i % len(ps)], -1, 1).astype(np.int8) for i in range(n_threads)])
    keys = np.arange(1, n_threads + 1, dtype=np.uint64)
    thrs = np.array([int(np.floor(-np.expm1(-2.0 / temps[(7 * i) % len(temps)]) * 2**32)) for i in range(n_threads)],
                    dtype=np.uint64)
    # Calibrate: one sweep per chain, then size the sample to ~seconds.
    t0 = time.perf_counter()
    _, _, spins, used = oracle.run_chains(L, J, keys, thrs, n_therm=0, n_bins=1, sweeps_per_bin=1, n_threads=n_threads)
    per = time.perf_counter() - t0
    sweeps = max(1, int(seconds / max(per, 1e-4)))
    t0 = time.perf_counter()
    oracle.run_chains(L, J, keys, thrs, n_therm=0, n_bins=1, sweeps_per_bin=sweeps, spins=spins, n_threads=n_threads)
    dt = time.perf_counter() - t0
    value = n_threads * sweeps / dt
    return {"value": value, "unit": "lattice-sweeps/s", "cores": used, "kind": "port",
            "sample": f"{n_threads} chains of L={L} x {sweeps} measured sweeps, one chain per thread ({dt:.1f} s)"}


def time_sweeps(cs, n, plain=False):
    """Device time of n sweeps of every chain of a ChainSet (CUDA events on the current stream)."""
    import torch

    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    if plain:
        cs.run_plain(n)
    else:
        cs.run_batched(n)
    e1.record()
    e1.synchronize()
    cs.check_status()
    return e0.elapsed_time(e1) / 1000.0


def config_lines(rb, dev, seed):
    """Throughput of the other configurations: batched vs plain at L = 64 (256 realizations x 64 T),
    the L = 512 slice of the uneven-size mix and L = 1024 (cluster engine), one L = 1024 lattice."""
    out = {}

    # The reference's own headline scan (plain method, small): L = 32, p = 0.05, 32 realizations x 40 T,
    # 20,000 measured + 2,000 thermalisation sweeps, 20 bins, end to end through run_temperature_scan.
    import torch

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rb.run_temperature_scan(32, 0.05, np.linspace(1.0, 3.0, 40), n_realizations=32, n_sweeps=20000, n_therm=2000,
                            n_bins=20, seed=0, device=dev, chunk=5000)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    sweeps = 32 * 40 * 22000
    out["c1_L32_scan"] = {"wall_s": wall, "lattice_sweeps_per_s": sweeps / wall,
                          "site_updates_per_s": sweeps * 1024 / wall, "chains": 1280, "sweeps_per_chain": 22000,
                          "api": "run_temperature_scan, host disorder, copies and jackknife included"}

    def chainset(L, p, n_real, temps, n_total, s):
        specs, couplings = build_chains(rb, L, [p], n_real, temps, s, n_total)
        cs = rb.ChainSet(specs, couplings, device=dev)
        cs.init_spins(hot=True)
        return cs, specs, couplings

    # Batched, uniform size: L = 64, p = 0.05, 256 x 64 chains.
    cs, specs, couplings = chainset(64, 0.05, 256, np.linspace(1.0, 3.0, 64), 1000, seed)
    cs.run_batched(3)
    t = time_sweeps(cs, 10)
    b = len(specs) * 10 / t
    pcs = rb.ChainSet(specs[:1], couplings[:1], device=dev)
    pcs.init_spins(hot=True)
    pcs.run_plain(5)
    pt = time_sweeps(pcs, 200, plain=True)
    pv = 200 / pt
    out["c3_L64"] = {"batched_lattice_sweeps_per_s": b, "batched_site_updates_per_s": b * 4096,
                     "plain_lattice_sweeps_per_s": pv, "plain_site_updates_per_s": pv * 4096,
                     "batched_over_plain": b / pv, "chains": len(specs), "engine": "resident"}
    del cs, pcs
    # The L = 512 slice of the uneven-size mix: 16 realizations x 4 p x 32 T.
    specs, couplings = build_chains(rb, 512, [0.02, 0.05, 0.08, 0.10], 16, np.linspace(1.2, 2.4, 32), seed, 1000)
    cs = rb.ChainSet(specs, couplings, device=dev)
    cs.init_spins(hot=True)
    cs.run_batched(1)
    t = time_sweeps(cs, 3)
    b = len(specs) * 3 / t
    pcs = rb.ChainSet(specs[:1], couplings[:1], device=dev)
    pcs.init_spins(hot=True)
    pcs.run_plain(3)
    pv = 50 / time_sweeps(pcs, 50, plain=True)
    out["c4_L512"] = {"batched_lattice_sweeps_per_s": b, "batched_site_updates_per_s": b * 512 * 512,
                      "plain_lattice_sweeps_per_s": pv, "batched_over_plain": b / pv, "chains": len(specs),
                      "engine": "cluster (4 CTAs per lattice)"}
    del cs, pcs
    # L = 1024: one lattice (p = 0.10, T = 1.6) on the plain and the cluster engine, and 128 lattices batched.
    cs, specs, couplings = chainset(1024, 0.10, 4, np.linspace(1.5, 1.7, 32), 1000, seed)
    cs.run_batched(1)
    t = time_sweeps(cs, 3)
    b = len(specs) * 3 / t
    one = rb.ChainSet([rb.ChainSpec(L=1024, realization=0, key=specs[0].key, beta=1 / 1.6, n_therm=0, n_bins=1,
                                    sweeps_per_bin=1000)], couplings[:1], device=dev)
    one.init_spins(hot=True)
    one.run_batched(2)
    ov = 20 / time_sweeps(one, 20)
    one.run_plain(2)
    pv = 20 / time_sweeps(one, 20, plain=True)
    out["c2_L1024"] = {"batched_lattice_sweeps_per_s": b, "batched_site_updates_per_s": b * 1024 * 1024,
                       "one_lattice_cluster_sweeps_per_s": ov, "one_lattice_plain_sweeps_per_s": pv,
                       "batched_over_plain": b / pv, "chains": len(specs), "engine": "cluster (16 CTAs per lattice)"}
    return out


def c4_full_line(rb, dev, seed, sweeps=2):
    """The whole uneven-size configuration in one ChainSet: L in {32, 48, 64, 96, 128, 192, 256, 512},
    p in {0.02, 0.05, 0.08, 0.10}, 4096 (32/L)^2 realizations (rounded up to 8) x 32 temperatures per (L, p);
    one run_batched call advances every lattice (one launch per size bucket)."""
    import torch

    temps = np.linspace(1.2, 2.4, 32)
    ps = [0.02, 0.05, 0.08, 0.10]
    t0 = time.perf_counter()
    specs, couplings = [], []
    for L in (32, 48, 64, 96, 128, 192, 256, 512):
        n_real = int(np.ceil(4096 * (32 / L) ** 2 / 8) * 8)
        sp, cp = build_chains(rb, L, ps, n_real, temps, seed + L, 1000)
        base = len(couplings)
        for s_ in sp:
            s_.realization += base
        specs += sp
        couplings += cp
    cs = rb.ChainSet(specs, couplings, device=dev)
    cs.init_spins(hot=True)
    setup = time.perf_counter() - t0
    sites = float(sum(s_.L * s_.L for s_ in specs))
    cs.run_batched(1)
    t = time_sweeps(cs, sweeps)
    return {"lattices": len(specs), "sites": sites, "sweeps": sweeps, "ms_per_sweep_of_all": 1e3 * t / sweeps,
            "lattice_sweeps_per_s": len(specs) * sweeps / t, "site_updates_per_s": sites * sweeps / t,
            "host_setup_s": setup, "launches_per_sweep": len(cs.buckets)}


def serving_leg(rb, dev, seconds, rate, scale, seed, quantum):
    """Poisson stream of temperature-scan requests (the serving configuration's distribution of L, p,
    temperatures and realizations, sweeps scaled by `scale`) through the continuous-batching server."""
    rng = np.random.default_rng(seed)
    arrivals, reqs, work = [], [], 0
    t = 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > seconds:
            break
        L = int(rng.choice([16, 32, 64, 128, 256, 512]))
        n_t = int(rng.integers(8, 65))
        n_r = int(rng.integers(4, 65))
        sweeps = max(10, int(round(int(rng.integers(1000, 10001)) * scale)))
        req = rb.ScanRequest(L=L, p=float(rng.uniform(0.0, 0.12)), temperatures=np.linspace(1.0, 3.0, n_t),
                             n_realizations=n_r, n_sweeps=sweeps, n_bins=10, seed=int(rng.integers(2**31)))
        arrivals.append(t)
        reqs.append(req)
        work += n_t * n_r * (sweeps + max(1, sweeps // 10)) * L * L
    server = rb.ScanServer(device=dev, memory_bytes=8 << 30, quantum=quantum)
    with server:
        t0 = time.perf_counter()
        futs = []
        for at, req in zip(arrivals, reqs):
            now = time.perf_counter() - t0
            if at > now:
                time.sleep(at - now)
            futs.append(server.submit(req))
        for f in futs:
            f.result()
        t_end = time.perf_counter() - t0
    pct = server.latency_percentiles((50, 99))
    served = sum(c["site_updates"] for c in server.completed)
    return {"p50_s": pct["p50"], "p99_s": pct["p99"], "requests": len(reqs), "arrival_window_s": seconds,
            "rate_per_s": rate, "sweep_scale": scale, "quantum_sweeps": quantum, "wall_s": t_end,
            "offered_site_updates_per_s": work / seconds, "served_site_updates_per_s": served / t_end,
            "launches": server.launches}


def run_reference(args, L, ps, temps, metric):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    values = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(L, temps, ps, seconds=args.ref_seconds)
        if i >= args.warmup:
            values.append(r["value"])
    value = float(np.mean(values))
    line = {
        "metric": metric, "value": value, "unit": "lattice-sweeps/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * args.ref_seconds, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": args.workload, "L": L, "sample": "bounded CPU sample per step"},
        "site_updates_per_s": value * L * L,
        "cpu_baseline": dict(r, value=value),
        "e2e": {"value": value, "unit": "lattice-sweeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--workload", default="c4_L256")
    ap.add_argument("--sweeps-per-step", type=int, default=5)
    ap.add_argument("--threads", type=int, default=0, help="resident CTA size (0 = default)")
    ap.add_argument("--e2e-sweeps", type=int, default=200)
    ap.add_argument("--plain-sweeps", type=int, default=200)
    ap.add_argument("--ref-seconds", type=float, default=3.0)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--chains", type=int, default=0, help="use only the first N chains (profiling runs)")
    ap.add_argument("--no-configs", action="store_true", help="skip the other configurations' lines")
    ap.add_argument("--c4-full", action="store_true",
                    help="also time the whole uneven-size configuration (about 1e6 lattices; slow host setup)")
    ap.add_argument("--serve-seconds", type=float, default=12.0, help="serving leg arrival window (0 = skip)")
    ap.add_argument("--serve-rate", type=float, default=20.0)
    ap.add_argument("--serve-scale", type=float, default=0.004, help="sweeps per request scaled by this factor")
    ap.add_argument("--serve-quantum", type=int, default=10)
    args = ap.parse_args()

    L, ps, n_real, temps = workload(args.workload)
    metric = "L=256 SW sweeps/s batched vs plain on 1 B200 (obs within 2σ); scan p99 latency"
    if args.impl == "reference":
        return run_reference(args, L, ps, temps, metric)

    import torch
    import torch.distributed as dist

    rb = importlib.import_module("rbim-fk-percolation_b200")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    S = args.sweeps_per_step
    n_total = (args.warmup + args.steps) * S + 1
    specs, couplings = build_chains(rb, L, ps, n_real, temps, args.seed + 1000 * rank, n_total)
    if args.chains > 0:
        specs = specs[: args.chains]
    cs = rb.ChainSet(specs, couplings, device=dev)
    cs.init_spins(hot=True)
    n_chains = len(specs)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device=dev)

    for _ in range(args.warmup):
        cs.run_batched(S, threads=args.threads)
    torch.cuda.synchronize()
    cs.check_status()

    stream = torch.cuda.current_stream(dev)
    times = []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            cs.run_batched(S, threads=args.threads)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1) / 1000.0)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    cs.check_status()
    t_local = float(np.sum(times))
    t_max = t_local
    if world > 1:
        t = torch.tensor([t_local], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    sweeps_total = n_chains * S * args.steps * world
    value = sweeps_total / t_max
    launch_s = float(np.mean(times))
    site_updates_launch = n_chains * S * L * L
    peak, peak_kind = measured_peak_hbm()
    achieved = BYTES_PER_SITE_UPDATE * site_updates_launch / launch_s / 1e9
    kernel = "k_resident_sweeps" if L <= rb._native.resident_max_l() else "k_cluster_sweeps"
    traffic = profiled_traffic(os.path.join(PROFILES, f"{kernel}_L{L}.txt"))
    sm_pct = profiled_sm_throughput(os.path.join(PROFILES, f"{kernel}_L{L}.txt"))

    # Plain engine: one lattice per launch sequence, same L.
    plain = None
    if rank == 0 and args.plain_sweeps > 0:
        pspec = rb.ChainSpec(L=L, realization=0, key=99, beta=1 / 1.8, n_therm=0, n_bins=1,
                             sweeps_per_bin=args.plain_sweeps + 20)
        pcs = rb.ChainSet([pspec], [couplings[0]], device=dev)
        pcs.init_spins(hot=True)
        pcs.run_plain(10)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        pcs.run_plain(args.plain_sweeps)
        e1.record(stream)
        e1.synchronize()
        pcs.check_status()
        plain_v = args.plain_sweeps / (e0.elapsed_time(e1) / 1000.0)
        plain = {"value": plain_v, "unit": "lattice-sweeps/s", "engine": "plain (global-memory, per-phase launches)",
                 "batched_over_plain": value / world / plain_v}

    # End to end through the public API: one run_temperature_scan per p per step.
    e2e = None
    if not args.no_e2e:
        E = args.e2e_sweeps
        n_bins = 4
        e2e_steps = max(1, min(3, args.steps))

        def scan_once(i):
            for pi, p in enumerate(ps):
                rb.run_temperature_scan(L, p, temps, n_realizations=n_real, n_sweeps=E, n_therm=E // 10,
                                        n_bins=n_bins, seed=args.seed + 17 * i + pi, device=dev, chunk=E)

        scan_once(-1)
        torch.cuda.synchronize()
        tt = []
        for i in range(e2e_steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            scan_once(i)
            e1.record(stream)
            e1.synchronize()
            tt.append(e0.elapsed_time(e1) / 1000.0)
        t_e = float(np.sum(tt))
        if world > 1:
            t = torch.tensor([t_e], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            t_e = float(t.item())
        lat_sweeps = len(ps) * len(temps) * n_real * (E + E // 10) * e2e_steps * world
        nw = rb.packing.words_for(L)
        h2d = len(ps) * (n_real * 2 * nw * 4 + len(temps) * n_real * (nw * 4 + 96))
        d2h = len(ps) * len(temps) * n_real * n_bins * 14 * 8
        e2e = {"value": lat_sweeps / t_e, "unit": "lattice-sweeps/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "api": "run_temperature_scan (4 calls per step)",
               "sweeps_per_chain": E + E // 10}

    configs = None
    if rank == 0 and not args.no_configs:
        configs = config_lines(rb, dev, args.seed)
    if rank == 0 and args.c4_full:
        configs = dict(configs or {}, c4_full=c4_full_line(rb, dev, args.seed))
    serving = None
    if rank == 0 and args.serve_seconds > 0:
        serving = serving_leg(rb, dev, args.serve_seconds, args.serve_rate, args.serve_scale, args.seed,
                              args.serve_quantum)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(L, temps, ps, seconds=args.cpu_seconds)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": metric,
        "value": value,
        "unit": "lattice-sweeps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1000.0 * t_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int32",
        "data": "synthetic (seeded +-J disorder from the reference's generator)",
        "config": {"workload": args.workload, "L": L, "p": ps, "realizations_per_p": n_real,
                   "temperatures": [float(temps[0]), float(temps[-1]), len(temps)], "chains_per_gpu": n_chains,
                   "sweeps_per_step": S, "measured": True,
                   "engine": "resident (batched)" if kernel == "k_resident_sweeps" else "cluster (batched)",
                   "l2": "flushed between steps (256 MB write)", "parallelism": f"independent chains x{world}"},
        "site_updates_per_s": value * L * L,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                     "bytes_per_site_update": BYTES_PER_SITE_UPDATE, "kernel": kernel,
                     "sm_throughput_pct_of_peak": sm_pct,
                     "sm_throughput_source": f"ncu summary profiles/{kernel}_L{L}.txt" if sm_pct is not None else None},
        "clocks": clocks.summary(),
        "gpu_launches": args.steps,
        "e2e": e2e,
        "plain": plain,
        "serving": serving,
        "configs": configs,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
