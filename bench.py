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
the other configurations (the reference's L = 32 scan, L = 64 batched vs
plain, the L = 512 slice, the whole uneven-size mix with concurrent bucket
launches, one L = 1024 lattice for 2,000 sweeps), a serving load curve with
the same requests run alone for comparison, the roofline of the resident
kernel against the measured HBM bandwidth, clocks sampled during the timed
region, and the CPU baseline (the oracle's C restatement of the reference
sweep on the host cores, on chains of the same workload).

``--impl reference`` times only that CPU implementation (rank 0), on the same
metric, config and chains, with all host threads.
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
METRIC = "L=256 SW sweeps/s batched vs plain on 1 B200 (obs within 2σ); scan p99 latency"
C4_SIZES = (32, 48, 64, 96, 128, 192, 256, 512)
C4_PS = (0.02, 0.05, 0.08, 0.10)


def c4_realizations(L: int) -> int:
    """Realizations per (L, p) of the uneven-size configuration: 4096 (32/L)^2 rounded up to 8."""
    return int(np.ceil(4096 * (32 / L) ** 2 / 8) * 8)


def workload(name: str):
    if name == "c4_L256":
        return 256, list(C4_PS), c4_realizations(256), np.linspace(1.2, 2.4, 32)
    if name == "c3_L64":
        return 64, [0.05], 256, np.linspace(1.0, 3.0, 64)
    if name == "c4_L512":
        return 512, list(C4_PS), c4_realizations(512), np.linspace(1.2, 2.4, 32)
    if name == "c2_L1024":
        return 1024, [0.10], 4, np.linspace(1.5, 1.7, 32)
    raise SystemExit(f"unknown workload {name}")


def workload_config(args, L, ps, n_real, temps):
    """The ``config`` of the JSON line: the workload only, identical for the engine and the reference arm."""
    return {"workload": args.workload, "L": L, "p": list(ps), "realizations_per_p": n_real,
            "temperatures": [float(temps[0]), float(temps[-1]), len(temps)], "chains": len(ps) * n_real * len(temps),
            "sweeps_per_step": args.sweeps_per_step, "measured": True, "seed": args.seed,
            "l2": "flushed between steps (256 MB write)", "parallelism": f"independent chains x{args.gpus}"}


def build_chains(rb, L, ps, n_real, temps, seed, n_total, keep_bonds=False):
    """Chains (T-major per p, as the reference orders tasks), packed couplings and, on request, the bond couplings.

    Per p: ``SeedSequence([seed, p index]).spawn(2)`` gives the disorder and the run seeds; realizations are drawn
    with the reference's generator calls, and chain k's key is that of run-seed child k.
    """
    specs, couplings, bonds = [], [], []
    for pi, p in enumerate(ps):
        dseed, rseed = np.random.SeedSequence([seed, pi]).spawn(2)
        base = len(couplings)
        for J_h, J_v in rb.generate_disorders(L, p, np.random.default_rng(dseed), n_real):
            J = rb.couplings_from_disorder(J_h, J_v)
            couplings.append(rb.packing.pack_couplings(J, L))
            if keep_bonds:
                bonds.append(J)
        keys = rb.seeding.child_keys(rseed, len(temps) * n_real)
        for k in range(len(temps) * n_real):
            t_index, r = divmod(k, n_real)
            specs.append(rb.ChainSpec(L=L, realization=base + r, key=int(keys[k]), beta=1.0 / temps[t_index],
                                      n_therm=0, n_bins=1, sweeps_per_bin=n_total))
    return (specs, couplings, bonds) if keep_bonds else (specs, couplings)


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


def profiled_figure(path, prefix):
    """A figure from a committed ncu summary: the first number after ``prefix`` on its line, or None."""
    try:
        with open(path) as f:
            for line in f:
                if line.strip().startswith(prefix):
                    rest = line.strip()[len(prefix):].lstrip(" :=")
                    return float(rest.split()[0].rstrip("%"))
    except (OSError, ValueError, IndexError):
        pass
    return None


# ---------------------------------------------------------------------------
# CPU baseline: the oracle's restatement of the reference sweep, on chains of the workload itself.
# ---------------------------------------------------------------------------
def cpu_sample(rb, L, ps, n_real, temps, seed, n_chains):
    """``n_chains`` chains of the workload, evenly spread over its (p, temperature, realization) list."""
    specs, _, bonds = build_chains(rb, L, ps, n_real, temps, seed, 1, keep_bonds=True)
    pick = np.linspace(0, len(specs) - 1, n_chains).round().astype(int)
    J = np.stack([bonds[specs[i].realization] for i in pick])
    keys = np.array([specs[i].key for i in pick], dtype=np.uint64)
    thrs = np.array([rb.packing.threshold(specs[i].beta) for i in pick], dtype=np.uint64)
    return J, keys, thrs, [int(i) for i in pick]


def cpu_run(L, sample, sweeps, threads, spins=None):
    """One timed run of ``sweeps`` measured sweeps of every sample chain, one chain per host thread."""
    import oracle

    J, keys, thrs, _ = sample
    t0 = time.perf_counter()
    _, _, spins, used = oracle.run_chains(L, J, keys, thrs, n_therm=0, n_bins=1, sweeps_per_bin=sweeps,
                                          spins=spins, n_threads=threads)
    return time.perf_counter() - t0, spins, used


def cpu_baseline(rb, L, ps, n_real, temps, seed, seconds=10.0, threads=0):
    """Lattice-sweeps/s of the oracle on the host cores (a bounded sample of the workload's chains)."""
    threads = threads or os.cpu_count() or 1
    sample = cpu_sample(rb, L, ps, n_real, temps, seed, threads)
    per, spins, used = cpu_run(L, sample, 1, threads)
    sweeps = max(1, int(seconds / max(per, 1e-4)))
    dt, _, used = cpu_run(L, sample, sweeps, threads, spins)
    value = len(sample[1]) * sweeps / dt
    return {"value": value, "unit": "lattice-sweeps/s", "cores": used, "kind": "port",
            "sample": f"{len(sample[1])} chains of the workload (indices {sample[3][0]}..{sample[3][-1]}, evenly "
                      f"spread over p and T), L={L}, {sweeps} measured sweeps each, one chain per thread "
                      f"({dt:.1f} s)"}


def run_reference(args, L, ps, n_real, temps):
    """The reference arm: the oracle's C sweep on the host cores, on chains of the same workload and config."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    rb = importlib.import_module("rbim-fk-percolation_b200")
    threads = os.cpu_count() or 1
    sample = cpu_sample(rb, L, ps, n_real, temps, args.seed, threads)
    per, spins, used = cpu_run(L, sample, 1, threads)
    sweeps = max(1, int(args.ref_seconds / max(per, 1e-4)))
    times = []
    for i in range(args.warmup + args.steps):
        dt, spins, used = cpu_run(L, sample, sweeps, threads, spins)
        if i >= args.warmup:
            times.append(dt)
    t = float(np.sum(times))
    value = len(sample[1]) * sweeps * args.steps / t
    line = {
        "metric": METRIC, "value": value, "unit": "lattice-sweeps/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * t / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded +-J disorder from the reference's generator)",
        "config": workload_config(args, L, ps, n_real, temps),
        "site_updates_per_s": value * L * L,
        "cpu_baseline": {"value": value, "unit": "lattice-sweeps/s", "cores": used, "kind": "port",
                         "sample": f"each step: {len(sample[1])} chains of the workload (evenly spread over p and T), "
                                   f"{sweeps} measured sweeps each, one chain per host thread"},
        "e2e": {"value": value, "unit": "lattice-sweeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU legs.
# ---------------------------------------------------------------------------
def time_sweeps(cs, n, plain=False, concurrent=True, grid=False):
    """Device time of n sweeps of every chain of a ChainSet (CUDA events on the current stream)."""
    import torch

    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    if grid:
        cs.run_grid(n)
    elif plain:
        cs.run_plain(n)
    else:
        cs.run_batched(n, concurrent=concurrent)
    e1.record()
    e1.synchronize()
    cs.check_status()
    return e0.elapsed_time(e1) / 1000.0


def c2_line(rb, dev, seed, sweeps):
    """One L = 1024 lattice (p = 0.10, T = 1.6) for ``sweeps`` measured sweeps, and the pure model at T_c, on the
    engine ``engine="auto"`` picks for one lattice (the grid engine), device-timed, with E/N and <|m|>; the same
    runs on the plain engine beside it (its launch sequence replayed as a CUDA graph)."""
    out = {}
    L = 1024
    tc = 2.0 / np.log(1.0 + np.sqrt(2.0))
    for name, p, T in (("p0.10_T1.6", 0.10, 1.6), ("p0_Tc", 0.0, tc)):
        specs, couplings = build_chains(rb, L, [p], 1, [T], seed, sweeps)
        assert rb.engine.auto_engine(specs) == "grid"
        res = {}
        for engine in ("grid", "plain"):
            cs = rb.ChainSet(specs, couplings, device=dev)
            cs.init_spins(hot=True)
            if engine == "plain":
                cs.capture_plain(sweeps)  # the launch sequence as a CUDA graph, outside the timed region
            res[engine] = (time_sweeps(cs, sweeps, plain=engine == "plain", grid=engine == "grid"), cs.bins(0)[0])
        t, ib = res["grid"]
        assert np.array_equal(ib, res["plain"][1])  # same chain, same sums on both engines
        n = L * L
        out[name] = {"p": p, "T": float(T), "sweeps": sweeps, "device_s": t, "lattice_sweeps_per_s": sweeps / t,
                     "site_updates_per_s": sweeps * n / t, "us_per_sweep": 1e6 * t / sweeps,
                     "plain_us_per_sweep": 1e6 * res["plain"][0] / sweeps,
                     "grid_over_plain": res["plain"][0] / t,
                     "E_per_site": float(ib[0, 0]) / sweeps / n, "abs_m": float(ib[0, 3]) / sweeps / n,
                     "S1_over_N": float(ib[0, 5]) / sweeps / n}
    out["engine"] = "grid (engine='auto' for one lattice with L > 64: one cooperative launch per call, tiles on every SM)"
    out["note"] = "2,000 measured sweeps from a hot start, no thermalisation excluded; bin sums equal on both engines"
    return out


def config_lines(rb, dev, seed, c2_sweeps):
    """Throughput of the other configurations: the reference's L = 32 scan, batched vs plain at L = 64 (256
    realizations x 64 T), the L = 512 slice of the uneven-size mix and L = 1024 (cluster engine, and one lattice
    for 2,000 sweeps on the plain engine)."""
    import torch

    out = {}
    # The reference's own headline scan (plain method, small): L = 32, p = 0.05, 32 realizations x 40 T,
    # 20,000 measured + 2,000 thermalisation sweeps, 20 bins, end to end through run_temperature_scan.
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

    def chainset(L, ps, n_real, temps, n_total, s):
        specs, couplings = build_chains(rb, L, ps, n_real, temps, s, n_total)
        cs = rb.ChainSet(specs, couplings, device=dev)
        cs.init_spins(hot=True)
        return cs, specs, couplings

    def plain_rate(specs, couplings, n):
        pcs = rb.ChainSet(specs[:1], couplings[:1], device=dev)
        pcs.init_spins(hot=True)
        pcs.run_plain(3)
        pcs.capture_plain(n)
        return n / time_sweeps(pcs, n, plain=True)

    # Batched, uniform size: L = 64, p = 0.05, 256 x 64 chains.
    cs, specs, couplings = chainset(64, [0.05], 256, np.linspace(1.0, 3.0, 64), 1000, seed)
    cs.run_batched(3)
    b = len(specs) * 10 / time_sweeps(cs, 10)
    pv = plain_rate(specs, couplings, 200)
    out["c3_L64"] = {"batched_lattice_sweeps_per_s": b, "batched_site_updates_per_s": b * 4096,
                     "plain_lattice_sweeps_per_s": pv, "plain_site_updates_per_s": pv * 4096,
                     "batched_over_plain": b / pv, "chains": len(specs), "engine": "resident"}
    del cs
    # The L = 512 slice of the uneven-size mix: 16 realizations x 4 p x 32 T.
    cs, specs, couplings = chainset(512, list(C4_PS), 16, np.linspace(1.2, 2.4, 32), 1000, seed)
    cs.run_batched(1)
    b = len(specs) * 3 / time_sweeps(cs, 3)
    pv = plain_rate(specs, couplings, 50)
    out["c4_L512"] = {"batched_lattice_sweeps_per_s": b, "batched_site_updates_per_s": b * 512 * 512,
                      "plain_lattice_sweeps_per_s": pv, "batched_over_plain": b / pv, "chains": len(specs),
                      "engine": "cluster (4 CTAs per lattice)"}
    del cs
    # L = 1024: 128 lattices batched (cluster engine) and one lattice on the cluster engine.
    cs, specs, couplings = chainset(1024, [0.10], 4, np.linspace(1.5, 1.7, 32), 1000, seed)
    cs.run_batched(1)
    b = len(specs) * 3 / time_sweeps(cs, 3)
    one = rb.ChainSet(specs[:1], couplings[:1], device=dev)
    one.init_spins(hot=True)
    one.run_batched(2)
    ov = 20 / time_sweeps(one, 20)
    out["L1024_batched"] = {"batched_lattice_sweeps_per_s": b, "batched_site_updates_per_s": b * 1024 * 1024,
                            "one_lattice_cluster_sweeps_per_s": ov, "chains": len(specs),
                            "engine": "cluster (16 CTAs per lattice)"}
    del cs, one
    # The single-lattice configuration itself: one L = 1024 lattice, 2,000 sweeps.
    out["c2_L1024"] = c2_line(rb, dev, seed, c2_sweeps)
    return out


def c4_full_line(rb, dev, seed, sweeps=2):
    """The whole uneven-size configuration in one ChainSet: L in {32, 48, 64, 96, 128, 192, 256, 512},
    p in {0.02, 0.05, 0.08, 0.10}, 4096 (32/L)^2 realizations (rounded up to 8) x 32 temperatures per (L, p);
    each run_batched call advances every lattice, its bucket launches running concurrently (and, for
    comparison, one after another)."""
    temps = np.linspace(1.2, 2.4, 32)
    t0 = time.perf_counter()
    specs, couplings = [], []
    for L in C4_SIZES:
        sp, cp = build_chains(rb, L, list(C4_PS), c4_realizations(L), temps, seed + L, 1000)
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
    t_conc = min(time_sweeps(cs, sweeps) for _ in range(2))
    t_ser = time_sweeps(cs, sweeps, concurrent=False)
    return {"lattices": len(specs), "sites": sites, "sweeps_per_call": sweeps,
            "ms_per_sweep_of_all": 1e3 * t_conc / sweeps, "lattice_sweeps_per_s": len(specs) * sweeps / t_conc,
            "site_updates_per_s": sites * sweeps / t_conc,
            "serial_launches_ms_per_sweep_of_all": 1e3 * t_ser / sweeps,
            "concurrent_over_serial": t_ser / t_conc, "host_setup_s": setup,
            "launches_per_call": sum(1 for b in cs.buckets if b[0] != 2),
            "launch_mode": "one launch per bucket, all buckets concurrent on forked streams (own queue counters)"}


def serving_requests(rb, seconds, rate, scale, seed):
    """A seeded Poisson stream of scan requests with the serving configuration's distributions of L, p,
    temperatures, realizations and sweeps (sweeps scaled by ``scale``, at least 10)."""
    rng = np.random.default_rng(seed)
    arrivals, reqs, work = [], [], []
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
        work.append(n_t * n_r * (sweeps + max(1, sweeps // 10)) * L * L)
    return arrivals, reqs, work


def serving_point(rb, dev, seconds, rate, scale, seed, quantum):
    """Latency and throughput of one arrival rate through the continuous-batching server."""
    arrivals, reqs, work = serving_requests(rb, seconds, rate, scale, seed)
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
    return {"rate_per_s": rate, "requests": len(reqs), "p50_s": pct["p50"], "p99_s": pct["p99"],
            "offered_site_updates_per_s": sum(work) / seconds, "served_site_updates_per_s": served / t_end,
            "wall_s": t_end, "launches": server.launches}


def serving_leg(rb, dev, args):
    """Serving: a latency-vs-offered-load curve (the spec's request shapes, sweeps scaled by ``--serve-scale``,
    arrival rates up to the spec's 20/s), and the stream's first requests each run alone, one after another,
    through ``run_temperature_scan`` on the plain engine and on the batched engines."""
    import torch

    rates = [float(r) for r in args.serve_rates.split(",") if r]
    curve = [serving_point(rb, dev, args.serve_seconds, r, args.serve_scale, args.seed, args.serve_quantum)
             for r in rates]
    _, reqs, work = serving_requests(rb, args.serve_seconds, max(rates), args.serve_scale, args.seed)
    alone = {}
    sample = list(zip(reqs, work))[: args.serve_alone]
    for engine in ("plain", "batched"):
        t = 0.0
        for req, _ in sample:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rb.run_temperature_scan(req.L, req.p, req.temperatures, n_realizations=req.n_realizations,
                                    n_sweeps=req.n_sweeps, n_bins=req.n_bins, seed=req.seed, device=dev,
                                    engine=engine)
            torch.cuda.synchronize()
            t += time.perf_counter() - t0
        alone[engine] = sum(w for _, w in sample) / t
    top = curve[-1]
    return {"curve": curve, "p50_s": top["p50_s"], "p99_s": top["p99_s"], "rate_per_s": top["rate_per_s"],
            "offered_site_updates_per_s": top["offered_site_updates_per_s"],
            "served_site_updates_per_s": top["served_site_updates_per_s"],
            "alone_plain_site_updates_per_s": alone["plain"], "alone_batched_site_updates_per_s": alone["batched"],
            "alone_sample": f"the stream's first {len(sample)} requests, each run alone through "
                            "run_temperature_scan, one after another (wall clock, disorder and jackknife included)",
            "arrival_window_s": args.serve_seconds, "sweep_scale": args.serve_scale,
            "quantum_sweeps": args.serve_quantum,
            "note": "request shapes follow the serving configuration (L, p, T, realizations); sweeps are scaled so "
                    "that the offered load is near what one B200 serves (unscaled, the stream offers ~7.8e12 "
                    "site-updates/s, far beyond it)"}


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
    ap.add_argument("--ref-seconds", type=float, default=1.5, help="CPU seconds per reference-arm step")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--chains", type=int, default=0, help="use only the first N chains (profiling runs)")
    ap.add_argument("--no-configs", action="store_true", help="skip the other configurations' lines")
    ap.add_argument("--c2-sweeps", type=int, default=2000)
    ap.add_argument("--no-c4-full", action="store_true", help="skip the whole uneven-size configuration (1e6 lattices)")
    ap.add_argument("--serve-seconds", type=float, default=8.0, help="serving arrival window per rate (0 = skip)")
    ap.add_argument("--serve-rates", default="5,10,15,20", help="arrival rates of the serving curve (per s)")
    ap.add_argument("--serve-scale", type=float, default=0.004, help="sweeps per request scaled by this factor")
    ap.add_argument("--serve-quantum", type=int, default=10)
    ap.add_argument("--serve-alone", type=int, default=8, help="requests run alone for the comparison")
    args = ap.parse_args()

    L, ps, n_real, temps = workload(args.workload)
    if args.impl == "reference":
        return run_reference(args, L, ps, n_real, temps)

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
    summary = os.path.join(PROFILES, f"{kernel}_L{L}.txt")
    traffic = profiled_figure(summary, "dram_bytes_per_launch_scaled")
    sm_pct = profiled_figure(summary, "sm__throughput (pct of peak)")
    del cs

    # Plain engine: one lattice per launch sequence, same L.
    plain = None
    if rank == 0 and args.plain_sweeps > 0:
        pspec = rb.ChainSpec(L=L, realization=0, key=99, beta=1 / 1.8, n_therm=0, n_bins=1,
                             sweeps_per_bin=args.plain_sweeps + 20)
        pcs = rb.ChainSet([pspec], [couplings[0]], device=dev)
        pcs.init_spins(hot=True)
        pcs.run_plain(10)
        pcs.capture_plain(args.plain_sweeps)
        torch.cuda.synchronize()
        plain_v = args.plain_sweeps / time_sweeps(pcs, args.plain_sweeps, plain=True)
        gcs = rb.ChainSet([pspec], [couplings[0]], device=dev)
        gcs.init_spins(hot=True)
        gcs.run_grid(10)
        torch.cuda.synchronize()
        grid_v = args.plain_sweeps / time_sweeps(gcs, args.plain_sweeps, grid=True)
        plain = {"value": plain_v, "unit": "lattice-sweeps/s",
                 "engine": "plain (global-memory, 7 launches per sweep replayed as a CUDA graph)",
                 "batched_over_plain": value / world / plain_v,
                 "grid_value": grid_v,
                 "grid_engine": "grid (one cooperative launch per call, the lattice in tiles on every SM)"}

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
        configs = config_lines(rb, dev, args.seed, args.c2_sweeps)
    if rank == 0 and not args.no_c4_full:
        configs = dict(configs or {}, c4_full=c4_full_line(rb, dev, args.seed))
    serving = None
    if rank == 0 and args.serve_seconds > 0:
        serving = serving_leg(rb, dev, args)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(rb, L, ps, n_real, temps, args.seed, seconds=args.cpu_seconds)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC,
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
        "config": workload_config(args, L, ps, n_real, temps),
        "engine": "resident (batched)" if kernel == "k_resident_sweeps" else "cluster (batched)",
        "chains_per_gpu": n_chains,
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
