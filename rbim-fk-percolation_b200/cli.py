#!/usr/bin/env python3
"""Command-line front end of the B200 engine: the reference's scripts on the GPU path.

Subcommands mirror the reference's scripts, with the same options:

  run-sweep               scripts/run_sweep.py: one temperature scan to .npz
  validate-pure-ising     scripts/validate_pure_ising.py: Binder and wrapping crossings at p = 0
  measure-autocorrelation scripts/measure_autocorrelation.py: tau_int of the cluster observables
  generate-disorder       scripts/generate_disorder.py: seeded +-J realizations to .npz

``run-sweep`` takes ``--backend cuda`` (the only backend here; the reference's
numba path stays in the reference) plus ``--engine`` and ``--chunk``.  The
sizes of ``validate-pure-ising`` run as concurrent requests of one scan server.

Usage:  python rbim-fk-percolation_b200/cli.py run-sweep --L 32 --p 0.05 --out results/L32.npz
"""

from __future__ import annotations

import argparse
import glob
import importlib
import itertools
import os
import sys
import time
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np


def _package():
    here = os.path.dirname(os.path.abspath(__file__))
    parent = os.path.dirname(here)
    if parent not in sys.path:
        sys.path.insert(0, parent)
    return importlib.import_module(os.path.basename(here))


TC_EXACT = 2.0 / np.log(1.0 + np.sqrt(2.0))


# --------------------------------------------------------------------------- run-sweep
def _load_disorder_directory(rb, pattern: str, n_realizations: int) -> List[Tuple[np.ndarray, np.ndarray]]:
    paths = sorted(glob.glob(pattern))
    if not paths:
        raise FileNotFoundError(f"no disorder files matched {pattern!r}")
    if len(paths) < n_realizations:
        raise ValueError(f"{len(paths)} disorder files matched {pattern!r} but --realizations={n_realizations}")
    return [rb.load_disorder(path) for path in paths[:n_realizations]]


def run_sweep(args) -> int:
    rb = _package()
    temperatures = np.linspace(args.t_min, args.t_max, args.n_temps)
    disorder = None
    if args.disorder_glob is not None:
        disorder = _load_disorder_directory(rb, args.disorder_glob, args.realizations)
    print(f"L={args.L}  p={args.p}  {args.n_temps} temperatures in [{args.t_min}, {args.t_max}]  "
          f"{args.realizations} realization(s)  {args.sweeps} sweeps  backend={args.backend}")
    t0 = time.time()
    results = rb.run_temperature_scan(args.L, args.p, temperatures, n_realizations=args.realizations,
                                      n_sweeps=args.sweeps, n_therm=args.therm, n_bins=args.bins, seed=args.seed,
                                      n_workers=args.workers, measure_percolation=not args.no_percolation,
                                      start=args.start, disorder=disorder, engine=args.engine, chunk=args.chunk)
    elapsed = time.time() - t0
    rb.save_results(args.out, results)
    print(f"finished in {elapsed:.1f} s; wrote {args.out}")
    if args.realizations == 1:
        print("warning: a single disorder realization was used, so the reported error is "
              "thermal only and does not include sample-to-sample fluctuation.")
    return 0


# --------------------------------------------------------------------------- validate-pure-ising
def crossing(temperatures: np.ndarray, curve_a: np.ndarray, curve_b: np.ndarray) -> Optional[float]:
    """Temperature where two curves intersect (linear interpolation), or None."""
    d = np.asarray(curve_a) - np.asarray(curve_b)
    s = np.sign(d)
    for i in range(len(d) - 1):
        if s[i] == 0:
            return float(temperatures[i])
        if s[i] * s[i + 1] < 0:
            t0, t1 = temperatures[i], temperatures[i + 1]
            return float(t0 - d[i] * (t1 - t0) / (d[i + 1] - d[i]))
    return None


def pairwise_crossings(temperatures: np.ndarray, curves: Dict[int, np.ndarray]) -> List[Tuple[int, int, float]]:
    found = []
    for La, Lb in itertools.combinations(sorted(curves), 2):
        loc = crossing(temperatures, curves[La], curves[Lb])
        if loc is not None:
            found.append((La, Lb, loc))
    return found


def _report(name: str, temperatures: np.ndarray, curves: Dict[int, np.ndarray]) -> Optional[float]:
    found = pairwise_crossings(temperatures, curves)
    print(f"\n{name} crossings")
    if not found:
        print("  none found on this temperature grid")
        return None
    for La, Lb, loc in found:
        print(f"  L={La:3d} vs L={Lb:3d}:  T = {loc:.4f}   ({loc - TC_EXACT:+.4f} from exact)")
    est = float(np.mean([c[2] for c in found]))
    print(f"  mean: T = {est:.4f}   ({est - TC_EXACT:+.4f} from exact, {100 * abs(est - TC_EXACT) / TC_EXACT:.2f}%)")
    return est


def pure_ising_curves(sizes: Sequence[int], temperatures: np.ndarray, sweeps: int, bins: int, seed: int,
                      chunk: int = 500, verbose: bool = False):
    """Binder-cumulant and wrap_y curves of the pure model (p = 0, one realization) for every size.

    Same scans as the reference's ``validate_pure_ising.py:99-113`` (seed ``seed + L`` per size), run as
    concurrent requests of one scan server.  Returns ``(binder, wrapping)``, dicts keyed by L.
    """
    rb = _package()
    binder, wrapping = {}, {}
    with rb.ScanServer(quantum=chunk) as server:
        futs = {L: server.submit(rb.ScanRequest(L=L, p=0.0, temperatures=temperatures, n_realizations=1,
                                                n_sweeps=sweeps, n_bins=bins, seed=seed + L))
                for L in sizes}
        for L, f in futs.items():
            res = f.result()
            binder[L] = res["observables"]["binder"]["value"]
            wrapping[L] = res["observables"]["wrap_y"]["value"]
            if verbose:
                print(f"  L={L:3d} done")
    return binder, wrapping


def validate_pure_ising(args) -> Tuple[Optional[float], Optional[float]]:
    temperatures = np.linspace(args.t_min, args.t_max, args.n_temps)
    print(f"exact T_c = {TC_EXACT:.6f}")
    print(f"sizes {args.sizes}, {args.n_temps} temperatures in [{args.t_min}, {args.t_max}], {args.sweeps} sweeps")
    binder, wrapping = pure_ising_curves(args.sizes, temperatures, args.sweeps, args.bins, args.seed, args.chunk,
                                         verbose=True)
    b = _report("Binder cumulant", temperatures, binder)
    w = _report("FK wrapping probability", temperatures, wrapping)
    if b is not None and w is not None:
        print(f"\nConiglio-Klein check: magnetic and geometric estimates differ by {abs(b - w):.4f}")
    return b, w


# --------------------------------------------------------------------------- measure-autocorrelation
def measure_autocorrelation(args) -> Dict[float, Dict[str, float]]:
    rb = _package()
    from importlib import import_module

    ts = import_module(rb.__name__ + ".timeseries")
    table = {}
    for p in args.p:
        print(f"\n=== L = {args.L}, p = {p} ===")
        header = f"{'T':>6} " + " ".join(f"{name[:16]:>17}" for name in ts.TRACKED)
        print(header)
        print("-" * len(header))
        series = ts.collect_series(args.L, p, args.temperatures, n_sweeps=args.sweeps, n_therm=args.therm,
                                   n_realizations=args.realizations, seed=args.seed)
        for t, T in enumerate(args.temperatures):
            row = f"{T:6.2f} "
            taus = {}
            for name in ts.TRACKED:
                tau = float(np.mean([ts.integrated_autocorrelation(series[name][t, r])[0]
                                     for r in range(args.realizations)]))
                taus[name] = tau
                row += f" {tau:7.1f} ({args.sweeps / (2.0 * tau):6.0f})"
            table[(p, T)] = taus
            print(row)
        print("  values are tau_int (effectively independent measurements in parentheses)")
    return table


# --------------------------------------------------------------------------- generate-disorder
def generate_disorder(args) -> int:
    rb = _package()
    os.makedirs(args.out, exist_ok=True)
    densities = []
    for i, child in enumerate(np.random.SeedSequence(args.seed).spawn(args.realizations)):
        rng = np.random.default_rng(child)
        J_h, J_v = rb.generate_disorder(args.L, args.p, rng)
        densities.append(rb.frustration_density(J_h, J_v))
        rb.save_disorder(os.path.join(args.out, rb.default_disorder_filename(args.L, args.p, i)), J_h, J_v, p=args.p,
                         seed=args.seed)
    expected = 4 * args.p * (1 - args.p) * ((1 - args.p) ** 2 + args.p**2)
    print(f"wrote {args.realizations} realization(s) for L={args.L}, p={args.p} to {args.out}")
    print(f"frustrated plaquette density: {np.mean(densities):.4f} (expected {expected:.4f})")
    return 0


def build_parser() -> argparse.ArgumentParser:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = ap.add_subparsers(dest="cmd", required=True)

    r = sub.add_parser("run-sweep", help="temperature scan to .npz (scripts/run_sweep.py)")
    r.add_argument("--L", type=int, required=True)
    r.add_argument("--p", type=float, required=True)
    r.add_argument("--t-min", type=float, default=1.0)
    r.add_argument("--t-max", type=float, default=3.0)
    r.add_argument("--n-temps", type=int, default=30)
    r.add_argument("--realizations", type=int, default=1)
    r.add_argument("--sweeps", type=int, default=10_000)
    r.add_argument("--therm", type=int, default=None)
    r.add_argument("--bins", type=int, default=10)
    r.add_argument("--seed", type=int, default=0)
    r.add_argument("--workers", type=int, default=None, help="accepted for compatibility; ignored")
    r.add_argument("--no-percolation", action="store_true")
    r.add_argument("--start", choices=["hot", "cold"], default="hot")
    r.add_argument("--disorder-glob", type=str, default=None)
    r.add_argument("--out", type=str, required=True)
    r.add_argument("--backend", choices=["cuda"], default="cuda")
    r.add_argument("--engine", choices=["auto", "batched", "plain", "grid"], default="auto")
    r.add_argument("--chunk", type=int, default=1000, help="sweeps per engine call")
    r.set_defaults(func=run_sweep)

    v = sub.add_parser("validate-pure-ising", help="Binder and wrapping crossings at p = 0")
    v.add_argument("--sizes", type=int, nargs="+", default=[8, 16, 24])
    v.add_argument("--t-min", type=float, default=2.15)
    v.add_argument("--t-max", type=float, default=2.40)
    v.add_argument("--n-temps", type=int, default=11)
    v.add_argument("--sweeps", type=int, default=8000)
    v.add_argument("--bins", type=int, default=10)
    v.add_argument("--seed", type=int, default=0)
    v.add_argument("--workers", type=int, default=None, help="accepted for compatibility; ignored")
    v.add_argument("--chunk", type=int, default=500, help="sweeps per engine launch")
    v.set_defaults(func=validate_pure_ising)

    a = sub.add_parser("measure-autocorrelation", help="integrated autocorrelation times")
    a.add_argument("--L", type=int, default=32)
    a.add_argument("--p", type=float, nargs="+", default=[0.05, 0.20])
    a.add_argument("--temperatures", type=float, nargs="+", default=[2.6, 2.3, 2.1, 1.9, 1.7, 1.5, 1.3, 1.1])
    a.add_argument("--sweeps", type=int, default=20000)
    a.add_argument("--therm", type=int, default=2000)
    a.add_argument("--realizations", type=int, default=4)
    a.add_argument("--seed", type=int, default=0)
    a.set_defaults(func=measure_autocorrelation)

    g = sub.add_parser("generate-disorder", help="seeded +-J realizations to .npz")
    g.add_argument("--L", type=int, required=True)
    g.add_argument("--p", type=float, required=True)
    g.add_argument("--realizations", type=int, default=1)
    g.add_argument("--out", type=str, default="data/disorder")
    g.add_argument("--seed", type=int, default=0)
    g.set_defaults(func=generate_disorder)
    return ap


def main(argv: Optional[Sequence[str]] = None) -> int:
    args = build_parser().parse_args(argv)
    rb = _package()
    try:
        out = args.func(args)
    except rb.RbimError as exc:
        print(f"error: {exc}", file=sys.stderr)
        return 2
    return out if isinstance(out, int) else 0


if __name__ == "__main__":
    sys.exit(main())
