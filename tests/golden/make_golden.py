"""Generate the golden fixtures of this directory by running the reference itself.

Run in a container that has the reference checked out and numba installed,
with ``RBIM_REFERENCE`` naming the reference's checkout (the directory that
holds its ``src/rbim`` and ``tests``)::

    RBIM_REFERENCE=<path to the reference> python tests/golden/make_golden.py [--scan-c1]

It imports the reference package ``rbim`` from ``<reference>/src`` and the
spanning-forest winding oracle from ``<reference>/tests/test_wrapping.py``, and
writes small ``.npz`` fixtures that the test suite compares the oracle and
the CUDA engine against.  Nothing here runs at test time.

Fixtures:
  label_kat.npz      frozen masks (random and Swendsen-Wang-sampled) with the
                     reference union-find's labels, cluster counts and wrap
                     flags, plus the spanning-forest wraps for small L
  label_kat_big.npz  masks of bond probability 1/2 at L = 256, 512, 1024
                     (seeded numpy generator) with n_clusters, wraps, S1, S2
                     and a SHA-1 of the int32 labels
  stats.npz          cluster statistics, two largest, energy, magnetization
  combine.npz        the reference's disorder average and jackknife on
                     synthetic realization results
  scan_small.npz     a full reference temperature scan (statistical parity)
  scan_c1.npz        (--scan-c1) the 32 x 40 x 22k-sweep L = 32 scan
  results_format.npz a scan written by the reference's save_results
"""

from __future__ import annotations

import argparse
import hashlib
import importlib.util
import os
import sys
import tempfile
import time

import numpy as np

REF = os.environ.get("RBIM_REFERENCE")
if not REF or not os.path.isdir(os.path.join(REF, "src", "rbim")):
    raise SystemExit("set RBIM_REFERENCE to the reference checkout (the directory holding src/rbim and tests)")
OUT = os.path.dirname(os.path.abspath(__file__))
os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(tempfile.gettempdir(), "rbim_numba_cache"))
sys.path.insert(0, os.path.join(REF, "src"))

import rbim  # noqa: E402  (the reference package)
from rbim._unionfind import label_and_wrap_unionfind  # noqa: E402
from rbim.clusters import activate_bonds, cluster_statistics  # noqa: E402
from rbim.disorder import generate_disorder  # noqa: E402
from rbim.lattice import build_lattice, couplings_from_disorder  # noqa: E402
from rbim.simulation import (  # noqa: E402
    PRIMITIVES,
    RealizationResult,
    _combine_realizations,
    run_temperature_scan,
    save_results,
)
from rbim.swendsen_wang import _two_largest, energy, magnetization, random_spins, sw_sweep  # noqa: E402


def _load_ref_test(name):
    spec = importlib.util.spec_from_file_location(f"ref_{name}", os.path.join(REF, "tests", f"{name}.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _label_record(L, active, lattice, with_bf, bf):
    n, labels, wx, wy = label_and_wrap_unionfind(active, lattice)
    rec = dict(L=L, n=int(n), wx=bool(wx), wy=bool(wy), labels=labels.astype(np.int32),
               mask=np.packbits(active, bitorder="little"))
    if with_bf:
        bx, by = bf(active, lattice)
        rec["bf"] = (bool(bx), bool(by))
    return rec


def make_label_kat():
    bf = _load_ref_test("test_wrapping").brute_force_winding
    recs = []
    # Random masks of bond probability q.
    for L in (3, 4, 5, 6, 7, 8, 10, 12, 16, 20, 31, 32, 33, 48, 64, 100):
        lattice = build_lattice(L)
        for q in (0.3, 0.5, 0.7):
            for s in range(6 if L <= 32 else 3):
                rng = np.random.default_rng(1000 * L + int(100 * q) + s)
                active = rng.random(2 * L * L) < q
                recs.append(_label_record(L, active, lattice, L <= 16, bf))
    # Masks from Swendsen-Wang configurations (large, multiply connected clusters).
    rng = np.random.default_rng(2024)
    for L in (3, 6, 10, 16, 24):
        lattice = build_lattice(L)
        for p in (0.0, 0.1, 0.5):
            J = couplings_from_disorder(*generate_disorder(L, p, rng))
            for T in (1.0, 2.27, 4.0):
                spins = random_spins(lattice.n_sites, rng)
                for _ in range(3):
                    sw_sweep(spins, lattice, J, 1.0 / T, rng, measure=False)
                    active = activate_bonds(spins, lattice, J, 1.0 / T, rng)
                    recs.append(_label_record(L, active, lattice, L <= 16, bf))
    # Hand-built cases: empty, full, one open column, one closed ring, a
    # cluster that winds only through several seam crossings (a staircase).
    for L in (3, 6, 9):
        lattice = build_lattice(L)
        empty = np.zeros(2 * L * L, bool)
        full = np.ones(2 * L * L, bool)
        column = np.zeros(2 * L * L, bool)
        column[[2 * y + 1 for y in range(L - 1)]] = True
        ring = column.copy()
        ring[2 * (L - 1) + 1] = True
        stair = np.zeros(2 * L * L, bool)
        for x in range(L):
            n = x * L + x
            stair[2 * n] = True                    # (x, x) -> (x+1, x)
            n2 = ((x + 1) % L) * L + x
            stair[2 * n2 + 1] = True               # (x+1, x) -> (x+1, x+1)
        for a in (empty, full, column, ring, stair):
            recs.append(_label_record(L, a, lattice, True, bf))
    Ls = np.array([r["L"] for r in recs], np.int32)
    out = dict(
        L=Ls,
        n_clusters=np.array([r["n"] for r in recs], np.int32),
        wraps=np.array([(r["wx"], r["wy"]) for r in recs], bool),
        bf_wraps=np.array([r.get("bf", (False, False)) for r in recs], bool),
        has_bf=np.array(["bf" in r for r in recs], bool),
        mask_offsets=np.cumsum([0] + [r["mask"].size for r in recs]).astype(np.int64),
        masks=np.concatenate([r["mask"] for r in recs]),
        label_offsets=np.cumsum([0] + [r["labels"].size for r in recs]).astype(np.int64),
        labels=np.concatenate([r["labels"] for r in recs]),
    )
    np.savez_compressed(os.path.join(OUT, "label_kat.npz"), **out)
    print("label_kat:", len(recs), "masks;", int(out["wraps"].any(axis=1).sum()), "wrapping")


def big_mask(L, seed):
    """The mask of the large-lattice KAT: bond probability 1/2 from default_rng(seed)."""
    return np.random.default_rng(seed).random(2 * L * L) < 0.5


def make_label_kat_big(n1024=1000):
    rows = []
    for L, seeds in ((256, range(40)), (512, range(20)), (1024, range(n1024))):
        lattice = build_lattice(L)
        t0 = time.time()
        for s in seeds:
            active = big_mask(L, s)
            n, labels, wx, wy = label_and_wrap_unionfind(active, lattice)
            sizes = np.bincount(labels, minlength=n)
            first, second = _two_largest(sizes)
            s2 = 0 if second is None else int(sizes[second])
            h = hashlib.sha1(labels.astype("<i4").tobytes()).hexdigest()
            rows.append((L, s, int(n), bool(wx), bool(wy), int(sizes[first]), s2, h))
        print(f"label_kat_big L={L}: {len(seeds)} masks, {time.time() - t0:.1f} s")
    np.savez_compressed(
        os.path.join(OUT, "label_kat_big.npz"),
        L=np.array([r[0] for r in rows], np.int32),
        seed=np.array([r[1] for r in rows], np.int64),
        n_clusters=np.array([r[2] for r in rows], np.int64),
        wraps=np.array([(r[3], r[4]) for r in rows], bool),
        s1=np.array([r[5] for r in rows], np.int64),
        s2=np.array([r[6] for r in rows], np.int64),
        sha1=np.array([r[7] for r in rows]),
    )


def make_stats():
    rng = np.random.default_rng(77)
    rows = []
    spins_all, masks_all, J_all = [], [], []
    for L in (3, 5, 8, 12, 16, 32):
        lattice = build_lattice(L)
        for q in (0.2, 0.5, 0.8):
            for _ in range(4):
                J = couplings_from_disorder(*generate_disorder(L, 0.2, rng))
                spins = random_spins(lattice.n_sites, rng)
                active = rng.random(2 * L * L) < q
                n, labels, wx, wy = label_and_wrap_unionfind(active, lattice)
                sizes, mags = cluster_statistics(labels, spins, n)
                first, second = _two_largest(sizes)
                top_tied = bool(n > 1 and np.sum(sizes == sizes[first]) > 1)
                rows.append((L, int(n), int(sizes[first]), abs(float(mags[first])),
                             0 if second is None else int(sizes[second]), energy(spins, lattice, J),
                             magnetization(spins), top_tied))
                spins_all.append(spins.astype(np.int8))
                masks_all.append(np.packbits(active, bitorder="little"))
                J_all.append(J)
    np.savez_compressed(
        os.path.join(OUT, "stats.npz"),
        L=np.array([r[0] for r in rows], np.int32),
        n_clusters=np.array([r[1] for r in rows], np.int64),
        s1=np.array([r[2] for r in rows], np.int64),
        mc1=np.array([r[3] for r in rows], np.float64),
        s2=np.array([r[4] for r in rows], np.int64),
        energy=np.array([r[5] for r in rows], np.float64),
        magnetization=np.array([r[6] for r in rows], np.float64),
        top_tied=np.array([r[7] for r in rows], bool),
        spin_offsets=np.cumsum([0] + [s.size for s in spins_all]).astype(np.int64),
        spins=np.concatenate(spins_all),
        mask_offsets=np.cumsum([0] + [m.size for m in masks_all]).astype(np.int64),
        masks=np.concatenate(masks_all),
        J_offsets=np.cumsum([0] + [j.size for j in J_all]).astype(np.int64),
        J=np.concatenate(J_all),
    )
    print("stats:", len(rows), "cases")


def make_combine():
    rng = np.random.default_rng(5)
    out = {}
    cases = [(8, 10, 2.3, 64), (1, 5, 1.7, 16), (5, 1, 3.0, 36)]
    for ci, (n_r, n_bins, T, N) in enumerate(cases):
        results = []
        prim = np.zeros((n_r, len(PRIMITIVES)))
        bins = np.zeros((n_r, len(PRIMITIVES), n_bins))
        for r in range(n_r):
            b = np.abs(rng.normal(1.0, 0.3, size=(len(PRIMITIVES), n_bins))) * np.arange(1, len(PRIMITIVES) + 1)[:, None]
            b[1] = b[0] ** 2 + np.abs(rng.normal(0, 0.1, n_bins))
            b[4] = b[3] ** 2 + np.abs(rng.normal(0, 0.1, n_bins))
            b[5] = b[4] ** 2 * 1.1
            bins[r] = b
            prim[r] = b.mean(axis=1)
            results.append(RealizationResult(
                primitives={n: float(prim[r, k]) for k, n in enumerate(PRIMITIVES)},
                bin_primitives={n: b[k].copy() for k, n in enumerate(PRIMITIVES)}))
        combined = _combine_realizations(results, T, N)
        names = list(combined)
        out[f"c{ci}_meta"] = np.array([n_r, n_bins, T, N], dtype=np.float64)
        out[f"c{ci}_prim"] = prim
        out[f"c{ci}_bins"] = bins
        out[f"c{ci}_value"] = np.array([combined[n]["value"] for n in names])
        out[f"c{ci}_error"] = np.array([combined[n]["error"] for n in names])
        out[f"c{ci}_thermal"] = np.array([combined[n]["thermal_error"] for n in names])
    out["observables"] = np.array(names)
    np.savez_compressed(os.path.join(OUT, "combine.npz"), **out)
    print("combine:", len(cases), "cases")


def _save_scan(name, res, params):
    flat = {"temperatures": res["temperatures"]}
    for obs, entry in res["observables"].items():
        for key, arr in entry.items():
            flat[f"{obs}__{key}"] = arr
    for k, v in params.items():
        flat[f"param__{k}"] = np.asarray(v)
    np.savez_compressed(os.path.join(OUT, name), **flat)


def make_scan_small(workers):
    params = dict(L=8, p=0.1, n_realizations=16, n_sweeps=4000, n_therm=400, n_bins=10, seed=3)
    temps = np.linspace(1.5, 3.5, 6)
    t0 = time.time()
    res = run_temperature_scan(params["L"], params["p"], temps, n_realizations=params["n_realizations"],
                               n_sweeps=params["n_sweeps"], n_therm=params["n_therm"], n_bins=params["n_bins"],
                               seed=params["seed"], n_workers=workers)
    _save_scan("scan_small.npz", res, dict(params, t_min=1.5, t_max=3.5, n_temps=6))
    print(f"scan_small: {time.time() - t0:.1f} s")
    # p = 0 scan for the Onsager / Coniglio-Klein checks.
    params0 = dict(L=16, p=0.0, n_realizations=4, n_sweeps=8000, n_therm=1000, n_bins=10, seed=11)
    temps0 = np.array([2.0, 2.269185314213022, 3.0])
    res0 = run_temperature_scan(params0["L"], params0["p"], temps0, n_realizations=params0["n_realizations"],
                                n_sweeps=params0["n_sweeps"], n_therm=params0["n_therm"], n_bins=params0["n_bins"],
                                seed=params0["seed"], n_workers=workers)
    _save_scan("scan_pure.npz", res0, params0)
    save_results(os.path.join(OUT, "results_format.npz"), res0)
    print(f"scan_pure + results_format: {time.time() - t0:.1f} s")


def make_scan_c1(workers):
    params = dict(L=32, p=0.05, n_realizations=32, n_sweeps=20000, n_therm=2000, n_bins=20, seed=0)
    temps = np.linspace(1.0, 3.0, 40)
    t0 = time.time()
    res = run_temperature_scan(params["L"], params["p"], temps, n_realizations=params["n_realizations"],
                               n_sweeps=params["n_sweeps"], n_therm=params["n_therm"], n_bins=params["n_bins"],
                               seed=params["seed"], n_workers=workers)
    wall = time.time() - t0
    params["wall_s"] = wall
    params["workers"] = workers
    _save_scan("scan_c1.npz", res, dict(params, t_min=1.0, t_max=3.0, n_temps=40))
    print(f"scan_c1: {wall:.1f} s on {workers} workers")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*", default=None)
    ap.add_argument("--scan-c1", action="store_true")
    ap.add_argument("--workers", type=int, default=os.cpu_count())
    ap.add_argument("--n1024", type=int, default=1000)
    args = ap.parse_args()
    todo = args.only or ["label_kat", "stats", "combine", "scan_small", "label_kat_big"]
    if "label_kat" in todo:
        make_label_kat()
    if "stats" in todo:
        make_stats()
    if "combine" in todo:
        make_combine()
    if "scan_small" in todo:
        make_scan_small(args.workers)
    if "label_kat_big" in todo:
        make_label_kat_big(args.n1024)
    if args.scan_c1:
        make_scan_c1(args.workers)
    print("reference version:", rbim.__version__)


if __name__ == "__main__":
    main()
