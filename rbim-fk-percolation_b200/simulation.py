"""Temperature scans on the GPU engine, with the reference's estimators and file format.

Mirror of the reference's ``src/rbim/simulation.py``: the same ``PRIMITIVES``
and ``OBSERVABLES``, the same ``derive_observables`` conventions, the same
disorder average with jackknife ``error`` and bin-based ``thermal_error``, and
the same ``.npz`` result format.  What changes is below the task boundary:
instead of one OS process per ``(T, realization)`` task running
``run_single_realization`` (``simulation.py:245-258, 395-399``), every task
becomes a chain of one device-resident :class:`~.engine.ChainSet`, all chains
advance together on the B200, and only per-bin sums come back.
"""

from __future__ import annotations

import json
import os
from dataclasses import dataclass, field
from typing import Dict, Iterable, Optional, Sequence

import numpy as np

from .disorder import generate_disorders
from .engine import ChainSet, ChainSpec, chain_key
from .lattice import couplings_from_disorder
from .packing import pack_couplings
from .seeding import child_keys

__all__ = [
    "OBSERVABLES",
    "PRIMITIVES",
    "RealizationResult",
    "derive_observables",
    "realization_from_sums",
    "combine_realizations",
    "run_single_realization",
    "run_temperature_scan",
    "ScanPlan",
    "plan_temperature_scan",
    "run_scan_tasks",
    "assemble_scan",
    "save_results",
    "load_results",
]

#: Per-sweep primitives accumulated over each run (reference ``simulation.py:56-71``).
PRIMITIVES = (
    "energy",
    "energy_sq",
    "magnetization",
    "abs_magnetization",
    "magnetization_sq",
    "magnetization_4",
    "largest_size",
    "largest_abs_mag",
    "second_size",
    "mag_ratio",
    "n_clusters",
    "wrap_x",
    "wrap_y",
    "wrap_any",
)

#: Reported observables, in the reference's order (``simulation.py:74-91``).
OBSERVABLES = (
    "energy",
    "specific_heat",
    "magnetization",
    "abs_magnetization",
    "susceptibility",
    "binder",
    "p_infinity",
    "largest_size",
    "largest_abs_magnetization",
    "cluster_magnetization_ratio",
    "second_size_fraction",
    "cluster_density_gap",
    "n_clusters_per_site",
    "wrap_x",
    "wrap_y",
    "wrap_any",
)

# Where each primitive lives in the engine's accumulator rows: ("i", k) for the
# int64 sums (E, E^2, M, |M|, M^2, S1, |M_C1|, S2, n_clusters, wx, wy, wany),
# ("f", k) for the double sums (M^4, |M_C1|/S1).
_SOURCE = {
    "energy": ("i", 0),
    "energy_sq": ("i", 1),
    "magnetization": ("i", 2),
    "abs_magnetization": ("i", 3),
    "magnetization_sq": ("i", 4),
    "magnetization_4": ("f", 0),
    "largest_size": ("i", 5),
    "largest_abs_mag": ("i", 6),
    "second_size": ("i", 7),
    "mag_ratio": ("f", 1),
    "n_clusters": ("i", 8),
    "wrap_x": ("i", 9),
    "wrap_y": ("i", 10),
    "wrap_any": ("i", 11),
}


@dataclass
class RealizationResult:
    """Full-run mean of each primitive plus per-bin means (reference ``simulation.py:94-105``)."""

    primitives: Dict[str, float]
    bin_primitives: Dict[str, np.ndarray] = field(default_factory=dict)


def derive_observables(primitives, temperature: float, n_sites: int):
    """Physical observables from (disorder-averaged) primitive moments.

    Conventions of the reference (``simulation.py:108-145``): specific heat
    ``[<E^2> - <E>^2] / (T^2 N)``, susceptibility ``[<M^2> - <|M|>^2] / (T N)``,
    Binder ``1 - [<m^4>] / (3 [<m^2>]^2)`` (0 when ``<m^2> = 0``).  Works on
    scalars and, elementwise, on numpy arrays of primitives.
    """
    N = n_sites
    p = primitives
    energy_var = p["energy_sq"] - p["energy"] ** 2
    abs_mag_var = p["magnetization_sq"] - p["abs_magnetization"] ** 2
    m2 = p["magnetization_sq"] / N**2
    m4 = p["magnetization_4"] / N**4
    if np.ndim(m2) == 0:
        binder = 1.0 - m4 / (3.0 * m2**2) if m2 > 0.0 else 0.0
    else:
        with np.errstate(divide="ignore", invalid="ignore"):
            binder = np.where(m2 > 0.0, 1.0 - m4 / (3.0 * np.where(m2 > 0.0, m2, 1.0) ** 2), 0.0)
    return {
        "energy": p["energy"] / N,
        "specific_heat": energy_var / (temperature**2 * N),
        "magnetization": p["magnetization"] / N,
        "abs_magnetization": p["abs_magnetization"] / N,
        "susceptibility": abs_mag_var / (temperature * N),
        "binder": binder,
        "p_infinity": p["largest_size"] / N,
        "largest_size": p["largest_size"],
        "largest_abs_magnetization": p["largest_abs_mag"],
        "cluster_magnetization_ratio": p["mag_ratio"],
        "second_size_fraction": p["second_size"] / N,
        "cluster_density_gap": (p["largest_size"] - p["second_size"]) / N,
        "n_clusters_per_site": p["n_clusters"] / N,
        "wrap_x": p["wrap_x"],
        "wrap_y": p["wrap_y"],
        "wrap_any": p["wrap_any"],
    }


def realization_from_sums(int_bins: np.ndarray, f_bins: np.ndarray, sweeps_per_bin: int,
                          measure_percolation: bool = True) -> RealizationResult:
    """Turn one chain's per-bin sums into the reference's ``RealizationResult``.

    Full-run means are exact integer sums divided once (the reference averages
    the float series, ``simulation.py:238-241``); the wrap primitives are NaN
    when percolation is not measured (``simulation.py:233-236``).
    """
    n_bins = int_bins.shape[0]
    total = n_bins * sweeps_per_bin
    prim: Dict[str, float] = {}
    bins: Dict[str, np.ndarray] = {}
    for name in PRIMITIVES:
        kind, k = _SOURCE[name]
        if not measure_percolation and name.startswith("wrap"):
            prim[name] = float("nan")
            bins[name] = np.full(n_bins, np.nan)
            continue
        if kind == "i":
            col = int_bins[:, k]
            prim[name] = float(sum(int(v) for v in col)) / total
            bins[name] = col.astype(np.float64) / sweeps_per_bin
        else:
            col = f_bins[:, k]
            prim[name] = float(col.sum()) / total
            bins[name] = col / sweeps_per_bin
    return RealizationResult(primitives=prim, bin_primitives=bins)


def combine_realizations(results: Sequence[RealizationResult], temperature: float, n_sites: int):
    """Disorder average with jackknife ``error`` and bin-based ``thermal_error``.

    Same estimator as the reference's ``_combine_realizations``
    (``simulation.py:261-333``): central values from disorder-averaged
    primitives; leave-one-out jackknife over realizations applied to the
    derived observables; thermal error = per-realization standard error across
    bins, combined in quadrature; with one realization the thermal error stands
    in for the disorder error.  Vectorised over realizations.
    """
    n_r = len(results)
    stacked = {name: np.array([r.primitives[name] for r in results], dtype=float) for name in PRIMITIVES}
    mean_prim = {name: float(v.mean()) for name, v in stacked.items()}
    central = derive_observables(mean_prim, temperature, n_sites)
    combined: Dict[str, Dict[str, float]] = {}
    if n_r > 1:
        loo = {name: (v.sum() - v) / (n_r - 1) for name, v in stacked.items()}
        derived = derive_observables(loo, temperature, n_sites)
        factor = (n_r - 1) / n_r
        for name in OBSERVABLES:
            samples = np.asarray(derived[name], dtype=float)
            var = factor * float(np.sum((samples - samples.mean()) ** 2))
            combined[name] = {"value": float(central[name]), "error": float(np.sqrt(var))}
    else:
        for name in OBSERVABLES:
            combined[name] = {"value": float(central[name]), "error": float("nan")}

    n_bins = len(next(iter(results[0].bin_primitives.values())))
    if n_bins > 1:
        per_bin = {name: np.stack([r.bin_primitives[name] for r in results]) for name in PRIMITIVES}
        derived = derive_observables(per_bin, temperature, n_sites)
        for name in OBSERVABLES:
            values = np.asarray(derived[name], dtype=float).reshape(n_r, n_bins)
            spread = np.std(values, axis=1, ddof=1) / np.sqrt(n_bins)
            combined[name]["thermal_error"] = float(np.sqrt(np.mean(spread**2) / n_r))
    else:
        for name in OBSERVABLES:
            combined[name]["thermal_error"] = float("nan")
    if n_r == 1:
        for name in OBSERVABLES:
            combined[name]["error"] = combined[name]["thermal_error"]
    return combined


def _check_run(n_sweeps: int, n_bins: int) -> int:
    if n_bins < 1:
        raise ValueError(f"n_bins must be positive, got {n_bins}")
    sweeps_per_bin = n_sweeps // n_bins
    if sweeps_per_bin < 1:
        raise ValueError(
            f"n_sweeps ({n_sweeps}) must be at least n_bins ({n_bins}) so every bin contains at least one sweep."
        )
    return sweeps_per_bin


def _check_start(start: str) -> bool:
    if start not in ("hot", "cold"):
        raise ValueError(f"start must be 'hot' or 'cold', got {start!r}")
    return start == "hot"


def run_single_realization(L: int, J: np.ndarray, temperature: float, *, n_sweeps: int, n_therm: int,
                           n_bins: int = 10, seed=None, measure_percolation: bool = True, start: str = "hot",
                           engine: str = "auto", device=None) -> RealizationResult:
    """One realization at one temperature on the GPU (reference ``simulation.py:148-242``).

    ``engine``: ``"grid"`` (one cooperative launch per call, the lattice in
    shared-memory tiles on every SM), ``"plain"`` (global-memory engine, one
    lattice per launch sequence), ``"batched"`` (resident or cluster engine,
    one CTA or one cluster for the lattice) or ``"auto"`` (``auto_engine``:
    one resident CTA for L <= 64, grid above where it has a plan, else plain).
    Every engine gives the same result.
    """
    spb = _check_run(n_sweeps, n_bins)
    hot = _check_start(start)
    if L < 3:
        raise ValueError(f"L must be at least 3 (got {L})")
    spec = ChainSpec(L=L, realization=0, key=chain_key(seed), beta=1.0 / temperature, n_therm=n_therm,
                     n_bins=n_bins, sweeps_per_bin=spb)
    cs = ChainSet([spec], [pack_couplings(J, L)], device=device)
    cs.init_spins(hot)
    cs.run_to_end(engine=engine)
    ib, fb = cs.bins(0)
    return realization_from_sums(ib, fb, spb, measure_percolation)


@dataclass
class ScanPlan:
    """Everything a temperature scan computes before any sweep: tasks, keys, couplings, run lengths.

    Task ``k`` is temperature ``k // n_realizations`` and realization
    ``k % n_realizations``, the reference's T-major order
    (``simulation.py:384-399``); ``keys[k]`` is the Philox key drawn from that
    task's ``SeedSequence`` child.
    """

    L: int
    p: float
    temperatures: list
    couplings: list
    keys: np.ndarray
    n_sweeps: int
    n_therm: int
    n_bins: int
    sweeps_per_bin: int
    seed: int
    hot: bool
    start: str
    measure_percolation: bool

    @property
    def n_realizations(self) -> int:
        return len(self.couplings)

    @property
    def n_tasks(self) -> int:
        return len(self.temperatures) * len(self.couplings)

    def spec(self, k: int) -> ChainSpec:
        t_index, r = divmod(k, self.n_realizations)
        return ChainSpec(L=self.L, realization=r, key=int(self.keys[k]), beta=1.0 / self.temperatures[t_index],
                         n_therm=self.n_therm, n_bins=self.n_bins, sweeps_per_bin=self.sweeps_per_bin)


def plan_temperature_scan(L: int, p: float, temperatures: Sequence[float], *, n_realizations: int = 1,
                          n_sweeps: int = 10_000, n_therm: Optional[int] = None, n_bins: int = 10, seed: int = 0,
                          measure_percolation: bool = True, start: str = "hot",
                          disorder: Optional[Iterable[tuple]] = None) -> ScanPlan:
    """Argument checks, disorder and per-task keys of a scan (reference ``simulation.py:362-399``)."""
    temperatures = [float(t) for t in temperatures]
    if n_therm is None:
        n_therm = max(1, n_sweeps // 10)
    spb = _check_run(n_sweeps, n_bins)
    hot = _check_start(start)
    if L < 3:
        raise ValueError(f"L must be at least 3 (got {L})")

    seed_sequence = np.random.SeedSequence(seed)
    disorder_seeds, run_seeds = seed_sequence.spawn(2)
    if disorder is None:
        disorder_rng = np.random.default_rng(disorder_seeds)
        realizations = generate_disorders(L, p, disorder_rng, n_realizations)
    else:
        realizations = list(disorder)[:n_realizations]
        if len(realizations) < n_realizations:
            raise ValueError(
                f"only {len(realizations)} disorder realizations supplied but n_realizations={n_realizations}"
            )
    couplings = [couplings_from_disorder(J_h, J_v) for J_h, J_v in realizations]
    for J in couplings:
        if J.size != 2 * L * L:
            raise ValueError(f"disorder realization has {J.size // 2} sites, expected {L * L}")
    keys = child_keys(run_seeds, len(temperatures) * len(couplings))
    return ScanPlan(L=L, p=p, temperatures=temperatures, couplings=couplings, keys=keys, n_sweeps=n_sweeps,
                    n_therm=n_therm, n_bins=n_bins, sweeps_per_bin=spb, seed=seed, hot=hot, start=start,
                    measure_percolation=measure_percolation)


def run_scan_tasks(plan: ScanPlan, tasks: Optional[Sequence[int]] = None, *, engine: str = "auto", device=None,
                   chunk: int = 1000):
    """Run some tasks of a plan on one GPU; returns their per-bin sums.

    ``(int_sums, f64_sums)`` with shapes ``(len(tasks), n_bins, 12)`` int64
    and ``(len(tasks), n_bins, 2)`` float64.  A task's sums do not depend on
    which other tasks share the batch.
    """
    tasks = list(range(plan.n_tasks)) if tasks is None else [int(k) for k in tasks]
    nb = plan.n_bins
    int_sums = np.zeros((len(tasks), nb, 12), dtype=np.int64)
    f_sums = np.zeros((len(tasks), nb, 2), dtype=np.float64)
    if not tasks:
        return int_sums, f_sums
    cs = ChainSet([plan.spec(k) for k in tasks], [pack_couplings(J, plan.L) for J in plan.couplings], device=device)
    cs.init_spins(plan.hot)
    cs.run_to_end(engine=engine, chunk=chunk)
    acc_i, acc_f = cs.all_bins()
    for i in range(len(tasks)):
        a = cs.acc_off[i]
        int_sums[i] = acc_i[a: a + nb]
        f_sums[i] = acc_f[a: a + nb]
    return int_sums, f_sums


def assemble_scan(plan: ScanPlan, int_sums: np.ndarray, f_sums: np.ndarray) -> Dict[str, object]:
    """Jackknife-combined observables and metadata from every task's sums (reference ``simulation.py:401-444``).

    The estimators of :func:`combine_realizations` (per-realization full-run
    and per-bin means, disorder average, leave-one-out jackknife, bin-based
    thermal error), evaluated for all temperatures at once.
    """
    n_r = plan.n_realizations
    temperatures = plan.temperatures
    n_t, nb, spb = len(temperatures), plan.n_bins, plan.sweeps_per_bin
    total = nb * spb
    n_sites = plan.L * plan.L
    ii = np.asarray(int_sums).reshape(n_t, n_r, nb, -1)
    ff = np.asarray(f_sums, dtype=np.float64).reshape(n_t, n_r, nb, -1)
    prim: Dict[str, np.ndarray] = {}
    bins: Dict[str, np.ndarray] = {}
    for name in PRIMITIVES:
        kind, k = _SOURCE[name]
        if not plan.measure_percolation and name.startswith("wrap"):
            prim[name] = np.full((n_t, n_r), np.nan)
            bins[name] = np.full((n_t, n_r, nb), np.nan)
        elif kind == "i":
            col = ii[..., k]
            prim[name] = col.sum(axis=2).astype(np.float64) / total
            bins[name] = col.astype(np.float64) / spb
        else:
            col = np.ascontiguousarray(ff[..., k])
            prim[name] = col.sum(axis=2) / total
            bins[name] = col / spb
    temps = np.asarray(temperatures, dtype=np.float64)
    results = {name: {"value": np.empty(n_t), "error": np.full(n_t, np.nan), "thermal_error": np.full(n_t, np.nan)}
               for name in OBSERVABLES}
    if n_t and n_r:
        central = derive_observables({name: v.mean(axis=1) for name, v in prim.items()}, temps, n_sites)
        for name in OBSERVABLES:
            results[name]["value"][:] = central[name]
        if n_r > 1:
            loo = {name: (v.sum(axis=1, keepdims=True) - v) / (n_r - 1) for name, v in prim.items()}
            derived = derive_observables(loo, temps[:, None], n_sites)
            factor = (n_r - 1) / n_r
            for name in OBSERVABLES:
                samples = np.broadcast_to(np.asarray(derived[name], dtype=float), (n_t, n_r))
                dev = samples - samples.mean(axis=1, keepdims=True)
                results[name]["error"][:] = np.sqrt(factor * np.sum(dev * dev, axis=1))
        if nb > 1:
            derived = derive_observables(bins, temps[:, None, None], n_sites)
            for name in OBSERVABLES:
                values = np.broadcast_to(np.asarray(derived[name], dtype=float), (n_t, n_r, nb))
                spread = np.std(values, axis=2, ddof=1) / np.sqrt(nb)
                results[name]["thermal_error"][:] = np.sqrt(np.mean(spread**2, axis=1) / n_r)
        if n_r == 1:
            for name in OBSERVABLES:
                results[name]["error"][:] = results[name]["thermal_error"]

    metadata = {
        "L": plan.L,
        "p": plan.p,
        "n_realizations": n_r,
        "n_sweeps": plan.n_sweeps,
        "n_therm": plan.n_therm,
        "n_bins": plan.n_bins,
        "seed": plan.seed,
        "measure_percolation": plan.measure_percolation,
        "start": plan.start,
        "algorithm": "Swendsen-Wang cluster update on satisfied bonds",
        "estimator": (
            "primitive moments accumulated over the full run of each realization; "
            "derived observables formed after disorder averaging; "
            "uncertainties by jackknife over realizations"
        ),
        "binder_convention": "1 - [<m^4>] / (3 [<m^2>]^2), from disorder-averaged moments",
        "specific_heat_convention": "[<E^2> - <E>^2] / (T^2 N)",
        "susceptibility_convention": "[<M^2> - <|M|>^2] / (T N)",
        "error_convention": (
            "error = jackknife over disorder realizations; "
            "thermal_error = mean within-realization standard error across bins"
        ),
        "backend": "cuda-sm100a",
        "rng": "philox4x32-10 per chain (key from the task's SeedSequence child)",
    }
    return {"temperatures": np.asarray(temperatures), "observables": results, "metadata": metadata}


def run_temperature_scan(L: int, p: float, temperatures: Sequence[float], *, n_realizations: int = 1,
                         n_sweeps: int = 10_000, n_therm: Optional[int] = None, n_bins: int = 10, seed: int = 0,
                         n_workers: Optional[int] = None, measure_percolation: bool = True, start: str = "hot",
                         disorder: Optional[Iterable[tuple]] = None, engine: str = "auto", device=None,
                         chunk: int = 1000) -> Dict[str, object]:
    """Scan temperatures, averaging over disorder realizations (reference ``simulation.py:336-444``).

    Same arguments, seeding, realizations and return value as the reference.
    ``n_workers`` is accepted for compatibility and ignored: all
    ``len(temperatures) * n_realizations`` tasks run as chains of one GPU
    batch.  Extra keywords: ``engine`` (see :func:`run_single_realization`),
    ``device`` and ``chunk`` (sweeps per engine call).
    """
    plan = plan_temperature_scan(L, p, temperatures, n_realizations=n_realizations, n_sweeps=n_sweeps,
                                 n_therm=n_therm, n_bins=n_bins, seed=seed, measure_percolation=measure_percolation,
                                 start=start, disorder=disorder)
    int_sums, f_sums = run_scan_tasks(plan, engine=engine, device=device, chunk=chunk)
    return assemble_scan(plan, int_sums, f_sums)


def save_results(path: str, results: Dict[str, object]) -> None:
    """Write a scan to ``.npz`` in the reference's layout (``simulation.py:447-458``)."""
    directory = os.path.dirname(os.path.abspath(path))
    os.makedirs(directory, exist_ok=True)
    flat = {"temperatures": results["temperatures"]}
    for name, entry in results["observables"].items():
        for key, array in entry.items():
            flat[f"{name}__{key}"] = array
    flat["metadata_json"] = np.asarray(json.dumps(results["metadata"]))
    np.savez_compressed(path, **flat)


def load_results(path: str) -> Dict[str, object]:
    """Read a scan written by :func:`save_results` or by the reference (``simulation.py:461-472``)."""
    with np.load(path, allow_pickle=False) as data:
        temperatures = data["temperatures"]
        metadata = json.loads(str(data["metadata_json"]))
        observables: Dict[str, Dict[str, np.ndarray]] = {}
        for key in data.files:
            if "__" not in key:
                continue
            name, field_name = key.split("__", 1)
            observables.setdefault(name, {})[field_name] = data[key]
    return {"temperatures": temperatures, "observables": observables, "metadata": metadata}
