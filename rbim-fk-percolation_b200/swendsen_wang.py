"""A single Swendsen-Wang update on the GPU (mirror of ``src/rbim/swendsen_wang.py``).

``sw_sweep`` runs one sweep of one lattice through the plain engine and
returns the reference's ``SweepResult``.  It is the per-sweep API; throughput
work goes through :class:`~.engine.ChainSet` and ``run_temperature_scan``,
which keep the state on the device across sweeps.
"""

from __future__ import annotations

import threading
from dataclasses import dataclass
from typing import Optional

import numpy as np

from .engine import ChainSet, ChainSpec, _torch, auto_engine, require_cuda, single_cta_threads
from .lattice import Lattice
from .packing import pack_couplings, pack_spins, threshold, unpack_spins, words_for

__all__ = [
    "SweepResult",
    "energy",
    "magnetization",
    "random_spins",
    "aligned_spins",
    "initial_spins",
    "sw_sweep",
]


@dataclass(frozen=True)
class SweepResult:
    """Observables of one sweep (reference ``swendsen_wang.py:24-53``).

    Every field is measured on the device in the sweep's record, including
    ``second_abs_magnetization`` (|M| of the second-largest cluster,
    reference ``swendsen_wang.py:151-154``).
    """

    energy: float
    magnetization: float
    n_clusters: int
    largest_size: int
    largest_abs_magnetization: float
    second_size: int
    second_abs_magnetization: float
    wraps_x: Optional[bool]
    wraps_y: Optional[bool]


def random_spins(n_sites: int, rng: np.random.Generator) -> np.ndarray:
    """Random ``+-1`` configuration (reference ``swendsen_wang.py:56-58``)."""
    return rng.integers(0, 2, size=n_sites, dtype=np.int64) * 2 - 1


def aligned_spins(n_sites: int) -> np.ndarray:
    """All spins up (reference ``swendsen_wang.py:61-63``)."""
    return np.ones(n_sites, dtype=np.int64)


def initial_spins(n_sites: int, rng: np.random.Generator, start: str = "hot") -> np.ndarray:
    """Hot or cold start (reference ``swendsen_wang.py:66-78``)."""
    if start == "hot":
        return random_spins(n_sites, rng)
    if start == "cold":
        return aligned_spins(n_sites)
    raise ValueError(f"start must be 'hot' or 'cold', got {start!r}")


def energy(spins: np.ndarray, lattice: Lattice, J: np.ndarray) -> float:
    """``-sum J s s`` over bonds (host helper, reference ``swendsen_wang.py:81-84``)."""
    ends = lattice.bonds
    return -float(np.sum(J * spins[ends[:, 0]] * spins[ends[:, 1]]))


def magnetization(spins: np.ndarray) -> float:
    """``sum s`` (host helper, reference ``swendsen_wang.py:87-89``)."""
    return float(np.sum(spins))


def sw_sweep(spins: np.ndarray, lattice: Lattice, J: np.ndarray, beta: float, rng=None, *, key: Optional[int] = None,
             sweep: int = 0, measure: bool = True, measure_percolation: bool = True,
             device=None) -> Optional[SweepResult]:
    """One Swendsen-Wang update of ``spins`` in place (reference ``swendsen_wang.py:103-172``).

    Randomness comes from the Philox stream of ``key`` at sweep counter
    ``sweep``; when ``key`` is omitted it is drawn from ``rng``.  The device
    buffers of L x L lattices are kept between calls (one chain set per device
    and L, used under a lock), so a loop over ``sw_sweep`` allocates device
    memory only on its first call; each call still copies the spins and
    couplings in and the spins and the record out.
    """
    L = lattice.L
    if key is None:
        if rng is None:
            raise ValueError("sw_sweep needs a key or a numpy Generator")
        key = int(rng.integers(0, 2**63, dtype=np.int64))
    cs, lock, engine = _sweep_chain_set(L, device)
    with lock:
        # One chain whose only sweep is `sweep`: measured when n_therm == sweep.
        cs.coupling_pool[: 2 * words_for(L)].copy_(_torch().from_numpy(pack_couplings(J, L).view(np.int32)))
        cs.set_spins(0, pack_spins(spins, L))
        cs.set_descriptor_fields(0, key=int(key) & (2**64 - 1), thr=threshold(beta), sweep=sweep,
                                 n_therm=sweep if measure else sweep + 1, n_bins=1, sweeps_per_bin=1)
        cs.acc_int.zero_()
        cs.acc_f64.zero_()
        if engine == "grid":
            cs.run_grid(1)  # one cooperative launch over every SM
        elif engine == "batched":
            cs.run_batched(1, threads=single_cta_threads(L))  # one resident CTA
        else:
            cs.run_plain(1)
        cs.check_status()
        spins[...] = unpack_spins(cs.spin_words(0), L, dtype=spins.dtype)
        if not measure:
            return None
        rec = cs.chain_records(0)[0]
    wx = bool(rec[7]) if measure_percolation else None
    wy = bool(rec[8]) if measure_percolation else None
    return SweepResult(energy=float(rec[0]), magnetization=float(rec[1]), n_clusters=int(rec[2]),
                       largest_size=int(rec[3]), largest_abs_magnetization=float(rec[4]), second_size=int(rec[5]),
                       second_abs_magnetization=float(rec[6]), wraps_x=wx, wraps_y=wy)


_sets_lock = threading.Lock()
_sets = {}  # (device, L) -> (ChainSet of one chain with a one-row record buffer, its lock, engine)


def _sweep_chain_set(L: int, device):
    """The device state ``sw_sweep`` reuses for L x L lattices: one chain set per (device, L), created on first
    use, so that a caller looping over ``sw_sweep`` does not allocate and free device buffers every sweep, and
    and the engine the sweep runs on: ``auto_engine``'s choice for one lattice."""
    dev = require_cuda(device)
    key = (str(dev), int(L))
    with _sets_lock:
        entry = _sets.get(key)
        if entry is None:
            spec = ChainSpec(L=L, realization=0, key=0, beta=1.0, n_therm=0, n_bins=1, sweeps_per_bin=1, records=True)
            cs = ChainSet([spec], [np.zeros(2 * words_for(L), dtype="<u4")], device=dev)
            with _torch().cuda.device(dev):
                engine = auto_engine([spec])
            entry = (cs, threading.Lock(), engine)
            _sets[key] = entry
        return entry
