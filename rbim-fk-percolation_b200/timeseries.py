"""Per-sweep time series of the cluster observables, and their integrated autocorrelation times.

The reference's ``scripts/measure_autocorrelation.py`` runs one realization
at a time through ``sw_sweep`` and keeps the raw series of the energy, the
largest cluster's size and magnetization, their ratio and ``wrap_y``
(``measure_autocorrelation.py:69-90``).  Here every (temperature,
realization) chain of a scan runs in one device batch with per-sweep records
(9 int32 per sweep, written by the sweep kernels), and only the records come
back; the series and the autocorrelation estimate are formed on the host.
"""

from __future__ import annotations

from typing import Dict, Optional, Sequence, Tuple

import numpy as np

from .engine import ChainSet
from .packing import pack_couplings
from .simulation import plan_temperature_scan

__all__ = ["TRACKED", "SERIES", "collect_series", "integrated_autocorrelation"]

#: Observables the reference tracks (``measure_autocorrelation.py:37``).
TRACKED = ("energy", "largest_size", "largest_abs_mag", "mag_ratio", "wrap_y")

#: Every series available from the records, in record order plus the ratio.
SERIES = ("energy", "magnetization", "n_clusters", "largest_size", "largest_abs_mag", "second_size",
          "second_abs_mag", "wrap_x", "wrap_y", "mag_ratio")


def collect_series(L: int, p: float, temperatures: Sequence[float], *, n_sweeps: int, n_therm: int,
                   n_realizations: int = 1, seed: int = 0, start: str = "hot", disorder=None, device=None,
                   chunk: int = 2000) -> Dict[str, np.ndarray]:
    """Raw per-sweep series of every chain of a scan.

    Seeding follows the reference script (``SeedSequence(seed).spawn(2)``,
    then one child per task in temperature-major order), the same tasks as
    :func:`~.simulation.run_temperature_scan`.  Returns arrays of shape
    ``(n_temperatures, n_realizations, n_sweeps)`` keyed by :data:`SERIES`.
    """
    plan = plan_temperature_scan(L, p, temperatures, n_realizations=n_realizations, n_sweeps=n_sweeps,
                                 n_therm=n_therm, n_bins=1, seed=seed, start=start, disorder=disorder)
    specs = []
    for k in range(plan.n_tasks):
        s = plan.spec(k)
        s.records = True
        specs.append(s)
    cs = ChainSet(specs, [pack_couplings(J, L) for J in plan.couplings], device=device)
    cs.init_spins(plan.hot)
    cs.run_to_end(engine="batched", chunk=chunk)
    n_t, n_r = len(plan.temperatures), plan.n_realizations
    rec = cs.records.cpu().numpy().reshape(n_t, n_r, n_sweeps, -1).astype(np.float64)
    out = {name: rec[..., i] for i, name in enumerate(SERIES[:9])}
    largest = out["largest_size"]
    with np.errstate(divide="ignore", invalid="ignore"):
        out["mag_ratio"] = np.where(largest > 0, out["largest_abs_mag"] / np.where(largest > 0, largest, 1.0), 0.0)
    return out


def integrated_autocorrelation(series: np.ndarray, c: float = 6.0) -> Tuple[float, int]:
    """``tau_int = 1/2 + sum_t rho(t)`` with Sokal's self-consistent window.

    The autocorrelation function comes from an FFT of the mean-subtracted
    series (zero-padded to a power of two >= 2n); the window grows until it
    reaches ``c`` times the running estimate.  Returns ``(tau_int, window)``;
    constant or very short series give ``(0.5, 0)``.  Same estimator as the
    reference's ``measure_autocorrelation.py:40-66``.
    """
    x = np.asarray(series, dtype=float)
    x = x - x.mean()
    n = x.size
    if n < 16 or not np.any(x):
        return 0.5, 0
    size = 1 << int(np.ceil(np.log2(2 * n)))
    f = np.fft.rfft(x, size)
    acf = np.fft.irfft(f * np.conjugate(f), size)[:n].real
    if acf[0] <= 0:
        return 0.5, 0
    rho = acf / acf[0]
    tau = 0.5
    for window in range(1, n):
        tau += rho[window]
        if window >= c * tau:
            return float(max(tau, 0.5)), window
    return float(max(tau, 0.5)), n - 1
