"""Exact results of the pure square-lattice Ising model (test infrastructure only).

The reference pins its p = 0 physics only through the magnetization
(``tests/test_physics.py:32-36, 92-101``); the energy check added here uses
the exact partition function of the periodic ``L x L`` lattice, restated from
the published formula of B. Kaufman, Phys. Rev. 76, 1232 (1949), in the form
of A. E. Ferdinand and M. E. Fisher, Phys. Rev. 185, 832 (1969):

    Z = 1/2 (2 sinh 2K)^(L^2/2) (Z1 + Z2 + Z3 + Z4),
    Z1 = prod_{r=0}^{L-1} 2 cosh(L g_{2r+1} / 2),   Z2 = same with sinh,
    Z3 = prod_{r=0}^{L-1} 2 cosh(L g_{2r} / 2),     Z4 = same with sinh,
    cosh g_l = cosh 2K coth 2K - cos(pi l / L)  (l >= 1),  g_0 = 2K + ln tanh K,

with K = beta J.  The energy per site is u = -(1/L^2) d ln Z / dK.  The
formula is checked against brute-force enumeration for L = 3 and 4 in the
test suite.
"""

from __future__ import annotations

import itertools

import mpmath as mp
import numpy as np

__all__ = ["TC_EXACT", "log_partition_torus", "energy_per_site_torus", "brute_force_energy_per_site",
           "onsager_magnetization"]

TC_EXACT = 2.0 / np.log(1.0 + np.sqrt(2.0))


def log_partition_torus(K, L: int):
    """``ln Z`` of the periodic ``L x L`` Ising model at coupling ``K`` (mpmath number)."""
    K = mp.mpf(K)
    c = mp.cosh(2 * K) * mp.coth(2 * K)

    def gamma(l):
        if l == 0:
            return 2 * K + mp.log(mp.tanh(K))
        return mp.acosh(c - mp.cos(mp.pi * l / L))

    z1 = z2 = z3 = z4 = mp.mpf(1)
    for r in range(L):
        go, ge = gamma(2 * r + 1), gamma(2 * r)
        z1 *= 2 * mp.cosh(L * go / 2)
        z2 *= 2 * mp.sinh(L * go / 2)
        z3 *= 2 * mp.cosh(L * ge / 2)
        z4 *= 2 * mp.sinh(L * ge / 2)
    return mp.log(mp.mpf(1) / 2) + (L * L / mp.mpf(2)) * mp.log(2 * mp.sinh(2 * K)) + mp.log(z1 + z2 + z3 + z4)


def energy_per_site_torus(T: float, L: int, dps: int = 40) -> float:
    """Exact ``<E>/N`` of the periodic ``L x L`` ferromagnet (J = 1) at temperature ``T``."""
    with mp.workdps(dps):
        K = mp.mpf(1) / mp.mpf(T)
        d = mp.diff(lambda k: log_partition_torus(k, L), K)
        return float(-d / (L * L))


def brute_force_energy_per_site(T: float, L: int) -> float:
    """``<E>/N`` by enumerating all ``2^(L*L)`` states (L <= 4)."""
    N = L * L
    beta = 1.0 / T
    states = np.array(list(itertools.product((1, -1), repeat=N)), dtype=np.int64).reshape(-1, L, L)
    e = -(states * np.roll(states, -1, axis=1)).sum(axis=(1, 2)) - (states * np.roll(states, -1, axis=2)).sum(
        axis=(1, 2))
    w = np.exp(-beta * (e - e.min()))
    return float((w * e).sum() / w.sum() / N)


def onsager_magnetization(T: float) -> float:
    """Spontaneous magnetization of the infinite lattice (reference ``tests/test_physics.py:32-36``)."""
    if T >= TC_EXACT:
        return 0.0
    return float((1.0 - np.sinh(2.0 / T) ** -4) ** 0.125)
