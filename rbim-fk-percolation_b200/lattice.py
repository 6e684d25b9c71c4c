"""Square-lattice geometry, host side (mirror of the reference's ``src/rbim/lattice.py``).

Site ``n = x * L + y`` (x slow, y fast); bond ``2n`` joins ``(x, y)`` to
``(x + 1, y)`` and bond ``2n + 1`` joins ``(x, y)`` to ``(x, y + 1)``, both
periodic (reference ``lattice.py:1-23``).  The GPU engine does not use the
explicit bond table: it stores every per-site quantity as a linear bit plane
(``pack_plane``) and derives neighbours arithmetically.  The table is kept for
API compatibility with ``label_and_wrap(active, lattice)``.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

__all__ = ["Lattice", "build_lattice", "site_index", "couplings_from_disorder"]


@dataclass(frozen=True)
class Lattice:
    """Bond structure of a periodic ``L x L`` square lattice (reference ``lattice.py:35-81``)."""

    L: int
    bonds: np.ndarray
    wraps_x: np.ndarray
    wraps_y: np.ndarray
    bond_dx: np.ndarray
    bond_dy: np.ndarray

    @property
    def n_sites(self) -> int:
        return self.L * self.L

    @property
    def n_bonds(self) -> int:
        return 2 * self.n_sites

    def wrap_mask(self, axis: str) -> np.ndarray:
        if axis == "x":
            return self.wraps_x
        if axis == "y":
            return self.wraps_y
        raise ValueError(f"axis must be 'x' or 'y', got {axis!r}")


def site_index(x, y, L: int):
    """Flat site index ``n = x * L + y`` (reference ``lattice.py:84-86``)."""
    return x * L + y


def build_lattice(L: int) -> Lattice:
    """Periodic ``L x L`` lattice; ``L < 3`` is rejected as in the reference (``lattice.py:89-135``)."""
    if L < 3:
        raise ValueError(
            f"L must be at least 3 (got {L}); smaller lattices produce duplicate bonds under periodic "
            "boundary conditions."
        )
    n = np.arange(L * L, dtype=np.int64)
    x, y = n // L, n % L
    bonds = np.empty((2 * L * L, 2), dtype=np.int64)
    bonds[0::2, 0] = n
    bonds[0::2, 1] = ((x + 1) % L) * L + y
    bonds[1::2, 0] = n
    bonds[1::2, 1] = x * L + (y + 1) % L
    wraps_x = np.zeros(2 * L * L, dtype=bool)
    wraps_y = np.zeros(2 * L * L, dtype=bool)
    wraps_x[0::2] = x == L - 1
    wraps_y[1::2] = y == L - 1
    bond_dx = np.zeros(2 * L * L, dtype=np.int64)
    bond_dy = np.zeros(2 * L * L, dtype=np.int64)
    bond_dx[0::2] = 1
    bond_dy[1::2] = 1
    return Lattice(L=L, bonds=bonds, wraps_x=wraps_x, wraps_y=wraps_y, bond_dx=bond_dx, bond_dy=bond_dy)


def couplings_from_disorder(J_h: np.ndarray, J_v: np.ndarray) -> np.ndarray:
    """Interleave ``J_h``/``J_v`` into bond order (reference ``lattice.py:138-161``)."""
    if J_h.shape != J_v.shape:
        raise ValueError(f"J_h and J_v must have the same shape, got {J_h.shape} and {J_v.shape}")
    if J_h.ndim != 2 or J_h.shape[0] != J_h.shape[1]:
        raise ValueError(f"couplings must be square 2D arrays, got shape {J_h.shape}")
    L = J_h.shape[0]
    J = np.empty(2 * L * L, dtype=np.int8)
    J[0::2] = J_h.reshape(-1)
    J[1::2] = J_v.reshape(-1)
    return J
