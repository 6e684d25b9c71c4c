"""+-J bond disorder: generation, ``.npz`` storage and frustration (mirror of ``src/rbim/disorder.py``).

Generation draws exactly the numpy calls of the reference (``disorder.py:59-60``),
so a given generator state yields the same realization here and there; that is
what makes disorder-averaged GPU results comparable with the reference's at
equal realizations.  The file format is the reference's: ``J_h`` and ``J_v``
int8 ``(L, L)`` arrays plus optional ``p`` and ``seed`` (``disorder.py:69-108``).
"""

from __future__ import annotations

import os
from typing import Optional, Tuple

import numpy as np

__all__ = [
    "generate_disorder",
    "save_disorder",
    "load_disorder",
    "frustrated_plaquettes",
    "frustration_density",
    "default_disorder_filename",
]


def generate_disorder(L: int, p: float, rng: Optional[np.random.Generator] = None) -> Tuple[np.ndarray, np.ndarray]:
    """One realization with ``P(J = -1) = p`` (reference ``disorder.py:32-61``)."""
    if not 0.0 <= p <= 1.0:
        raise ValueError(f"p must lie in [0, 1], got {p}")
    if rng is None:
        rng = np.random.default_rng()
    J_h = np.where(rng.random((L, L)) < p, -1, 1).astype(np.int8)
    J_v = np.where(rng.random((L, L)) < p, -1, 1).astype(np.int8)
    return J_h, J_v


def default_disorder_filename(L: int, p: float, index: int = 0) -> str:
    """Canonical file name of a stored realization (reference ``disorder.py:64-66``)."""
    return f"disorder_L={L}_p={p:.3f}_r={index:04d}.npz"


def save_disorder(path: str, J_h: np.ndarray, J_v: np.ndarray, *, p: Optional[float] = None,
                  seed: Optional[int] = None) -> None:
    """Write a realization (reference ``disorder.py:69-92``)."""
    directory = os.path.dirname(os.path.abspath(path))
    os.makedirs(directory, exist_ok=True)
    metadata = {}
    if p is not None:
        metadata["p"] = np.asarray(p)
    if seed is not None:
        metadata["seed"] = np.asarray(seed)
    np.savez_compressed(path, J_h=J_h, J_v=J_v, **metadata)


def load_disorder(path: str) -> Tuple[np.ndarray, np.ndarray]:
    """Read a realization; ``KeyError`` if ``J_h``/``J_v`` are absent (reference ``disorder.py:95-108``)."""
    with np.load(path) as data:
        if "J_h" not in data or "J_v" not in data:
            raise KeyError(f"{path} does not contain 'J_h' and 'J_v' arrays; found {list(data.keys())}")
        J_h = data["J_h"].astype(np.int8)
        J_v = data["J_v"].astype(np.int8)
    return J_h, J_v


def frustrated_plaquettes(J_h: np.ndarray, J_v: np.ndarray) -> np.ndarray:
    """Plaquettes whose four couplings multiply to -1 (reference ``disorder.py:111-131``)."""
    bottom = J_h.astype(np.int64)
    top = np.roll(J_h, -1, axis=1).astype(np.int64)
    left = J_v.astype(np.int64)
    right = np.roll(J_v, -1, axis=0).astype(np.int64)
    return (bottom * top * left * right) < 0


def frustration_density(J_h: np.ndarray, J_v: np.ndarray) -> float:
    """Fraction of frustrated plaquettes (reference ``disorder.py:134-140``)."""
    return float(frustrated_plaquettes(J_h, J_v).mean())
