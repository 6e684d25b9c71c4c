"""+-J bond disorder: generation, ``.npz`` storage and frustration (mirror of ``src/rbim/disorder.py``).

Generation draws exactly the numpy calls of the reference (``disorder.py:59-60``),
so a given generator state yields the same realization here and there; that is
what makes disorder-averaged GPU results comparable with the reference's at
equal realizations.  The file format is the reference's: ``J_h`` and ``J_v``
int8 ``(L, L)`` arrays plus optional ``p`` and ``seed`` (``disorder.py:69-108``).
"""

from __future__ import annotations

import math
import os
from concurrent.futures import ThreadPoolExecutor
from typing import List, Optional, Tuple

import numpy as np

__all__ = [
    "generate_disorder",
    "generate_disorders",
    "save_disorder",
    "load_disorder",
    "frustrated_plaquettes",
    "frustration_density",
    "default_disorder_filename",
]


_PARALLEL_DRAWS = 1 << 20  # below this many draws one thread is as fast
_GROUP_DRAWS = 1 << 25     # most raw draws held at once by generate_disorders


def _raw_draws(rng: np.random.Generator, n: int) -> np.ndarray:
    """The next ``n`` raw 64-bit draws of a PCG64 generator, leaving it as if drawn in sequence.

    Large requests are cut into chunks drawn by several threads from copies
    of the generator jumped ahead to each chunk's start (PCG64 ``advance`` is
    exact, and ``random_raw`` runs without the GIL); the generator itself is
    then advanced past all of them.
    """
    bg = rng.bit_generator
    workers = min(8, os.cpu_count() or 1)
    if n < _PARALLEL_DRAWS or workers < 2:
        return bg.random_raw(n)
    state = bg.state
    bounds = [n * i // workers for i in range(workers + 1)]
    out = np.empty(n, dtype=np.uint64)

    def part(i: int) -> None:
        g = np.random.PCG64()
        g.state = state
        g.advance(bounds[i])
        out[bounds[i]: bounds[i + 1]] = g.random_raw(bounds[i + 1] - bounds[i])

    with ThreadPoolExecutor(workers) as ex:
        list(ex.map(part, range(workers)))
    bg.advance(n)
    return out


def _pcg64_compare(rng: np.random.Generator, n: int, p: float) -> np.ndarray:
    """``rng.random(n) < p`` from the raw 64-bit draws of a PCG64 generator.

    numpy's PCG64 double is the top 53 bits of one raw draw times 2**-53, so
    ``u < p`` is ``(raw >> 11) < ceil(p * 2**53)`` (``p * 2**53`` is exact),
    that is ``raw < ceil(p * 2**53) << 11``: one integer compare per draw, the
    same stream consumed, no float array.  For 0 < p < 1 only.
    """
    t = math.ceil(p * 9007199254740992.0) << 11
    return _raw_draws(rng, n) < np.uint64(t)


def _check_pcg64_compare() -> bool:
    """Whether _pcg64_compare reproduces ``rng.random() < p`` with this numpy (checked once)."""
    for seed, p, n in ((1, 0.05, 4099), (2, 0.5, 4099), (3, 1e-300, 4099), (4, 1.0 - 2.0**-53, 4099),
                       (5, 0.1, _PARALLEL_DRAWS + 4099)):
        a = np.random.default_rng(seed)
        b = np.random.default_rng(seed)
        if not np.array_equal(a.random(n) < p, _pcg64_compare(b, n, p)):
            return False
        if a.random() != b.random():
            return False
    return True


def _fast_path(rng: np.random.Generator, p: float) -> bool:
    global _PCG64_COMPARE_OK
    if not (0.0 < p < 1.0 and type(rng.bit_generator) is np.random.PCG64):
        return False
    if rng.bit_generator.state.get("has_uint32", 0):
        return False  # a buffered 32-bit half would be dropped by advance()
    if _PCG64_COMPARE_OK is None:
        _PCG64_COMPARE_OK = _check_pcg64_compare()
    return _PCG64_COMPARE_OK


_PCG64_COMPARE_OK: Optional[bool] = None


def generate_disorder(L: int, p: float, rng: Optional[np.random.Generator] = None) -> Tuple[np.ndarray, np.ndarray]:
    """One realization with ``P(J = -1) = p`` (reference ``disorder.py:32-61``).

    The reference draws ``rng.random((L, L)) < p`` for ``J_h``, then for
    ``J_v``.  With numpy's default PCG64 generator the same draws are compared
    as integers (:func:`_pcg64_compare`, checked against ``rng.random`` once
    per process), which gives the same couplings and leaves the generator in
    the same state.
    """
    return generate_disorders(L, p, rng, 1)[0]


def generate_disorders(L: int, p: float, rng: Optional[np.random.Generator] = None,
                       n: int = 1) -> List[Tuple[np.ndarray, np.ndarray]]:
    """``n`` realizations, the same as ``n`` calls of :func:`generate_disorder` with ``rng`` in a row.

    With numpy's default PCG64 generator all ``n * 2 * L * L`` draws are made
    at once (in parallel chunks when many) and compared as integers.
    """
    if not 0.0 <= p <= 1.0:
        raise ValueError(f"p must lie in [0, 1], got {p}")
    if rng is None:
        rng = np.random.default_rng()
    n = int(n)
    if n > 0 and _fast_path(rng, p):
        # Groups of realizations of at most _GROUP_DRAWS draws (256 MB of raw
        # draws), one after the other, so the stream order is kept.
        per = 2 * L * L
        group = max(1, _GROUP_DRAWS // per)
        out = []
        for k0 in range(0, n, group):
            m = min(group, n - k0)
            neg = _pcg64_compare(rng, m * per, p).view(np.int8).reshape(m, 2, L, L)
            J = np.int8(1) - (neg + neg)
            out += [(J[k, 0], J[k, 1]) for k in range(m)]
        return out
    out = []
    for _ in range(n):
        J_h = np.where(rng.random((L, L)) < p, -1, 1).astype(np.int8)
        J_v = np.where(rng.random((L, L)) < p, -1, 1).astype(np.int8)
        out.append((J_h, J_v))
    return out


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
