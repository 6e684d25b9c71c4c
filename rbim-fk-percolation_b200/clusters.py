"""FK bond activation, labelling and percolation tests on the GPU (mirror of ``src/rbim/clusters.py``).

``activate_bonds`` and ``label_and_wrap`` are the kernel-level seams of the
sweep: they run the same device code as the sweep engines, on one lattice at a
time, and are what the bit-exact parity tests call.  ``cluster_statistics`` is
a host helper on labels the caller already holds, as in the reference.
"""

from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import numpy as np

from . import _native
from .engine import require_cuda
from .lattice import Lattice
from .packing import pack_couplings, pack_spins, threshold

__all__ = [
    "bond_activation_probability",
    "activate_bonds",
    "label_clusters",
    "label_and_wrap",
    "label_and_wrap_many",
    "cluster_statistics",
    "wraps_along",
    "spans_along",
]


def _torch():
    import torch

    return torch


def bond_activation_probability(beta: float) -> float:
    """``1 - exp(-2 beta)`` via ``expm1`` (reference ``clusters.py:40-45``)."""
    return float(-np.expm1(-2.0 * beta))


def _stream(dev):
    return ctypes.c_void_p(_torch().cuda.current_stream(dev).cuda_stream)


def activate_bonds(spins: np.ndarray, lattice: Lattice, J: np.ndarray, beta: float, rng=None, *,
                   key: Optional[int] = None, sweep: int = 0, device=None) -> np.ndarray:
    """Occupied FK bonds for ``spins`` (reference ``clusters.py:48-79``), drawn on the GPU.

    The uniforms come from the Philox stream of ``key`` at sweep counter
    ``sweep`` (bond ``k`` uses word ``k & 3`` of block ``k >> 2``).  When
    ``key`` is omitted it is drawn from ``rng`` (a numpy ``Generator``), which
    is consumed the way the reference consumes its generator.
    """
    torch = _torch()
    dev = require_cuda(device)
    L = lattice.L
    if key is None:
        if rng is None:
            raise ValueError("activate_bonds needs a key or a numpy Generator")
        key = int(rng.integers(0, 2**63, dtype=np.int64))
    lib = _native.lib()
    s = torch.from_numpy(pack_spins(spins, L).view(np.int32)).to(dev)
    j = torch.from_numpy(pack_couplings(J, L).view(np.int32)).to(dev)
    occ = torch.empty(2 * L * L, dtype=torch.uint8, device=dev)
    nbytes = int(lib.rbim_activate_workspace_bytes(L))
    ws = torch.empty(max(nbytes, 16), dtype=torch.uint8, device=dev)
    with torch.cuda.device(dev):
        rc = lib.rbim_activate(L, ctypes.c_void_p(s.data_ptr()), ctypes.c_void_p(j.data_ptr()), int(key) & (2**64 - 1),
                               threshold(beta), int(sweep), ctypes.c_void_p(occ.data_ptr()),
                               ctypes.c_void_p(ws.data_ptr()), ws.numel(), _stream(dev))
    _native.check(rc, "rbim_activate")
    return occ.cpu().numpy().astype(bool)


def label_and_wrap_many(active: np.ndarray, L: int, device=None):
    """Label many frozen masks of one size at once.

    ``active`` has shape ``(n, 2*L*L)``.  Returns ``(n_clusters (n,) int64,
    labels (n, L*L) int64, wraps (n, 2) bool)``.
    """
    torch = _torch()
    dev = require_cuda(device)
    a = np.ascontiguousarray(np.asarray(active).reshape(-1, 2 * L * L), dtype=np.uint8)
    n = a.shape[0]
    lib = _native.lib()
    occ = torch.from_numpy(a).to(dev)
    labels = torch.empty((n, L * L), dtype=torch.int32, device=dev)
    ncl = torch.empty(n, dtype=torch.int32, device=dev)
    wraps = torch.empty((n, 2), dtype=torch.uint8, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    nbytes = int(lib.rbim_label_wrap_workspace_bytes(L))
    ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=dev)
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    with torch.cuda.device(dev):
        rc = lib.rbim_label_wrap(L, n, p(occ), p(labels), p(ncl), p(wraps), p(status), p(ws), ws.numel(), _stream(dev))
    _native.check(rc, "rbim_label_wrap")
    st = int(status.item())
    if st:
        raise _native.RbimError(f"rbim_label_wrap device status {st:#x}")
    return (ncl.cpu().numpy().astype(np.int64), labels.cpu().numpy().astype(np.int64),
            wraps.cpu().numpy().astype(bool))


def label_and_wrap(active: np.ndarray, lattice: Lattice) -> Tuple[int, np.ndarray, bool, bool]:
    """Canonical labels and both wrap flags of one mask (reference ``clusters.py:144-159``).

    Returns ``(n_clusters, labels, wraps_x, wraps_y)``; clusters are numbered in
    order of their smallest site, as the reference's union-find numbers them.
    """
    ncl, labels, wraps = label_and_wrap_many(active, lattice.L)
    return int(ncl[0]), labels[0], bool(wraps[0, 0]), bool(wraps[0, 1])


def label_clusters(active: np.ndarray, lattice: Lattice) -> Tuple[int, np.ndarray]:
    """``(n_clusters, labels)`` (reference ``clusters.py:82-95``; same canonical numbering)."""
    n, labels, _, _ = label_and_wrap(active, lattice)
    return n, labels


def cluster_statistics(labels: np.ndarray, spins: np.ndarray, n_clusters: int):
    """Size and signed magnetization of every cluster (host; reference ``clusters.py:98-118``)."""
    sizes = np.bincount(labels, minlength=n_clusters)
    magnetizations = np.bincount(labels, weights=spins.astype(np.float64), minlength=n_clusters)
    return sizes, magnetizations


def wraps_along(active: np.ndarray, lattice: Lattice, axis: str) -> bool:
    """Exact winding test along ``axis`` (reference ``clusters.py:121-141``)."""
    _, _, wx, wy = label_and_wrap(active, lattice)
    if axis == "x":
        return bool(wx)
    if axis == "y":
        return bool(wy)
    raise ValueError(f"axis must be 'x' or 'y', got {axis!r}")


def spans_along(active: np.ndarray, lattice: Lattice, axis: str) -> bool:
    """Spanning along ``axis``: seam bonds removed, a cluster touches both open faces.

    Reference ``clusters.py:162-180``; the labelling runs on the GPU.
    """
    wrap_mask = lattice.wrap_mask(axis)
    _, labels, _, _ = label_and_wrap(np.asarray(active, dtype=bool) & ~wrap_mask, lattice)
    L = lattice.L
    sites = np.arange(lattice.n_sites)
    coordinate = sites // L if axis == "x" else sites % L
    low = np.unique(labels[coordinate == 0])
    high = np.unique(labels[coordinate == L - 1])
    return bool(np.intersect1d(low, high, assume_unique=True).size > 0)
