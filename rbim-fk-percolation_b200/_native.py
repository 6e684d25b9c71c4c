"""ctypes binding of ``librbim_sm100.so``, the C ABI declared in ``include/rbim_sm100.h``.

There is no CPU fallback: every compute entry point goes through this library
and raises if it is missing or if no CUDA device is present.
"""

from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

from . import build as _build

__all__ = [
    "RbimError",
    "lib",
    "check",
    "CHAIN_DTYPE",
    "ACC_INT",
    "ACC_F64",
    "REC_LEN",
    "plane_words",
    "resident_max_l",
    "cluster_max_l",
    "cluster_plans",
    "engine_buckets",
    "EXPORTED_SYMBOLS",
]

ACC_INT = 12
ACC_F64 = 2
REC_LEN = 9

#: numpy mirror of ``rbim_chain_t`` (96 bytes, every field 8 bytes).
CHAIN_DTYPE = np.dtype(
    [
        ("key", "<u8"),
        ("thr", "<u8"),
        ("spin_off", "<i8"),
        ("coupling_off", "<i8"),
        ("acc_off", "<i8"),
        ("rec_off", "<i8"),
        ("sweep", "<u8"),
        ("n_therm", "<i8"),
        ("n_bins", "<i8"),
        ("sweeps_per_bin", "<i8"),
        ("L", "<i8"),
        ("walk_cap", "<i8"),
    ]
)
assert CHAIN_DTYPE.itemsize == 96

#: Every function ``include/rbim_sm100.h`` declares.
EXPORTED_SYMBOLS = (
    "rbim_last_error",
    "rbim_abi_version",
    "rbim_plane_words",
    "rbim_resident_max_l",
    "rbim_resident_threads",
    "rbim_init_spins",
    "rbim_activate_workspace_bytes",
    "rbim_activate",
    "rbim_label_wrap_workspace_bytes",
    "rbim_label_wrap",
    "rbim_batched_workspace_bytes",
    "rbim_sweeps_batched",
    "rbim_plain_workspace_bytes",
    "rbim_sweeps_plain",
    "rbim_cluster_max_l",
    "rbim_cluster_size",
    "rbim_cluster_threads",
    "rbim_sweeps_clustered",
    "rbim_cluster_plans",
    "rbim_sweeps_clustered_plan",
    "rbim_noalloc_max_l",
    "rbim_sweeps_plain_noalloc",
    "rbim_grid_plan",
    "rbim_grid_workspace_bytes",
    "rbim_sweeps_grid",
)


class RbimError(RuntimeError):
    """A call into the CUDA engine failed."""


_lock = threading.Lock()
_lib = None


def _declare(l):
    c_int, c_i64, c_u64, c_size, p = ctypes.c_int, ctypes.c_int64, ctypes.c_uint64, ctypes.c_size_t, ctypes.c_void_p
    l.rbim_last_error.restype = ctypes.c_char_p
    l.rbim_last_error.argtypes = []
    l.rbim_abi_version.restype = c_int
    l.rbim_abi_version.argtypes = []
    l.rbim_plane_words.restype = c_i64
    l.rbim_plane_words.argtypes = [c_i64]
    l.rbim_resident_max_l.restype = c_int
    l.rbim_resident_max_l.argtypes = []
    l.rbim_resident_threads.restype = c_int
    l.rbim_resident_threads.argtypes = [c_i64]
    l.rbim_init_spins.restype = c_int
    l.rbim_init_spins.argtypes = [p, c_int, p, c_int, p]
    l.rbim_activate_workspace_bytes.restype = c_size
    l.rbim_activate_workspace_bytes.argtypes = [c_i64]
    l.rbim_activate.restype = c_int
    l.rbim_activate.argtypes = [c_i64, p, p, c_u64, c_u64, c_u64, p, p, c_size, p]
    l.rbim_label_wrap_workspace_bytes.restype = c_size
    l.rbim_label_wrap_workspace_bytes.argtypes = [c_i64]
    l.rbim_label_wrap.restype = c_int
    l.rbim_label_wrap.argtypes = [c_i64, c_int, p, p, p, p, p, p, c_size, p]
    l.rbim_batched_workspace_bytes.restype = c_size
    l.rbim_batched_workspace_bytes.argtypes = []
    l.rbim_sweeps_batched.restype = c_int
    l.rbim_sweeps_batched.argtypes = [p, c_int, c_i64, p, p, p, p, p, c_int, c_int, p, p, c_size, p]
    l.rbim_plain_workspace_bytes.restype = c_size
    l.rbim_plain_workspace_bytes.argtypes = [c_i64]
    l.rbim_sweeps_plain.restype = c_int
    l.rbim_sweeps_plain.argtypes = [c_i64, p, p, p, p, p, p, c_int, p, p, c_size, p]
    l.rbim_cluster_max_l.restype = c_int
    l.rbim_cluster_max_l.argtypes = []
    l.rbim_cluster_size.restype = c_int
    l.rbim_cluster_size.argtypes = [c_i64]
    l.rbim_cluster_threads.restype = c_int
    l.rbim_cluster_threads.argtypes = [c_i64]
    l.rbim_sweeps_clustered.restype = c_int
    l.rbim_sweeps_clustered.argtypes = [p, c_int, c_i64, p, p, p, p, p, c_int, p, p, c_size, p]
    l.rbim_cluster_plans.restype = c_int
    l.rbim_cluster_plans.argtypes = [c_i64, p, p, c_int]
    l.rbim_sweeps_clustered_plan.restype = c_int
    l.rbim_sweeps_clustered_plan.argtypes = [p, c_int, c_i64, c_int, c_int, p, p, p, p, p, c_int, p, p, c_size, p]
    l.rbim_noalloc_max_l.restype = c_int
    l.rbim_noalloc_max_l.argtypes = []
    l.rbim_sweeps_plain_noalloc.restype = c_int
    l.rbim_sweeps_plain_noalloc.argtypes = [c_i64, p, p, p, p, p, p, c_int, p, p]
    l.rbim_grid_plan.restype = c_int
    l.rbim_grid_plan.argtypes = [c_i64, p, p]
    l.rbim_grid_workspace_bytes.restype = c_size
    l.rbim_grid_workspace_bytes.argtypes = [c_i64, c_int]
    l.rbim_sweeps_grid.restype = c_int
    l.rbim_sweeps_grid.argtypes = [c_i64, p, p, p, p, p, p, c_int, p, c_int, c_int, c_i64, p, c_size, p]


def lib(build_if_missing: bool = True):
    """The loaded library (built from ``csrc/`` first if it is missing or stale).

    ``RBIM_LIBRARY`` in the environment names another build of the same ABI
    to load instead (a profiling or debug build).
    """
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = os.environ.get("RBIM_LIBRARY") or _build.LIB
        if build_if_missing and not os.environ.get("RBIM_LIBRARY"):
            try:
                path = _build.build()
            except Exception as exc:  # pragma: no cover - depends on the toolchain
                if not os.path.exists(path):
                    raise RbimError(f"librbim_sm100.so is missing and could not be built: {exc}") from exc
        if not os.path.exists(path):
            raise RbimError(f"librbim_sm100.so not found at {path}")
        l = ctypes.CDLL(path)
        _declare(l)
        _lib = l
        return l


def check(rc: int, what: str) -> None:
    """Raise :class:`RbimError` with the library's message when ``rc`` is not RBIM_OK."""
    if rc != 0:
        msg = lib().rbim_last_error().decode(errors="replace")
        raise RbimError(f"{what} failed ({rc}): {msg}")


def plane_words(L: int) -> int:
    """Words of one bit plane (``rbim_plane_words``)."""
    return int(lib().rbim_plane_words(int(L)))


def resident_max_l() -> int:
    """Largest L the on-chip engine takes (``rbim_resident_max_l``)."""
    return int(lib().rbim_resident_max_l())


def engine_buckets(Ls, r_max: int, c_max: int):
    """Launch bucket of every lattice size: a tuple ``(kind, ...)`` with kind 0 resident, 1 cluster, 2 plain.

    Resident lattices are bucketed by their default CTA size
    (``rbim_resident_threads``; the launch sizes its CTAs and shared memory
    for the bucket's largest L), cluster lattices by CTAs per cluster and CTA
    size (``rbim_cluster_size``, ``rbim_cluster_threads``: a launch runs every
    lattice in the plan of its largest L); buckets sort in launch order.
    """
    key_of = {}
    for L in set(int(L) for L in Ls):
        if L <= r_max:
            key_of[L] = (0, int(lib().rbim_resident_threads(L)))
        elif L <= c_max:
            key_of[L] = (1, int(lib().rbim_cluster_size(L)), int(lib().rbim_cluster_threads(L)))
        else:
            key_of[L] = (2, 0)
    return [key_of[int(L)] for L in Ls]


def cluster_plans(L: int):
    """Cluster-engine plans ``(CTAs per cluster, CTA size)`` that can run an L x L lattice on the current device,
    the default plan first (``rbim_cluster_plans``)."""
    import ctypes

    l = lib()
    n = int(l.rbim_cluster_plans(int(L), None, None, 0))
    if n <= 0:
        return []
    c = (ctypes.c_int * n)()
    t = (ctypes.c_int * n)()
    l.rbim_cluster_plans(int(L), c, t, n)
    return [(int(c[i]), int(t[i])) for i in range(n)]


def grid_plan(L: int):
    """Default grid-engine plan ``(CTAs, CTA size)`` for one L x L lattice on the current device, or None
    (``rbim_grid_plan``)."""
    import ctypes

    c, t = ctypes.c_int(0), ctypes.c_int(0)
    if lib().rbim_grid_plan(int(L), ctypes.byref(c), ctypes.byref(t)) != 0:
        return None
    return int(c.value), int(t.value)


def cluster_max_l() -> int:
    """Largest L the cluster engine takes on the current device (``rbim_cluster_max_l``; 0 if none)."""
    return int(lib().rbim_cluster_max_l())
