"""ctypes wrapper around the C oracle ``rbim_oracle.c`` (test infrastructure only).

Every function here is the CPU restatement of one reference function; the
citation is on the C side.  Arrays follow the reference layout: spins are int8
``+-1`` of shape ``(N,)``, couplings int8 ``+-1`` of shape ``(2N,)`` in bond
order (``lattice.py:138-161``), occupation masks bool ``(2N,)``.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

__all__ = [
    "ORACLE_LIB",
    "build_oracle",
    "load",
    "philox4x32_10",
    "bond_uniform",
    "flip_bit",
    "hot_spin_bit",
    "activate",
    "label_and_wrap",
    "cluster_statistics",
    "two_largest",
    "energy",
    "magnetization",
    "sw_sweep",
    "initial_spins",
    "run_chain",
    "run_chains",
    "label_many",
    "N_INT",
    "N_F64",
    "SweepRecord",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "rbim_oracle.c")
ORACLE_LIB = os.path.join(_HERE, "librbim_oracle.so")

N_INT = 12
N_F64 = 2

_lock = threading.Lock()
_lib = None


def build_oracle(force: bool = False) -> str:
    """Compile ``rbim_oracle.c`` into ``librbim_oracle.so`` next to it."""
    if not force and os.path.exists(ORACLE_LIB) and os.path.getmtime(ORACLE_LIB) >= os.path.getmtime(_SRC):
        return ORACLE_LIB
    tmp = ORACLE_LIB + f".tmp{os.getpid()}"
    cmd = ["gcc", "-O3", "-march=x86-64-v2", "-fopenmp", "-shared", "-fPIC", "-std=c11", "-o", tmp, _SRC]
    subprocess.run(cmd, check=True)
    os.replace(tmp, ORACLE_LIB)
    return ORACLE_LIB


def load():
    """Load (building if needed) the oracle shared library."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        build_oracle()
        lib = ctypes.CDLL(ORACLE_LIB)
        i64, u64, i32, p = ctypes.c_int64, ctypes.c_uint64, ctypes.c_int32, ctypes.c_void_p
        lib.orc_philox4x32_10.argtypes = [p, p, p]
        lib.orc_bond_uniform.argtypes = [u64, u64, u64]
        lib.orc_bond_uniform.restype = ctypes.c_uint32
        lib.orc_flip_bit.argtypes = [u64, u64, u64]
        lib.orc_flip_bit.restype = ctypes.c_int
        lib.orc_hot_spin_bit.argtypes = [u64, u64]
        lib.orc_hot_spin_bit.restype = ctypes.c_int
        lib.orc_activate.argtypes = [i64, p, p, u64, u64, u64, p]
        lib.orc_label_and_wrap.argtypes = [i64, p, p, p, p]
        lib.orc_label_and_wrap.restype = i64
        lib.orc_cluster_statistics.argtypes = [i64, p, p, i64, p, p]
        lib.orc_two_largest.argtypes = [p, i64, p, p]
        lib.orc_energy.argtypes = [i64, p, p]
        lib.orc_energy.restype = i64
        lib.orc_magnetization.argtypes = [i64, p]
        lib.orc_magnetization.restype = i64
        lib.orc_sw_sweep.argtypes = [i64, p, p, u64, u64, u64, ctypes.c_int, p]
        lib.orc_initial_spins.argtypes = [i64, u64, ctypes.c_int, p]
        lib.orc_run_chain.argtypes = [i64, p, u64, u64, ctypes.c_int, u64, i64, i64, i64, p, ctypes.c_int, p, p]
        lib.orc_run_chains.argtypes = [i64, i64, p, p, p, ctypes.c_int, u64, i64, i64, i64, p, ctypes.c_int, p, p,
                                       ctypes.c_int]
        lib.orc_run_chains.restype = ctypes.c_int
        lib.orc_label_many.argtypes = [i64, i64, p, p, p, ctypes.c_int]
        lib.orc_label_many.restype = ctypes.c_int
        _ = i32
        _lib = lib
        return lib


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.c_void_p)


def philox4x32_10(ctr, key) -> np.ndarray:
    """Philox4x32-10 block: four 32-bit counter words and two key words."""
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    load().orc_philox4x32_10(_ptr(c), _ptr(k), _ptr(out))
    return out


def bond_uniform(key: int, sweep: int, bond: int) -> int:
    return int(load().orc_bond_uniform(key, sweep, bond))


def flip_bit(key: int, sweep: int, root: int) -> int:
    return int(load().orc_flip_bit(key, sweep, root))


def hot_spin_bit(key: int, site: int) -> int:
    return int(load().orc_hot_spin_bit(key, site))


def activate(L: int, spins: np.ndarray, J: np.ndarray, key: int, thr: int, sweep: int) -> np.ndarray:
    """Philox replay of ``activate_bonds`` (``clusters.py:48-79``)."""
    s = np.ascontiguousarray(spins, dtype=np.int8)
    j = np.ascontiguousarray(J, dtype=np.int8)
    occ = np.zeros(2 * L * L, dtype=np.uint8)
    load().orc_activate(L, _ptr(s), _ptr(j), key, thr, sweep, _ptr(occ))
    return occ.astype(bool)


def label_and_wrap(active: np.ndarray, L: int):
    """Restatement of ``_label_and_wrap`` (``_unionfind.py:91-136``).

    Returns ``(n_clusters, labels int64 (N,), wraps_x, wraps_y)``.
    """
    occ = np.ascontiguousarray(active, dtype=np.uint8)
    if occ.size != 2 * L * L:
        raise ValueError("active must have 2*L*L entries")
    labels = np.empty(L * L, dtype=np.int64)
    wx = np.zeros(1, dtype=np.int32)
    wy = np.zeros(1, dtype=np.int32)
    n = load().orc_label_and_wrap(L, _ptr(occ), _ptr(labels), _ptr(wx), _ptr(wy))
    return int(n), labels, bool(wx[0]), bool(wy[0])


def cluster_statistics(labels: np.ndarray, spins: np.ndarray, n_clusters: int):
    """Restatement of ``cluster_statistics`` (``clusters.py:98-118``), integer mags."""
    lab = np.ascontiguousarray(labels, dtype=np.int64)
    s = np.ascontiguousarray(spins, dtype=np.int8)
    sizes = np.zeros(n_clusters, dtype=np.int64)
    mags = np.zeros(n_clusters, dtype=np.int64)
    load().orc_cluster_statistics(lab.size, _ptr(lab), _ptr(s), n_clusters, _ptr(sizes), _ptr(mags))
    return sizes, mags


def two_largest(sizes: np.ndarray):
    """``_two_largest`` (``swendsen_wang.py:92-100``) with the smallest-label tie rule."""
    sz = np.ascontiguousarray(sizes, dtype=np.int64)
    f = np.zeros(1, dtype=np.int64)
    s = np.zeros(1, dtype=np.int64)
    load().orc_two_largest(_ptr(sz), sz.size, _ptr(f), _ptr(s))
    return int(f[0]), (None if s[0] < 0 else int(s[0]))


def energy(L: int, spins: np.ndarray, J: np.ndarray) -> int:
    s = np.ascontiguousarray(spins, dtype=np.int8)
    j = np.ascontiguousarray(J, dtype=np.int8)
    return int(load().orc_energy(L, _ptr(s), _ptr(j)))


def magnetization(spins: np.ndarray) -> int:
    s = np.ascontiguousarray(spins, dtype=np.int8)
    return int(load().orc_magnetization(s.size, _ptr(s)))


class SweepRecord(tuple):
    """(energy, magnetization, n_clusters, S1, |M_C1|, S2, |M_C2|, wraps_x, wraps_y)."""


def sw_sweep(L: int, spins: np.ndarray, J: np.ndarray, key: int, thr: int, sweep: int, measure: bool = True):
    """Philox replay of ``sw_sweep`` (``swendsen_wang.py:103-172``); updates ``spins`` in place."""
    if spins.dtype != np.int8 or not spins.flags["C_CONTIGUOUS"]:
        raise TypeError("spins must be a contiguous int8 array")
    j = np.ascontiguousarray(J, dtype=np.int8)
    rec = np.zeros(9, dtype=np.int64)
    load().orc_sw_sweep(L, _ptr(spins), _ptr(j), key, thr, sweep, int(measure), _ptr(rec))
    return SweepRecord(int(v) for v in rec) if measure else None


def initial_spins(n_sites: int, key: int, hot: bool = True) -> np.ndarray:
    s = np.empty(n_sites, dtype=np.int8)
    load().orc_initial_spins(n_sites, key, int(hot), _ptr(s))
    return s


def run_chain(L, J, key, thr, *, hot=True, sweep0=0, n_therm, n_bins, sweeps_per_bin, spins=None):
    """Philox replay of ``run_single_realization``'s loop (``simulation.py:196-242``).

    Returns ``(int_bins (n_bins, 12) int64, f_bins (n_bins, 2) float64, spins)``.
    """
    j = np.ascontiguousarray(J, dtype=np.int8)
    init = spins is None
    s = np.empty(L * L, dtype=np.int8) if init else np.ascontiguousarray(spins, dtype=np.int8).copy()
    ib = np.zeros((n_bins, N_INT), dtype=np.int64)
    fb = np.zeros((n_bins, N_F64), dtype=np.float64)
    load().orc_run_chain(L, _ptr(j), key, thr, int(hot), sweep0, n_therm, n_bins, sweeps_per_bin, _ptr(s),
                         int(init), _ptr(ib), _ptr(fb))
    return ib, fb, s


def run_chains(L, J, keys, thrs, *, hot=True, sweep0=0, n_therm, n_bins, sweeps_per_bin, spins=None,
               n_threads=0):
    """Many chains in parallel on the host, one chain per thread (CPU baseline).

    ``J`` has shape ``(n_chains, 2N)``.  Returns ``(int_bins, f_bins, spins, threads_used)``.
    """
    j = np.ascontiguousarray(J, dtype=np.int8)
    n_chains = j.shape[0]
    k = np.ascontiguousarray(keys, dtype=np.uint64)
    t = np.ascontiguousarray(thrs, dtype=np.uint64)
    init = spins is None
    s = np.empty((n_chains, L * L), dtype=np.int8) if init else np.ascontiguousarray(spins, dtype=np.int8).copy()
    ib = np.zeros((n_chains, n_bins, N_INT), dtype=np.int64)
    fb = np.zeros((n_chains, n_bins, N_F64), dtype=np.float64)
    used = load().orc_run_chains(n_chains, L, _ptr(j), _ptr(k), _ptr(t), int(hot), sweep0, n_therm, n_bins,
                                 sweeps_per_bin, _ptr(s), int(init), _ptr(ib), _ptr(fb), int(n_threads))
    return ib, fb, s, int(used)


def label_many(L: int, masks: np.ndarray, n_threads: int = 0):
    """Label many frozen masks in parallel; returns ``(n_clusters, wraps (n,2), threads_used)``."""
    occ = np.ascontiguousarray(masks, dtype=np.uint8)
    n = occ.shape[0]
    ncl = np.zeros(n, dtype=np.int64)
    wr = np.zeros((n, 2), dtype=np.int32)
    used = load().orc_label_many(n, L, _ptr(occ), _ptr(ncl), _ptr(wr), int(n_threads))
    return ncl, wr.astype(bool), int(used)
