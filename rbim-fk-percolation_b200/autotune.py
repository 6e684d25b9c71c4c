"""Launch-shape autotuner for the on-chip engines.

* Resident engine (one lattice per CTA): the CTA size -- threads per lattice,
  hence sites per thread -- is a free parameter whose best value depends on
  the lattice size and on the device.  ``rbim_sweeps_batched`` picks it by a
  fixed rule when called with ``threads = 0``.
* Cluster engine (one lattice per thread-block cluster): the plan -- CTAs per
  cluster and CTA size, hence the tile shape, the number of tile boundaries
  the merge stage handles, and the CTAs per SM -- is picked by a fixed rule
  in ``rbim_sweeps_clustered``; ``rbim_cluster_plans`` lists the others the
  device can run.

This module times the candidates instead, on a synthetic batch of lattices of
the launch's largest L, once per (device, L), and keeps the winner.  Results
do not depend on either choice (canonical labels, sums in sweep order, the
same Philox numbers on every tile split), so tuning changes speed only.

Use ``enable()`` (or set ``RBIM_AUTOTUNE=1``) to make ``ChainSet.run_batched``
and the scan server consult the tuner for every on-chip launch;
``RBIM_TUNE_CACHE`` names a JSON file that keeps the choices across processes.
"""

from __future__ import annotations

import json
import os
import threading
from typing import Dict, Optional, Sequence

import numpy as np

__all__ = ["CANDIDATES", "size_class", "enabled", "enable", "disable", "tuned_threads", "tune", "cache",
           "tune_cluster", "tuned_cluster_plan"]

#: CTA sizes the resident engine accepts.
CANDIDATES = (32, 64, 128, 256, 512, 1024)

_lock = threading.Lock()
# "<device>|<L>" -> CTA size; "<device>|cluster|<L>" -> [CTAs per cluster, CTA size]
_cache: Dict[str, object] = {}
_plans: Dict[str, list] = {}  # "<device>|<L>" -> the plans rbim_cluster_plans lists
_enabled = os.environ.get("RBIM_AUTOTUNE", "") not in ("", "0")
_loaded = False


def size_class(L: int) -> int:
    """The power of two >= L (at least 16): lattices of one class share a tuned CTA size."""
    return max(16, 1 << (int(L) - 1).bit_length())


def _key(device_name: str, L: int) -> str:
    return f"{device_name}|{L}"


def _cluster_key(device_name: str, L: int) -> str:
    return f"{device_name}|cluster|{L}"


def _valid(key: str, v) -> bool:
    if "|cluster|" in key:
        return isinstance(v, (list, tuple)) and len(v) == 2 and all(isinstance(x, int) for x in v) and \
            v[1] in (512, 1024) and 2 <= v[0] <= 16
    return isinstance(v, int) and v in CANDIDATES


def _cache_path() -> Optional[str]:
    return os.environ.get("RBIM_TUNE_CACHE") or None


def _load() -> None:
    global _loaded
    if _loaded:
        return
    _loaded = True
    path = _cache_path()
    if path and os.path.exists(path):
        try:
            with open(path) as f:
                data = json.load(f)
            _cache.update({str(k): v for k, v in data.items() if _valid(str(k), v)})
        except (OSError, ValueError, TypeError):
            pass


def _save() -> None:
    path = _cache_path()
    if not path:
        return
    tmp = f"{path}.tmp{os.getpid()}"
    with open(tmp, "w") as f:
        json.dump(_cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def cache() -> Dict[str, object]:
    """A copy of the tuned choices: ``"<device name>|<L>"`` -> CTA size of the resident engine,
    ``"<device name>|cluster|<L>"`` -> ``[CTAs per cluster, CTA size]`` of the cluster engine."""
    with _lock:
        _load()
        return dict(_cache)


def enabled() -> bool:
    return _enabled


def enable() -> None:
    global _enabled
    _enabled = True


def disable() -> None:
    global _enabled
    _enabled = False


def _time_candidate(rb, L: int, threads: int, device, n_chains: int, sweeps: int) -> float:
    import torch

    rng = np.random.default_rng(L)
    n_real = max(1, n_chains // 8)
    couplings = [rb.packing.pack_couplings(np.where(rng.random(2 * L * L) < 0.05, -1, 1).astype(np.int8), L)
                 for _ in range(n_real)]
    temps = np.linspace(1.4, 2.6, 8)
    specs = [rb.ChainSpec(L=L, realization=k % n_real, key=7919 * (k + 1), beta=1.0 / temps[k % 8], n_therm=0,
                          n_bins=1, sweeps_per_bin=10 * sweeps + 10) for k in range(n_chains)]
    cs = rb.ChainSet(specs, couplings, device=device)
    cs.init_spins(hot=True)
    cs._run_batched_fixed(1, threads)
    torch.cuda.synchronize(cs.device)
    best = float("inf")
    for _ in range(3):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        cs._run_batched_fixed(sweeps, threads)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    cs.check_status()
    return best


def tune(L: int, device=None, candidates: Sequence[int] = CANDIDATES, sweeps: int = 3,
         n_chains: Optional[int] = None) -> int:
    """Time every candidate CTA size on a synthetic batch of L x L lattices; return and remember the fastest."""
    import torch

    from . import engine

    rb = engine._package()
    dev = engine.require_cuda(device)
    cls = min(int(L), rb._native.resident_max_l())
    name = torch.cuda.get_device_name(dev)
    if n_chains is None:
        # Enough lattices to keep every SM busy at the smallest CTA size, so
        # that the timing measures throughput rather than one chain's latency.
        per_sm = max(2, min(16, 2 * (65536 // (cls * cls))))
        n_chains = per_sm * torch.cuda.get_device_properties(dev).multi_processor_count
    times = {}
    for t in candidates:
        times[t] = _time_candidate(rb, cls, int(t), dev, n_chains, sweeps)
    best = min(times, key=times.get)
    with _lock:
        _load()
        _cache[_key(name, cls)] = int(best)
        _save()
    return int(best)


def tuned_threads(L: int, device) -> int:
    """The tuned CTA size for L x L lattices on ``device``, tuning it on first use; 0 when tuning is off."""
    if not _enabled:
        return 0
    import torch

    name = torch.cuda.get_device_name(device)
    key = _key(name, int(L))
    with _lock:
        _load()
        if key in _cache:
            return _cache[key]
    return tune(L, device)


# ---------------------------------------------------------------------------
# Cluster engine plans.
# ---------------------------------------------------------------------------
def plans(L: int, device) -> list:
    """The plans ``(CTAs per cluster, CTA size)`` that can run an L x L lattice on ``device``, default first."""
    import torch

    from . import engine

    rb = engine._package()
    dev = engine.require_cuda(device)
    key = _key(torch.cuda.get_device_name(dev), int(L))
    with _lock:
        if key in _plans:
            return list(_plans[key])
    with torch.cuda.device(dev):
        found = rb._native.cluster_plans(int(L))
    with _lock:
        _plans[key] = found
    return list(found)


def _time_plan(rb, L: int, plan, device, n_chains: int, sweeps: int) -> float:
    import torch

    rng = np.random.default_rng(L)
    n_real = max(1, n_chains // 4)
    couplings = [rb.packing.pack_couplings(np.where(rng.random(2 * L * L) < 0.05, -1, 1).astype(np.int8), L)
                 for _ in range(n_real)]
    temps = np.linspace(1.4, 2.6, 4)
    specs = [rb.ChainSpec(L=L, realization=k % n_real, key=104729 * (k + 1), beta=1.0 / temps[k % 4], n_therm=0,
                          n_bins=1, sweeps_per_bin=10 * sweeps + 10) for k in range(n_chains)]
    cs = rb.ChainSet(specs, couplings, device=device)
    cs.init_spins(hot=True)
    cs._run_batched_fixed(1, 0, cluster_plan=plan)
    torch.cuda.synchronize(cs.device)
    best = float("inf")
    for _ in range(2):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        cs._run_batched_fixed(sweeps, 0, cluster_plan=plan)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    cs.check_status()
    return best


def tune_cluster(L: int, device=None, sweeps: int = 2, n_chains: Optional[int] = None, candidates=None):
    """Time every plan of ``plans(L)`` (or ``candidates``) on a synthetic batch of L x L lattices; return and
    remember the fastest ``(CTAs per cluster, CTA size)``."""
    import torch

    from . import engine

    rb = engine._package()
    dev = engine.require_cuda(device)
    name = torch.cuda.get_device_name(dev)
    cands = [tuple(c) for c in (candidates or plans(L, dev))]
    if not cands:
        raise ValueError(f"no cluster plan can run L = {L} on this device")
    if n_chains is None:
        # Two full waves of the plan with the fewest CTAs per cluster.
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        n_chains = max(8, 2 * sms // min(c for c, _ in cands))
    times = {c: _time_plan(rb, int(L), c, dev, n_chains, sweeps) for c in cands}
    best = min(times, key=times.get)
    with _lock:
        _load()
        _cache[_cluster_key(name, int(L))] = [int(best[0]), int(best[1])]
        _save()
    return (int(best[0]), int(best[1]))


def tuned_cluster_plan(l_max: int, sizes: Sequence[int], device):
    """The tuned plan of a cluster launch of lattices ``sizes`` (largest ``l_max``), tuning it on first use; None
    when tuning is off, or when the tuned plan cannot run every size of the launch (the default plan then runs)."""
    if not _enabled:
        return None
    import torch

    name = torch.cuda.get_device_name(device)
    key = _cluster_key(name, int(l_max))
    with _lock:
        _load()
        plan = _cache.get(key)
    if plan is None:
        plan = tune_cluster(int(l_max), device)
    plan = (int(plan[0]), int(plan[1]))
    if all(plan in [tuple(p) for p in plans(L, device)] for L in sizes):
        return plan
    return None
