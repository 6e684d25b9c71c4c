"""Launch-shape autotuner for the resident engine.

The resident engine runs one lattice per CTA; the CTA size (threads per
lattice, hence sites per thread) is a free parameter whose best value depends
on the lattice size and on the device.  ``rbim_sweeps_batched`` picks it by a
fixed rule when called with ``threads = 0``; this module times the candidates
instead, on a synthetic batch of lattices of the launch's largest L, once per
(device, L), and keeps the winner.  Results do not depend on the CTA size (canonical
labels, sums in sweep order), so tuning changes speed only.

Use ``enable()`` (or set ``RBIM_AUTOTUNE=1``) to make ``ChainSet.run_batched``
consult the tuner for every resident launch; ``RBIM_TUNE_CACHE`` names a JSON
file that keeps the choices across processes.
"""

from __future__ import annotations

import json
import os
import threading
from typing import Dict, Optional, Sequence

import numpy as np

__all__ = ["CANDIDATES", "size_class", "enabled", "enable", "disable", "tuned_threads", "tune", "cache"]

#: CTA sizes the resident engine accepts.
CANDIDATES = (64, 128, 256, 512, 1024)

_lock = threading.Lock()
_cache: Dict[str, int] = {}
_enabled = os.environ.get("RBIM_AUTOTUNE", "") not in ("", "0")
_loaded = False


def size_class(L: int) -> int:
    """The power of two >= L (at least 16): lattices of one class share a tuned CTA size."""
    return max(16, 1 << (int(L) - 1).bit_length())


def _key(device_name: str, L: int) -> str:
    return f"{device_name}|{L}"


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
            _cache.update({str(k): int(v) for k, v in data.items() if int(v) in CANDIDATES})
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


def cache() -> Dict[str, int]:
    """A copy of the tuned choices, keyed ``"<device name>|<L>"``."""
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
