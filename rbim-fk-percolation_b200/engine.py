"""Device-resident chain sets and the two sweep engines behind the C ABI.

A *chain* is one disorder realization at one temperature, the task unit of the
reference's ``run_temperature_scan`` (``simulation.py:384-399``).  A
:class:`ChainSet` owns, in device memory, the spin planes of its chains, the
coupling planes of their realizations (shared by every temperature of a
realization), the ``rbim_chain_t`` descriptors, the per-bin accumulators and
optional per-sweep records; only accumulators (and, on request, spins and
records) ever come back to the host.  PyTorch provides the device memory and
the stream; every computation is a call into ``librbim_sm100.so``.
"""

from __future__ import annotations

import ctypes
import threading
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _native
from .packing import threshold, unpack_spins, words_for

__all__ = ["ChainSpec", "ChainSet", "chain_key", "require_cuda", "SINGLE_CTA_MAX_L", "single_cta_threads", "occupancy_threads", "auto_engine", "Launch",
           "launch_buckets"]

#: A set of one lattice runs under ``engine="auto"`` on one resident CTA when
#: L <= SINGLE_CTA_MAX_L, with the CTA size ``single_cta_threads(L)``, and
#: over the whole GPU above: on the grid engine where it has a plan for L, else
#: on the plain engine.  Measured on B200, one lattice, us per sweep: L = 32,
#: one CTA of 512 threads 16.5 (64 threads, the batch default, 32.7); L = 48,
#: one CTA of 1024 threads 22.8, grid engine 28.6; L = 64, 26.0 against 29.9;
#: L = 96, 42.9 against 32.2.
SINGLE_CTA_MAX_L = 64


def single_cta_threads(L: int) -> int:
    """CTA size for one lattice alone on the resident engine: the large sizes minimise the time per sweep (the
    batch default favours many CTAs per SM instead).  Measured on B200: 512 threads up to L = 32 (16.1 us at
    L = 24 and 16.5 at L = 32, against 17.3 with 1024), 1024 above (22.8 us at L = 48 against 25.9 with 512)."""
    return 512 if L <= 32 else 1024


_sm_counts = {}


def _sm_count(device) -> int:
    key = str(device)
    if key not in _sm_counts:
        _sm_counts[key] = int(_torch().cuda.get_device_properties(device).multi_processor_count)
    return _sm_counts[key]


def occupancy_threads(threads: int, n_lattices: int, sms: int) -> int:
    """Resident CTA size for a launch of ``n_lattices``: the library's default (small CTAs, many per SM: the most
    throughput when the lattices fill the GPU) doubled while every lattice of the launch would still be resident at
    once with twice the threads (at most 1024 threads a CTA, 1024 an SM), so that a launch of few lattices runs
    each on more threads.  Measured on B200, the reference's L = 32 scan (1280 lattices): one-warp CTAs 1.44 s,
    two-warp CTAs 1.01 s; the uneven-size mix (524,288 lattices of L = 32) is 3 % faster with one-warp CTAs."""
    while threads < 1024 and n_lattices * 2 * threads <= sms * 1024:
        threads *= 2
    return threads


def auto_engine(specs, grid_plan=None) -> str:
    """The engine ``engine="auto"`` picks for a set of chains: ``"batched"`` for several lattices, or one with
    L <= SINGLE_CTA_MAX_L (one resident CTA); for one larger lattice ``"grid"`` (one cooperative launch of tiles
    over every SM) where the grid engine has a plan for L on the current device, else ``"plain"``.
    ``grid_plan(L)`` returns the plan or None (default: ``_native.grid_plan``)."""
    specs = list(specs)
    if len(specs) != 1 or specs[0].L <= SINGLE_CTA_MAX_L:
        return "batched"
    return "grid" if (grid_plan or _native.grid_plan)(specs[0].L) else "plain"


def _torch():
    import torch

    return torch


def _package():
    import importlib

    return importlib.import_module(__package__)


#: Bytes of workspace per concurrent bucket launch: one work-queue counter.
QUEUE_SLOT = 256

_streams_lock = threading.Lock()
_side_streams = {}


def _side(device, n: int):
    """``n`` side streams of ``device``, created once per process and reused."""
    torch = _torch()
    with _streams_lock:
        pool = _side_streams.setdefault(device.index, [])
        while len(pool) < n:
            pool.append(torch.cuda.Stream(device))
        return pool[:n]


@dataclass
class Launch:
    """One on-chip launch of a call: ``kind`` 0 resident (``rbim_sweeps_batched``) or 1 cluster
    (``rbim_sweeps_clustered``), over ``count`` consecutive descriptors at device address ``chains``.
    A cluster launch with ``ctas > 0`` runs the plan (``ctas`` CTAs of ``threads``) through
    ``rbim_sweeps_clustered_plan``."""

    kind: int
    chains: int
    count: int
    l_max: int
    threads: int = 0
    ctas: int = 0


def launch_buckets(lib, device, stream, launches: Sequence[Launch], *, spin_pool: int, coupling_pool: int,
                   acc_int: int, acc_f64: int, records: Optional[int], n_sweeps: int, status: int, workspace: int,
                   workspace_bytes: int, concurrent: bool = True) -> None:
    """Advance every bucket of a call by ``n_sweeps``, the buckets running concurrently.

    Each launch is a persistent grid that pulls lattices from its own work
    queue (slot ``i`` of ``QUEUE_SLOT`` bytes of the workspace) and exits when
    the queue is empty; with several buckets they are issued on side streams
    forked from ``stream`` and joined back into it, so that a bucket's CTAs
    take the SMs that another bucket's tail leaves idle instead of waiting for
    the whole previous launch.  Cluster launches go first (a cluster needs
    whole SMs), then resident ones from the largest CTA size to the smallest,
    which fill what is left.  Results do not depend on the order: every chain
    is independent.  ``concurrent=False`` issues them one after another on
    ``stream`` instead.  Pointers are device addresses (ints); ``stream`` is a
    ``torch.cuda.Stream``.
    """
    torch = _torch()
    launches = list(launches)
    if not launches or n_sweeps <= 0:
        return
    if workspace_bytes < QUEUE_SLOT * len(launches):
        raise ValueError(f"workspace of {workspace_bytes} bytes is too small for {len(launches)} launches")
    order = sorted(launches, key=lambda b: (b.kind != 1, -b.threads, -b.count))
    p = ctypes.c_void_p
    rec = p(records) if records else None

    def issue(b: Launch, i: int, s) -> None:
        sp = p(s.cuda_stream)
        ws = p(workspace + QUEUE_SLOT * i)
        if b.kind == 0:
            rc = lib.rbim_sweeps_batched(p(b.chains), b.count, b.l_max, p(spin_pool), p(coupling_pool), p(acc_int),
                                         p(acc_f64), rec, int(n_sweeps), int(b.threads), p(status), ws, QUEUE_SLOT, sp)
            _native.check(rc, "rbim_sweeps_batched")
        elif b.kind == 1 and b.ctas > 0:
            rc = lib.rbim_sweeps_clustered_plan(p(b.chains), b.count, b.l_max, int(b.ctas), int(b.threads),
                                                p(spin_pool), p(coupling_pool), p(acc_int), p(acc_f64), rec,
                                                int(n_sweeps), p(status), ws, QUEUE_SLOT, sp)
            _native.check(rc, "rbim_sweeps_clustered_plan")
        elif b.kind == 1:
            rc = lib.rbim_sweeps_clustered(p(b.chains), b.count, b.l_max, p(spin_pool), p(coupling_pool), p(acc_int),
                                           p(acc_f64), rec, int(n_sweeps), p(status), ws, QUEUE_SLOT, sp)
            _native.check(rc, "rbim_sweeps_clustered")
        else:
            raise ValueError(f"launch kind {b.kind} is not an on-chip engine")

    if len(order) == 1 or not concurrent:
        for i, b in enumerate(order):
            issue(b, i, stream)
        return
    fork = torch.cuda.Event()
    fork.record(stream)
    side = _side(device, len(order))
    for i, (b, s) in enumerate(zip(order, side)):
        s.wait_event(fork)
        issue(b, i, s)
    for s in side:
        done = torch.cuda.Event()
        done.record(s)
        stream.wait_event(done)


def require_cuda(device=None):
    """Return the CUDA device to use; raise if there is none (no CPU fallback exists)."""
    torch = _torch()
    if not torch.cuda.is_available():
        raise _native.RbimError("the rbim B200 engine needs a CUDA device; none is available")
    if device is None:
        return torch.device("cuda", torch.cuda.current_device())
    d = torch.device(device)
    if d.type != "cuda":
        raise _native.RbimError(f"the rbim B200 engine runs on CUDA devices only, got {d}")
    return d


def chain_key(seed) -> int:
    """64-bit Philox key of a chain from an int, a ``SeedSequence`` or ``None``.

    The reference seeds each task with a ``SeedSequence`` child
    (``simulation.py:367-368, 384-393``); the engine turns that child into its
    key with ``generate_state(2, uint32)``.
    """
    ss = seed if isinstance(seed, np.random.SeedSequence) else np.random.SeedSequence(seed)
    w = ss.generate_state(2, dtype=np.uint32)
    return int(w[0]) | (int(w[1]) << 32)


@dataclass
class ChainSpec:
    """One chain: lattice size, index of its realization, key, inverse temperature, run layout."""

    L: int
    realization: int
    key: int
    beta: float
    n_therm: int
    n_bins: int
    sweeps_per_bin: int
    records: bool = False

    @property
    def n_total(self) -> int:
        return self.n_therm + self.n_bins * self.sweeps_per_bin


class ChainSet:
    """Device state of many chains plus the calls that advance them.

    ``couplings`` holds one packed coupling array (``pack_couplings``) per
    realization; ``specs[i].realization`` indexes it.
    """

    def __init__(self, specs: Sequence[ChainSpec], couplings: Sequence[np.ndarray], device=None):
        torch = _torch()
        self.device = require_cuda(device)
        self.lib = _native.lib()
        self.specs = list(specs)
        if not self.specs:
            raise ValueError("a ChainSet needs at least one chain")
        self.n = len(self.specs)
        Ls = np.array([s.L for s in self.specs], dtype=np.int64)
        if np.any(Ls < 3):
            raise ValueError("L must be at least 3")
        self.l_max = int(Ls.max())
        real_L = {}
        for s in self.specs:
            if s.realization < 0 or s.realization >= len(couplings):
                raise ValueError(f"chain refers to realization {s.realization} of {len(couplings)}")
            if real_L.setdefault(s.realization, s.L) != s.L:
                raise ValueError("all chains of one realization must share L")
            if s.sweeps_per_bin < 1 or s.n_bins < 1 or s.n_therm < 0:
                raise ValueError("n_bins and sweeps_per_bin must be >= 1 and n_therm >= 0")

        # Coupling pool: realizations back to back (JH plane then JV plane).
        c_off = np.zeros(len(couplings), dtype=np.int64)
        total = 0
        for r, c in enumerate(couplings):
            L = real_L.get(r)
            if L is None:
                c_off[r] = total
                continue
            if c.size != 2 * words_for(L):
                raise ValueError(f"realization {r}: packed couplings have {c.size} words, expected {2 * words_for(L)}")
            c_off[r] = total
            total += c.size
        pool = np.zeros(max(total, 4), dtype="<u4")
        for r, c in enumerate(couplings):
            if r in real_L:
                pool[c_off[r]: c_off[r] + c.size] = c
        self.coupling_pool = torch.from_numpy(pool.view(np.int32)).to(self.device)

        # Spin pool, accumulators, records.
        s_off = np.zeros(self.n, dtype=np.int64)
        a_off = np.zeros(self.n, dtype=np.int64)
        r_off = np.full(self.n, -1, dtype=np.int64)
        ts = ta = tr = 0
        for i, s in enumerate(self.specs):
            s_off[i] = ts
            ts += words_for(s.L)
            a_off[i] = ta
            ta += s.n_bins
            if s.records:
                r_off[i] = tr
                tr += s.n_bins * s.sweeps_per_bin
        self.spin_pool = torch.zeros(max(ts, 4), dtype=torch.int32, device=self.device)
        self.acc_int = torch.zeros((max(ta, 1), _native.ACC_INT), dtype=torch.int64, device=self.device)
        self.acc_f64 = torch.zeros((max(ta, 1), _native.ACC_F64), dtype=torch.float64, device=self.device)
        self.records = torch.zeros((tr, _native.REC_LEN), dtype=torch.int32, device=self.device) if tr else None
        self.spin_off, self.acc_off, self.rec_off = s_off, a_off, r_off

        # Descriptor slots grouped by launch bucket: resident lattices by size
        # class, cluster lattices by CTAs per cluster, then those only the plain
        # engine takes (engine_buckets).
        with torch.cuda.device(self.device):
            r_max = _native.resident_max_l()
            c_max = _native.cluster_max_l()
            keys = _native.engine_buckets(Ls, r_max, c_max)
        order = np.array(sorted(range(self.n), key=lambda i: keys[i]), dtype=np.int64)
        self.slot = np.empty(self.n, dtype=np.int64)
        self.slot[order] = np.arange(self.n)
        self.buckets = []  # (kind, first slot, count, l_max)
        self.bucket_sizes = []  # the distinct L of each bucket
        groups = {}
        for i, k in enumerate(keys):
            groups.setdefault(k, []).append(i)
        for k in sorted(groups):
            members = np.array(groups[k], dtype=np.int64)
            self.buckets.append((k[0], int(self.slot[members].min()), len(members), int(Ls[members].max())))
            self.bucket_sizes.append(sorted(set(int(v) for v in Ls[members])))
        self.plain_only = [int(i) for i in order if keys[i][0] == 2]

        desc = np.zeros(self.n, dtype=_native.CHAIN_DTYPE)
        desc["key"] = [s.key for s in self.specs]
        thr_of = {}
        desc["thr"] = [thr_of[s.beta] if s.beta in thr_of else thr_of.setdefault(s.beta, threshold(s.beta))
                       for s in self.specs]
        desc["spin_off"] = s_off
        desc["coupling_off"] = c_off[[s.realization for s in self.specs]]
        desc["acc_off"] = a_off
        desc["rec_off"] = r_off
        desc["n_therm"] = [s.n_therm for s in self.specs]
        desc["n_bins"] = [s.n_bins for s in self.specs]
        desc["sweeps_per_bin"] = [s.sweeps_per_bin for s in self.specs]
        desc["L"] = Ls
        desc = desc[order]
        self.desc_host = desc
        self.chains = torch.from_numpy(desc.view(np.uint8).copy()).to(self.device)
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.n_total = np.array([s.n_total for s in self.specs], dtype=np.int64)
        self._sweep_host = np.zeros(self.n, dtype=np.int64)
        self._ws = None
        self._pws = None  # plain-engine workspace; captured graphs hold its address
        self._gws = None  # grid-engine workspace
        self._grid_ok = {}  # L -> the grid engine has a plan for L on this device
        self._graphs = {}  # (sweeps, chain indices) -> torch.cuda.CUDAGraph of run_plain

    # -- helpers -----------------------------------------------------------
    @staticmethod
    def _ptr(t) -> ctypes.c_void_p:
        return ctypes.c_void_p(t.data_ptr())

    def _stream(self):
        return ctypes.c_void_p(_torch().cuda.current_stream(self.device).cuda_stream)

    def _workspace(self, nbytes: int):
        torch = _torch()
        if self._ws is None or self._ws.numel() < nbytes:
            self._ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.device)
        return self._ws

    # -- state -------------------------------------------------------------
    def init_spins(self, hot: bool = True) -> None:
        """Hot (Philox) or cold start of every chain (reference ``initial_spins``)."""
        with _torch().cuda.device(self.device):
            rc = self.lib.rbim_init_spins(self._ptr(self.chains), self.n, self._ptr(self.spin_pool), int(hot),
                                          self._stream())
        _native.check(rc, "rbim_init_spins")

    def set_spins(self, i: int, words: np.ndarray) -> None:
        nw = words_for(self.specs[i].L)
        src = _torch().from_numpy(np.ascontiguousarray(words, dtype="<u4").view(np.int32))
        self.spin_pool[self.spin_off[i]: self.spin_off[i] + nw].copy_(src)

    def set_descriptor_field(self, i: int, name: str, value: int) -> None:
        """Write one field of chain ``i``'s ``rbim_chain_t`` (host and device copies).

        No check is made beyond the field's type: this is how a caller sets
        ``walk_cap`` or, in tests, a descriptor the kernels must reject.
        """
        self.set_descriptor_fields(i, **{name: value})

    def set_descriptor_fields(self, i: int, **fields) -> None:
        """Write several fields of chain ``i``'s ``rbim_chain_t`` with one copy to the device."""
        k = int(self.slot[i])
        for name, value in fields.items():
            self.desc_host[name][k] = value
        row = _torch().from_numpy(self.desc_host[k: k + 1].view(np.uint8).copy())
        self.chains[96 * k: 96 * (k + 1)].copy_(row)

    def set_sweep(self, i: int, sweep: int) -> None:
        """Set chain ``i``'s sweep counter (host and device copies)."""
        self.set_descriptor_field(i, "sweep", sweep)
        self._sweep_host[i] = min(sweep, self.n_total[i])

    def spin_words(self, i: int) -> np.ndarray:
        nw = words_for(self.specs[i].L)
        return self.spin_pool[self.spin_off[i]: self.spin_off[i] + nw].cpu().numpy().view("<u4")

    def spins(self, i: int) -> np.ndarray:
        return unpack_spins(self.spin_words(i), self.specs[i].L)

    # -- sweeps ------------------------------------------------------------
    def run_batched(self, n_sweeps: int, threads: int = 0, concurrent: bool = True) -> None:
        """Advance every chain by up to ``n_sweeps`` sweeps.

        Chains with L up to ``rbim_resident_max_l()`` run on the resident
        engine (one lattice per CTA, one launch per CTA size class), larger
        ones up to ``rbim_cluster_max_l()`` on the cluster engine (one lattice
        per thread-block cluster, one launch per cluster plan), and any larger
        still on the plain engine.  The on-chip launches of one call run
        concurrently (:func:`launch_buckets`; ``concurrent=False`` issues them
        one after another).  ``threads`` fixes the resident
        CTA size; 0 takes the autotuner's choice when it is enabled
        (``autotune.enable()``), else the library's rule.
        """
        self._run_batched_fixed(n_sweeps, threads, tuned=threads == 0, concurrent=concurrent)

    def _run_batched_fixed(self, n_sweeps: int, threads: int, tuned: bool = False, concurrent: bool = True,
                           cluster_plan=None) -> None:
        """``cluster_plan`` ``(CTAs, CTA size)`` fixes the plan of every cluster launch (the tuner's timing runs)."""
        if n_sweeps <= 0:
            return
        from . import autotune
        torch = _torch()
        launches = []
        for (kind, first, count, l_max), sizes in zip(self.buckets, self.bucket_sizes):
            if kind == 2:
                continue
            ctas = 0
            if kind == 0:
                nt = autotune.tuned_threads(l_max, self.device) if tuned else threads
                if not nt:
                    nt = occupancy_threads(int(self.lib.rbim_resident_threads(l_max)), count,
                                           _sm_count(self.device))
            else:
                plan = cluster_plan or (autotune.tuned_cluster_plan(l_max, sizes, self.device) if tuned else None)
                if plan:
                    ctas, nt = int(plan[0]), int(plan[1])
                else:
                    nt = int(self.lib.rbim_cluster_threads(l_max))
            launches.append(Launch(kind, self.chains.data_ptr() + 96 * first, count, l_max, nt, ctas))
        if launches:
            ws = self._workspace(QUEUE_SLOT * len(launches))
            with torch.cuda.device(self.device):
                launch_buckets(self.lib, self.device, torch.cuda.current_stream(self.device), launches,
                               spin_pool=self.spin_pool.data_ptr(), coupling_pool=self.coupling_pool.data_ptr(),
                               acc_int=self.acc_int.data_ptr(), acc_f64=self.acc_f64.data_ptr(),
                               records=self.records.data_ptr() if self.records is not None else None,
                               n_sweeps=n_sweeps, status=self.status.data_ptr(), workspace=ws.data_ptr(),
                               workspace_bytes=ws.numel(), concurrent=concurrent)
        if self.plain_only:
            self.run_whole_gpu(n_sweeps, self.plain_only)
            done = np.ones(self.n, dtype=bool)
            done[self.plain_only] = False
            self._sweep_host[done] = np.minimum(self._sweep_host[done] + n_sweeps, self.n_total[done])
        else:
            self._sweep_host = np.minimum(self._sweep_host + n_sweeps, self.n_total)

    #: ``run_plain`` replays a captured CUDA graph for calls of at least this
    #: many sweeps: the plain engine issues 7 kernels per sweep, which at small
    #: L cost more to launch one by one than to run.
    PLAIN_GRAPH_MIN_SWEEPS = 8
    #: ... and of at most this many kernel nodes (7 per sweep per chain).
    PLAIN_GRAPH_MAX_NODES = 1 << 15

    def _plain_workspace(self, idx):
        nbytes = max(int(self.lib.rbim_plain_workspace_bytes(self.specs[i].L)) for i in idx)
        if self._pws is None or self._pws.numel() < nbytes:
            self._graphs.clear()  # they hold the old workspace's address
            self._pws = _torch().empty(max(nbytes, 256), dtype=_torch().uint8, device=self.device)
        return self._pws

    def _launch_plain(self, n_sweeps: int, idx, ws, stream) -> None:
        for i in idx:
            rc = self.lib.rbim_sweeps_plain(
                self.specs[i].L, ctypes.c_void_p(self.chains.data_ptr() + 96 * int(self.slot[i])), self._ptr(self.spin_pool),
                self._ptr(self.coupling_pool), self._ptr(self.acc_int), self._ptr(self.acc_f64),
                self._ptr(self.records) if self.records is not None else None, int(n_sweeps),
                self._ptr(self.status), self._ptr(ws), ws.numel(), stream)
            _native.check(rc, "rbim_sweeps_plain")

    def _plain_graph_ok(self, n_sweeps: int, idx) -> bool:
        return n_sweeps >= self.PLAIN_GRAPH_MIN_SWEEPS and 7 * n_sweeps * len(idx) <= self.PLAIN_GRAPH_MAX_NODES

    def capture_plain(self, n_sweeps: int, chains: Optional[Sequence[int]] = None) -> bool:
        """Capture the launch sequence of ``run_plain(n_sweeps, chains)`` as a CUDA graph without running it.

        Every kernel reads the chain descriptors from device memory (a finished
        chain's kernels return at once), so one graph serves every later call
        with the same arguments.  Returns False when the call is outside the
        graph limits and ``run_plain`` would launch directly.
        """
        idx = list(range(self.n)) if chains is None else [int(i) for i in chains]
        if n_sweeps <= 0 or not self._plain_graph_ok(n_sweeps, idx):
            return False
        key = (int(n_sweeps), tuple(idx))
        ws = self._plain_workspace(idx)
        if key not in self._graphs:
            torch = _torch()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.device(self.device):
                s = torch.cuda.Stream(self.device)
                with torch.cuda.graph(g, stream=s, capture_error_mode="thread_local"):
                    self._launch_plain(n_sweeps, idx, ws, ctypes.c_void_p(s.cuda_stream))
            self._graphs[key] = g
        return True

    def run_plain(self, n_sweeps: int, chains: Optional[Sequence[int]] = None, graph: bool = True) -> None:
        """Advance chains one at a time on the plain (global-memory) engine.

        With ``graph`` (the default), calls of at least
        ``PLAIN_GRAPH_MIN_SWEEPS`` sweeps replay a CUDA graph of the launch
        sequence, captured on the first such call (``capture_plain``); the
        results are the same as launching one by one.
        """
        if n_sweeps <= 0:
            return
        idx = list(range(self.n)) if chains is None else [int(i) for i in chains]
        torch = _torch()
        with torch.cuda.device(self.device):
            if graph and self.capture_plain(n_sweeps, idx):
                self._graphs[(int(n_sweeps), tuple(idx))].replay()
            else:
                self._launch_plain(n_sweeps, idx, self._plain_workspace(idx), self._stream())
        for i in idx:
            self._sweep_host[i] = min(self._sweep_host[i] + n_sweeps, self.n_total[i])

    def run_plain_noalloc(self, n_sweeps: int, chains: Optional[Sequence[int]] = None) -> None:
        """As :meth:`run_plain`, through ``rbim_sweeps_plain_noalloc`` (library-static scratch, L <= 512).

        Calls on one device share the scratch, so they are issued in order on
        this set's stream.
        """
        if n_sweeps <= 0:
            return
        idx = range(self.n) if chains is None else chains
        with _torch().cuda.device(self.device):
            for i in idx:
                rc = self.lib.rbim_sweeps_plain_noalloc(
                    self.specs[i].L, ctypes.c_void_p(self.chains.data_ptr() + 96 * int(self.slot[i])), self._ptr(self.spin_pool),
                    self._ptr(self.coupling_pool), self._ptr(self.acc_int), self._ptr(self.acc_f64),
                    self._ptr(self.records) if self.records is not None else None, int(n_sweeps),
                    self._ptr(self.status), self._stream())
                _native.check(rc, "rbim_sweeps_plain_noalloc")
                self._sweep_host[i] = min(self._sweep_host[i] + n_sweeps, self.n_total[i])

    def grid_ok(self, L: int) -> bool:
        """Whether the grid engine has a plan for an L x L lattice on this set's device (cached per L)."""
        if L not in self._grid_ok:
            with _torch().cuda.device(self.device):
                self._grid_ok[L] = _native.grid_plan(L) is not None
        return self._grid_ok[L]

    def run_whole_gpu(self, n_sweeps: int, chains: Sequence[int]) -> None:
        """Advance chains one at a time over the whole GPU: on the grid engine where it has a plan for the
        chain's L, else on the plain engine (the lattices beyond the on-chip engines' sizes)."""
        grid = [int(i) for i in chains if self.grid_ok(self.specs[i].L)]
        plain = [int(i) for i in chains if not self.grid_ok(self.specs[i].L)]
        if grid:
            self.run_grid(n_sweeps, grid)
        if plain:
            self.run_plain(n_sweeps, plain)

    def _grid_workspace(self, L: int, ctas: int):
        nbytes = int(self.lib.rbim_grid_workspace_bytes(int(L), int(ctas)))
        if nbytes <= 0:
            raise _native.RbimError(f"the grid engine has no plan for L = {L}")
        if self._gws is None or self._gws.numel() < nbytes:
            self._gws = _torch().empty(max(nbytes, 256), dtype=_torch().uint8, device=self.device)
        return self._gws

    def run_grid(self, n_sweeps: int, chains: Optional[Sequence[int]] = None, plan=None,
                 wait_cycles: int = 0) -> None:
        """Advance chains one at a time on the grid engine: one cooperative launch per chain and call, the
        lattice split in tiles over every SM (``rbim_sweeps_grid``).

        ``plan`` is ``(CTAs, CTA size)``, by default the device's (``_native.grid_plan``); results do not
        depend on it.  ``wait_cycles`` bounds each wait at a grid-wide barrier (0: about one second).
        """
        if n_sweeps <= 0:
            return
        idx = list(range(self.n)) if chains is None else [int(i) for i in chains]
        ctas, threads = (0, 0) if plan is None else (int(plan[0]), int(plan[1]))
        with _torch().cuda.device(self.device):
            for i in idx:
                L = self.specs[i].L
                ws = self._grid_workspace(L, ctas)
                rc = self.lib.rbim_sweeps_grid(
                    L, ctypes.c_void_p(self.chains.data_ptr() + 96 * int(self.slot[i])), self._ptr(self.spin_pool),
                    self._ptr(self.coupling_pool), self._ptr(self.acc_int), self._ptr(self.acc_f64),
                    self._ptr(self.records) if self.records is not None else None, int(n_sweeps),
                    self._ptr(self.status), ctas, threads, int(wait_cycles), self._ptr(ws), ws.numel(), self._stream())
                _native.check(rc, "rbim_sweeps_grid")
                self._sweep_host[i] = min(self._sweep_host[i] + n_sweeps, self.n_total[i])

    def remaining(self) -> int:
        """Sweeps still to run for the longest chain (host bookkeeping)."""
        return int(np.max(self.n_total - self._sweep_host))

    def run_to_end(self, engine: str = "auto", chunk: int = 1000, threads: int = 0) -> None:
        """Run every chain to the end of its run in chunks of ``chunk`` sweeps.

        ``engine="auto"`` (``auto_engine``) runs a set of one lattice with
        L <= 64 on one resident CTA of ``single_cta_threads(L)`` threads, one
        larger lattice over the whole GPU -- on the grid engine where it has a
        plan, else on the plain engine -- and any other set on the batched
        engines.  On B200 a sweep of one L = 256 lattice takes 38 us
        on the grid engine, 56 us on the plain engine and 158 us on one
        resident CTA; L = 1024 66 us, 160 us and 189 us on one 16-CTA cluster.
        Results are the same on every engine.
        """
        if engine == "auto":
            engine = auto_engine(self.specs)
        if engine == "batched" and threads == 0 and self.n == 1 and self.specs[0].L <= self.lib.rbim_resident_max_l():
            threads = single_cta_threads(self.specs[0].L)
        if engine not in ("batched", "plain", "grid"):
            raise ValueError(f"engine must be 'auto', 'batched', 'plain' or 'grid', got {engine!r}")
        while self.remaining() > 0:
            n = min(chunk, self.remaining())
            if engine == "batched":
                self.run_batched(n, threads)
            elif engine == "grid":
                self.run_grid(n)
            else:
                self.run_plain(n)
        self.check_status()

    def check_status(self) -> None:
        st = int(self.status.item())
        if st:
            raise _native.RbimError(f"device status word {st:#x} (1 = find bound, 2 = union bound, 4 = bad chain)")

    # -- results -----------------------------------------------------------
    def device_sweeps(self) -> np.ndarray:
        """The chains' sweep counters as stored on the device."""
        d = self.chains.cpu().numpy().view(_native.CHAIN_DTYPE)
        return d["sweep"].astype(np.int64)[self.slot]

    def bins(self, i: int):
        """``(int_sums (n_bins, 12), f64_sums (n_bins, 2))`` of chain ``i`` (host copies)."""
        s = self.specs[i]
        a = self.acc_off[i]
        return (self.acc_int[a: a + s.n_bins].cpu().numpy(), self.acc_f64[a: a + s.n_bins].cpu().numpy())

    def all_bins(self):
        return self.acc_int.cpu().numpy(), self.acc_f64.cpu().numpy()

    def chain_records(self, i: int) -> np.ndarray:
        s = self.specs[i]
        if self.records is None or self.rec_off[i] < 0:
            raise ValueError(f"chain {i} was created without records")
        r = self.rec_off[i]
        return self.records[r: r + s.n_bins * s.sweeps_per_bin].cpu().numpy()
