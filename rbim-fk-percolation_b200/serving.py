"""Continuous-batching server for temperature-scan requests.

A request is one call of the reference's ``run_temperature_scan`` (an L, a
p, a temperature grid, realizations, sweeps and a seed).  The server keeps
the state of every admitted request resident in device memory -- packed
spins, packed couplings and per-bin accumulators in pools that it allocates
once -- and advances all admitted chains together, one quantum of sweeps per
engine launch.  Requests that arrive while others run are admitted between
launches as soon as their footprint fits the free pool space; finished
requests leave between launches, their bin sums come back (a few hundred
bytes per chain) and are assembled with the reference's estimators.

A chain's sums depend only on its own key, couplings, temperature and run
layout, never on the other chains of a launch or on how its sweeps are split
into launches, so every result equals the one ``run_temperature_scan`` gives
for the same request alone, bit for bit.

Lattices with L up to ``rbim_resident_max_l()`` run on the resident engine,
one lattice per CTA; larger ones up to ``rbim_cluster_max_l()`` on the
cluster engine, one lattice per thread-block cluster; any larger still over
the whole GPU, one chain after the other inside each quantum: on the grid
engine where it has a plan for L, else on the plain engine.
"""

from __future__ import annotations

import ctypes
import queue
import threading
import time
from concurrent.futures import Future, ThreadPoolExecutor
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _native, autotune
from .engine import QUEUE_SLOT, Launch, _sm_count, _torch, launch_buckets, occupancy_threads, require_cuda
from .packing import pack_couplings, threshold, words_for
from .simulation import ScanPlan, assemble_scan, plan_temperature_scan

__all__ = ["ScanRequest", "ScanServer", "RangeAllocator", "request_footprint"]


@dataclass
class ScanRequest:
    """Arguments of one ``run_temperature_scan`` call (reference ``simulation.py:336-350``)."""

    L: int
    p: float
    temperatures: Sequence[float]
    n_realizations: int = 1
    n_sweeps: int = 10_000
    n_therm: Optional[int] = None
    n_bins: int = 10
    seed: int = 0
    measure_percolation: bool = True
    start: str = "hot"
    disorder: Optional[Sequence[tuple]] = None

    def plan(self) -> ScanPlan:
        return plan_temperature_scan(self.L, self.p, self.temperatures, n_realizations=self.n_realizations,
                                     n_sweeps=self.n_sweeps, n_therm=self.n_therm, n_bins=self.n_bins,
                                     seed=self.seed, measure_percolation=self.measure_percolation, start=self.start,
                                     disorder=self.disorder)


class RangeAllocator:
    """First-fit allocator of ``[offset, offset + size)`` ranges in a pool of ``capacity`` units.

    Offsets and sizes are multiples of ``align``; freed neighbours coalesce.
    """

    def __init__(self, capacity: int, align: int = 1):
        self.align = int(align)
        self.capacity = int(capacity) // self.align * self.align
        self.free: List[List[int]] = [[0, self.capacity]] if self.capacity > 0 else []
        self.used = 0

    def _round(self, n: int) -> int:
        return -(-int(n) // self.align) * self.align

    def alloc(self, n: int) -> Optional[int]:
        n = self._round(max(n, 1))
        for i, (off, size) in enumerate(self.free):
            if size >= n:
                if size == n:
                    self.free.pop(i)
                else:
                    self.free[i] = [off + n, size - n]
                self.used += n
                return off
        return None

    def release(self, off: int, n: int) -> None:
        n = self._round(max(n, 1))
        self.used -= n
        i = 0
        while i < len(self.free) and self.free[i][0] < off:
            i += 1
        self.free.insert(i, [off, n])
        # Merge with the right, then the left neighbour.
        if i + 1 < len(self.free) and self.free[i][0] + self.free[i][1] == self.free[i + 1][0]:
            self.free[i][1] += self.free.pop(i + 1)[1]
        if i > 0 and self.free[i - 1][0] + self.free[i - 1][1] == self.free[i][0]:
            self.free[i - 1][1] += self.free.pop(i)[1]

    @property
    def largest_free(self) -> int:
        return max((s for _, s in self.free), default=0)


def _plan_and_pack(req: ScanRequest):
    plan = req.plan()
    packed = [pack_couplings(J, plan.L) for J in plan.couplings]
    return plan, (np.concatenate(packed).view(np.int32) if packed else np.zeros(0, np.int32))


def request_footprint(L: int, n_temperatures: int, n_realizations: int, n_bins: int) -> Dict[str, int]:
    """Device footprint of a request: pool words (spins + couplings), accumulator rows, chains.

    Bytes: 4 per word, 112 per accumulator row (12 int64 + 2 double), 96 per
    chain descriptor.
    """
    nw = words_for(L)
    chains = n_temperatures * n_realizations
    return {"words": chains * nw + n_realizations * 2 * nw, "rows": chains * n_bins, "chains": chains}


@dataclass
class _Active:
    req: ScanRequest
    plan: ScanPlan
    future: Future
    submitted: float
    admitted: float
    spin_off: int
    coupling_off: int
    words: int
    row_off: int
    rows: int
    desc: np.ndarray  # CHAIN_DTYPE, one per chain, sweep tracked on the host
    n_total: int
    done: int = 0
    staged: object = None  # host and device staging of the admission copies


@dataclass
class _Pending:
    req: ScanRequest
    future: Future
    submitted: float
    planned: Optional[Future] = None  # -> (ScanPlan, packed couplings)


class ScanServer:
    """Admits scan requests as device memory frees up and runs them together.

    ``memory_bytes`` bounds the pools (spins and couplings: 75 %, accumulator
    rows: 25 %); ``max_chains`` bounds the chains of one launch; ``quantum``
    is the number of sweeps per engine launch.  Use as a context manager (a
    background thread runs the loop) or drive it with :meth:`step`.
    """

    def __init__(self, device=None, memory_bytes: int = 2 << 30, max_chains: int = 65536, quantum: int = 100,
                 threads: int = 0):
        torch = _torch()
        self.device = require_cuda(device)
        self.lib = _native.lib()
        self.quantum = int(quantum)
        self.threads = int(threads)
        self.max_chains = int(max_chains)
        with torch.cuda.device(self.device):
            self.resident_max_l = _native.resident_max_l()
            self.cluster_max_l = _native.cluster_max_l()
        words = int(memory_bytes * 0.75) // 4
        rows = int(memory_bytes * 0.25) // 112
        self.words = RangeAllocator(words, align=4)
        self.rows = RangeAllocator(rows, align=1)
        with torch.cuda.device(self.device):
            self.stream = torch.cuda.Stream(self.device)
            self.copy_stream = torch.cuda.Stream(self.device)
            self.word_pool = torch.zeros(max(self.words.capacity, 4), dtype=torch.int32, device=self.device)
            self.acc_int = torch.zeros((max(self.rows.capacity, 1), _native.ACC_INT), dtype=torch.int64,
                                       device=self.device)
            self.acc_f64 = torch.zeros((max(self.rows.capacity, 1), _native.ACC_F64), dtype=torch.float64,
                                       device=self.device)
            self.desc_dev = torch.zeros(96 * max(self.max_chains, 1), dtype=torch.uint8, device=self.device)
            self.desc_host = torch.zeros(96 * max(self.max_chains, 1), dtype=torch.uint8).pin_memory()
            self._desc_copied = torch.cuda.Event()
            self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
            # One work-queue counter per concurrent bucket launch.
            self.queue_ws = torch.zeros(QUEUE_SLOT * 64, dtype=torch.uint8, device=self.device)
        self._plain_ws = None  # workspace of the whole-GPU launches (grid or plain engine)
        self._grid_plans = {}  # L -> the grid engine has a plan for L on the server's device
        self._planner = ThreadPoolExecutor(max_workers=2, thread_name_prefix="rbim-scan-plan")
        self._inbox: "queue.Queue[_Pending]" = queue.Queue()
        self._waiting: List[_Pending] = []
        self._active: List[_Active] = []
        self._inflight: list = []  # (event after a launch, requests that launch finished)
        self._thread = None
        self._stop = threading.Event()
        self._error: Optional[BaseException] = None
        self.launches = 0
        self.completed: List[dict] = []

    # -- client side --------------------------------------------------------
    def submit(self, request: ScanRequest) -> Future:
        """Queue a request; the future resolves to the ``run_temperature_scan`` result dict."""
        if self._error is not None:
            raise _native.RbimError(f"server stopped after an error: {self._error}")
        fp = request_footprint(request.L, len(request.temperatures), request.n_realizations, request.n_bins)
        if fp["words"] > self.words.capacity or fp["rows"] > self.rows.capacity or fp["chains"] > self.max_chains:
            raise ValueError(f"request needs {fp} which exceeds the server's pools "
                             f"(words {self.words.capacity}, rows {self.rows.capacity}, chains {self.max_chains})")
        fut: Future = Future()
        p = _Pending(request, fut, time.perf_counter())
        # Disorder, keys and packed couplings are prepared on the host while
        # earlier requests run.
        p.planned = self._planner.submit(_plan_and_pack, request)
        self._inbox.put(p)
        return fut

    def __enter__(self):
        self._thread = threading.Thread(target=self._loop, name="rbim-scan-server", daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *exc):
        self.close()

    def close(self, drain: bool = True) -> None:
        if self._thread is None:
            return
        if drain:
            while self._thread.is_alive() and not self.idle():
                time.sleep(0.005)
        self._stop.set()
        self._thread.join()
        self._thread = None
        self._planner.shutdown(wait=False)

    def idle(self) -> bool:
        return not self._active and not self._waiting and not self._inflight and self._inbox.empty()

    # -- server side --------------------------------------------------------
    def _loop(self) -> None:
        torch = _torch()
        torch.cuda.set_device(self.device)
        while True:
            try:
                worked = self.step()
            except BaseException as exc:  # pragma: no cover - surfaced through the futures
                self._error = exc
                self._fail_all(exc)
                return
            if not worked:
                if self._stop.is_set() and self.idle():
                    return
                try:
                    p = self._inbox.get(timeout=0.005)
                    self._waiting.append(p)
                except queue.Empty:
                    pass

    def _fail_all(self, exc: BaseException) -> None:
        for a in self._active:
            if not a.future.done():
                a.future.set_exception(exc)
            self._inbox.task_done()
        self._active = []
        for p in self._waiting:
            p.future.set_exception(exc)
            self._inbox.task_done()
        self._waiting = []

    def _drain_inbox(self) -> None:
        while True:
            try:
                self._waiting.append(self._inbox.get_nowait())
            except queue.Empty:
                return

    def _admit(self) -> None:
        """Admit waiting requests in arrival order while their footprint fits."""
        torch = _torch()
        n_chains = sum(len(a.desc) for a in self._active)
        while self._waiting:
            p = self._waiting[0]
            if not p.planned.done() and self._active:
                return  # keep the device busy; admit once the plan is ready
            try:
                plan, packed = p.planned.result()
            except BaseException as exc:  # a bad request fails alone
                self._waiting.pop(0)
                p.future.set_exception(exc)
                self._inbox.task_done()
                continue
            nw = words_for(plan.L)
            n_r = plan.n_realizations
            chains = plan.n_tasks
            if chains == 0:
                self._waiting.pop(0)
                p.future.set_result(assemble_scan(plan, np.zeros((0, plan.n_bins, 12), np.int64),
                                                  np.zeros((0, plan.n_bins, 2), np.float64)))
                self._inbox.task_done()
                continue
            if n_chains + chains > self.max_chains:
                return
            words = chains * nw + n_r * 2 * nw
            w_off = self.words.alloc(words)
            if w_off is None:
                return
            r_off = self.rows.alloc(chains * plan.n_bins)
            if r_off is None:
                self.words.release(w_off, words)
                return
            self._waiting.pop(0)
            spin_off = w_off
            coup_off = w_off + chains * nw
            # Couplings and zeroed accumulators, then the hot or cold start.
            desc = np.zeros(chains, dtype=_native.CHAIN_DTYPE)
            t_index = np.arange(chains) // n_r
            real = np.arange(chains) % n_r
            desc["key"] = plan.keys
            desc["thr"] = [threshold(1.0 / plan.temperatures[t]) for t in t_index]
            desc["spin_off"] = spin_off + nw * np.arange(chains)
            desc["coupling_off"] = coup_off + 2 * nw * real
            desc["acc_off"] = r_off + plan.n_bins * np.arange(chains)
            desc["rec_off"] = -1
            desc["n_therm"] = plan.n_therm
            desc["n_bins"] = plan.n_bins
            desc["sweeps_per_bin"] = plan.sweeps_per_bin
            desc["L"] = plan.L
            # Pinned staging keeps the copies asynchronous behind the running
            # launch; the staging tensors live until the request retires.
            staged = (torch.from_numpy(packed).pin_memory(), torch.from_numpy(desc.view(np.uint8).copy()).pin_memory())
            with torch.cuda.stream(self.stream):
                self.word_pool[coup_off: coup_off + packed.size].copy_(staged[0], non_blocking=True)
                self.acc_int[r_off: r_off + chains * plan.n_bins].zero_()
                self.acc_f64[r_off: r_off + chains * plan.n_bins].zero_()
                d = torch.empty(staged[1].numel(), dtype=torch.uint8, device=self.device)
                d.copy_(staged[1], non_blocking=True)
                rc = self.lib.rbim_init_spins(ctypes.c_void_p(d.data_ptr()), chains,
                                              ctypes.c_void_p(self.word_pool.data_ptr()), int(plan.hot),
                                              ctypes.c_void_p(self.stream.cuda_stream))
                _native.check(rc, "rbim_init_spins")
            n_total = plan.n_therm + plan.n_bins * plan.sweeps_per_bin
            self._active.append(_Active(p.req, plan, p.future, p.submitted, time.perf_counter(), spin_off, coup_off,
                                        words, r_off, chains * plan.n_bins, desc, n_total, staged=(staged, d)))
            n_chains += chains

    def _grid_ok(self, L: int) -> bool:
        """Whether the grid engine has a plan for an L x L lattice on the server's device (cached per L)."""
        if L not in self._grid_plans:
            with _torch().cuda.device(self.device):
                self._grid_plans[L] = _native.grid_plan(L) is not None
        return self._grid_plans[L]

    def _launch(self) -> None:
        """One quantum of sweeps for every admitted chain."""
        torch = _torch()
        sp = ctypes.c_void_p(self.stream.cuda_stream)
        pool = ctypes.c_void_p(self.word_pool.data_ptr())
        ai, af = ctypes.c_void_p(self.acc_int.data_ptr()), ctypes.c_void_p(self.acc_f64.data_ptr())
        live = [a for a in self._active if a.done < a.n_total]
        if not live:
            return
        buckets: Dict[tuple, List[_Active]] = {}
        for a, key in zip(live, _native.engine_buckets([a.plan.L for a in live], self.resident_max_l,
                                                       self.cluster_max_l)):
            buckets.setdefault(key, []).append(a)
        keys = sorted(buckets)
        allc = np.concatenate([a.desc for k in keys for a in buckets[k]])
        # The previous launch's descriptor copy must have left the pinned buffer.
        self._desc_copied.synchronize()
        host = self.desc_host.numpy()[: 96 * len(allc)]
        host[:] = allc.view(np.uint8)
        n = len(allc)
        st = ctypes.c_void_p(self.status.data_ptr())
        with torch.cuda.stream(self.stream):
            self.desc_dev[: 96 * n].copy_(self.desc_host[: 96 * n], non_blocking=True)
            self._desc_copied.record(self.stream)
            first = 0
            on_chip, plain = [], []
            for key in keys:
                group = buckets[key]
                count = sum(len(a.desc) for a in group)
                l_max = max(a.plan.L for a in group)
                base = self.desc_dev.data_ptr() + 96 * first
                if key[0] == 0:
                    nt = self.threads or autotune.tuned_threads(l_max, self.device)
                    if not nt:
                        nt = occupancy_threads(int(self.lib.rbim_resident_threads(l_max)), count,
                                               _sm_count(self.device))
                    on_chip.append(Launch(0, base, count, l_max, nt))
                elif key[0] == 1:
                    plan = autotune.tuned_cluster_plan(l_max, sorted({a.plan.L for a in group}), self.device)
                    if plan:
                        on_chip.append(Launch(1, base, count, l_max, plan[1], plan[0]))
                    else:
                        on_chip.append(Launch(1, base, count, l_max, int(self.lib.rbim_cluster_threads(l_max))))
                else:
                    plain += [(int(allc["L"][first + k]), base + 96 * k) for k in range(count)]
                first += count
            # The on-chip buckets run concurrently, each with its own queue
            # counter; lattices only the plain engine takes follow on the
            # server stream.
            launch_buckets(self.lib, self.device, self.stream, on_chip, spin_pool=self.word_pool.data_ptr(),
                           coupling_pool=self.word_pool.data_ptr(), acc_int=self.acc_int.data_ptr(),
                           acc_f64=self.acc_f64.data_ptr(), records=None, n_sweeps=self.quantum,
                           status=self.status.data_ptr(), workspace=self.queue_ws.data_ptr(),
                           workspace_bytes=self.queue_ws.numel())
            self.launches += len(on_chip)
            if plain:
                need = max(int(self.lib.rbim_plain_workspace_bytes(L)) if not self._grid_ok(L)
                           else int(self.lib.rbim_grid_workspace_bytes(L, 0)) for L, _ in plain)
                if self._plain_ws is None or self._plain_ws.numel() < need:
                    self._plain_ws = torch.empty(need, dtype=torch.uint8, device=self.device)
                wsp, wsn = ctypes.c_void_p(self._plain_ws.data_ptr()), self._plain_ws.numel()
                for L, ptr in plain:
                    if self._grid_ok(L):
                        rc = self.lib.rbim_sweeps_grid(L, ctypes.c_void_p(ptr), pool, pool, ai, af, None,
                                                       self.quantum, st, 0, 0, 0, wsp, wsn, sp)
                        _native.check(rc, "rbim_sweeps_grid")
                    else:
                        rc = self.lib.rbim_sweeps_plain(L, ctypes.c_void_p(ptr), pool, pool, ai, af, None,
                                                        self.quantum, st, wsp, wsn, sp)
                        _native.check(rc, "rbim_sweeps_plain")
                    self.launches += 1
        finished = []
        for a in live:
            a.done = min(a.n_total, a.done + self.quantum)
            a.desc["sweep"] = a.done
            if a.done >= a.n_total:
                finished.append(a)
        ev = torch.cuda.Event()
        ev.record(self.stream)
        self._inflight.append((ev, finished))

    def _retire(self, block: bool) -> None:
        """Bring back and assemble the requests of completed launches; free their pool ranges.

        The sums of a launch are copied on a side stream once that launch's
        event has fired, so the next launch keeps the device busy meanwhile.
        With ``block`` the oldest launch in flight is waited for.
        """
        torch = _torch()
        while self._inflight:
            ev, finished = self._inflight[0]
            if not ev.query():
                if not block:
                    return
                ev.synchronize()
            self._inflight.pop(0)
            block = False
            copies = []
            with torch.cuda.stream(self.copy_stream):
                self.copy_stream.wait_event(ev)
                status = self.status.to("cpu", non_blocking=True)
                for a in finished:
                    copies.append((self.acc_int[a.row_off: a.row_off + a.rows].to("cpu", non_blocking=True),
                                   self.acc_f64[a.row_off: a.row_off + a.rows].to("cpu", non_blocking=True)))
            self.copy_stream.synchronize()
            st = int(status.item())
            if st:
                raise _native.RbimError(f"device status word {st:#x} (1 = find bound, 2 = union bound, 4 = bad chain)")
            for a, (ib, fb) in zip(finished, copies):
                nb = a.plan.n_bins
                result = assemble_scan(a.plan, ib.numpy().reshape(-1, nb, _native.ACC_INT),
                                       fb.numpy().reshape(-1, nb, _native.ACC_F64))
                now = time.perf_counter()
                self.words.release(a.spin_off, a.words)
                self.rows.release(a.row_off, a.rows)
                self._active.remove(a)
                self.completed.append({"L": a.plan.L, "chains": len(a.desc), "sweeps": a.n_total,
                                       "site_updates": len(a.desc) * a.n_total * a.plan.L * a.plan.L,
                                       "submitted": a.submitted, "admitted": a.admitted, "finished": now,
                                       "latency": now - a.submitted})
                a.future.set_result(result)
                self._inbox.task_done()

    def step(self) -> bool:
        """Admit, launch one quantum, retire what earlier launches finished.

        At most two launches are in flight: while one runs, the host admits,
        enqueues the next and retires the one before.  Returns False when there
        is nothing to run or to retire.
        """
        self._drain_inbox()
        self._admit()
        launched = any(a.done < a.n_total for a in self._active)
        if launched:
            self._launch()
        if not launched and not self._inflight:
            return False
        self._retire(block=len(self._inflight) > 1 or not launched)
        return True

    def run_until_idle(self) -> None:
        """Drive the loop on the calling thread until every submitted request has finished."""
        while True:
            if not self.step() and self._inbox.empty() and not self._waiting and not self._inflight:
                return

    def latency_percentiles(self, qs=(50, 99)) -> Dict[str, float]:
        lat = np.array([c["latency"] for c in self.completed])
        if lat.size == 0:
            return {f"p{q}": float("nan") for q in qs}
        return {f"p{q}": float(np.percentile(lat, q)) for q in qs}
