"""Temperature scans sharded over ranks: one process per GPU, independent chains.

The reference's tasks (one per temperature and realization,
``simulation.py:384-399``) share nothing while they run, so a scan splits
over ranks with no exchange on the data path: every rank builds the same
:class:`~.simulation.ScanPlan` (same disorder, same keys), runs a contiguous
block of tasks on its own GPU, and the per-bin sums -- a few hundred bytes per
task -- are all-gathered once at the end so that every rank assembles the same
result.  A task's sums do not depend on which other tasks share its batch, so
the sharded scan equals the single-GPU scan bit for bit.

The gather runs on the process group's own backend: device tensors for NCCL,
host tensors for gloo.
"""

from __future__ import annotations

from typing import Optional, Sequence, Tuple

import numpy as np

from .simulation import ScanPlan, assemble_scan, plan_temperature_scan, run_scan_tasks

__all__ = ["shard_bounds", "gather_task_sums", "run_temperature_scan_sharded"]

N_INT = 12
N_F64 = 2


def shard_bounds(n_tasks: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous block ``[lo, hi)`` of tasks for ``rank`` of ``world``; sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} is not in a world of {world}")
    if n_tasks < 0:
        raise ValueError("n_tasks must be >= 0")
    base, extra = divmod(n_tasks, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def _gather_device(group):
    import torch
    import torch.distributed as dist

    backend = dist.get_backend(group)
    if backend == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def gather_task_sums(int_local: np.ndarray, f_local: np.ndarray, n_tasks: int, n_bins: int, group=None):
    """All-gather every rank's block of task sums into the full ``(n_tasks, n_bins, ...)`` arrays.

    Rank ``r`` holds tasks ``shard_bounds(n_tasks, r, world)``.  The doubles
    travel as their int64 bit patterns, so nothing is rounded on the way.
    """
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    lo, hi = shard_bounds(n_tasks, rank, world)
    if int_local.shape != (hi - lo, n_bins, N_INT) or f_local.shape != (hi - lo, n_bins, N_F64):
        raise ValueError(f"rank {rank}: local sums have shapes {int_local.shape}, {f_local.shape}; "
                         f"expected {(hi - lo, n_bins, N_INT)}, {(hi - lo, n_bins, N_F64)}")
    width = n_bins * (N_INT + N_F64)
    block = -(-n_tasks // world) if n_tasks else 0
    dev = _gather_device(group)
    packed = np.zeros((max(block, 1), width), dtype=np.int64)
    if hi > lo:
        packed[: hi - lo, : n_bins * N_INT] = int_local.reshape(hi - lo, -1)
        packed[: hi - lo, n_bins * N_INT:] = np.ascontiguousarray(f_local, dtype=np.float64).reshape(
            hi - lo, -1).view(np.int64)
    mine = torch.from_numpy(packed).to(dev)
    parts = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    full_i = np.zeros((n_tasks, n_bins, N_INT), dtype=np.int64)
    full_f = np.zeros((n_tasks, n_bins, N_F64), dtype=np.float64)
    for r, part in enumerate(parts):
        a, b = shard_bounds(n_tasks, r, world)
        if b == a:
            continue
        rows = part.cpu().numpy()[: b - a]
        full_i[a:b] = rows[:, : n_bins * N_INT].reshape(b - a, n_bins, N_INT)
        full_f[a:b] = np.ascontiguousarray(rows[:, n_bins * N_INT:]).view(np.float64).reshape(b - a, n_bins, N_F64)
    return full_i, full_f


def run_temperature_scan_sharded(L: int, p: float, temperatures: Sequence[float], *, group=None,
                                 engine: str = "auto", device=None, chunk: int = 1000, **scan_kwargs):
    """:func:`~.simulation.run_temperature_scan` with its tasks split over the ranks of ``group``.

    Call it on every rank with the same arguments (one GPU per rank; ``device``
    defaults to the current CUDA device).  Every rank returns the same result,
    equal to the single-GPU scan's.
    """
    import torch.distributed as dist

    plan: ScanPlan = plan_temperature_scan(L, p, temperatures, **scan_kwargs)
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    lo, hi = shard_bounds(plan.n_tasks, rank, world)
    int_local, f_local = run_scan_tasks(plan, range(lo, hi), engine=engine, device=device, chunk=chunk)
    full_i, full_f = gather_task_sums(int_local, f_local, plan.n_tasks, plan.n_bins, group)
    result = assemble_scan(plan, full_i, full_f)
    result["metadata"]["ranks"] = world
    return result
