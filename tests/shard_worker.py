"""One rank of a sharded temperature scan on CPU (gloo), with the oracle standing in for the GPU.

Run as ``python tests/shard_worker.py RANK WORLD PORT OUT``; used by
``tests/test_sharding.py``.  Each rank builds the scan plan, computes the
sums of its own block of tasks with the oracle's chain runner (the same
Philox chains the engine runs), all-gathers them over gloo, assembles the
jackknife result and writes everything to ``OUT/rank{RANK}.npz``.
"""

import datetime
import importlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

SCAN = dict(L=8, p=0.1, temperatures=[1.4, 2.0, 2.6, 3.2], n_realizations=3, n_sweeps=40, n_therm=6, n_bins=4,
            seed=11)


def oracle_sums(rb, oracle, plan, tasks):
    tasks = list(tasks)
    nb = plan.n_bins
    if not tasks:
        return np.zeros((0, nb, 12), np.int64), np.zeros((0, nb, 2), np.float64)
    n_r = plan.n_realizations
    J = np.stack([plan.couplings[k % n_r] for k in tasks])
    keys = np.array([plan.keys[k] for k in tasks], dtype=np.uint64)
    thrs = np.array([rb.packing.threshold(1.0 / plan.temperatures[k // n_r]) for k in tasks], dtype=np.uint64)
    ib, fb, _, _ = oracle.run_chains(plan.L, J, keys, thrs, hot=plan.hot, n_therm=plan.n_therm, n_bins=nb,
                                     sweeps_per_bin=plan.sweeps_per_bin, n_threads=1)
    return ib, fb


def main():
    rank, world, port, out = int(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3]), sys.argv[4]
    scan = dict(SCAN)
    if len(sys.argv) > 5:
        scan["temperatures"] = scan["temperatures"][: int(sys.argv[5])]
        scan["n_realizations"] = 1
    import torch.distributed as dist

    import oracle

    rb = importlib.import_module("rbim-fk-percolation_b200")
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        plan = rb.plan_temperature_scan(**scan)
        lo, hi = rb.shard_bounds(plan.n_tasks, rank, world)
        ib, fb = oracle_sums(rb, oracle, plan, range(lo, hi))
        full_i, full_f = rb.gather_task_sums(ib, fb, plan.n_tasks, plan.n_bins)
        res = rb.assemble_scan(plan, full_i, full_f)
        flat = {f"{k}__{f}": v for k, e in res["observables"].items() for f, v in e.items()}
        np.savez(os.path.join(out, f"rank{rank}.npz"), full_i=full_i, full_f=full_f, lo=lo, hi=hi, **flat)
        dist.barrier()
    finally:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
