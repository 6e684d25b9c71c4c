"""Task blocks on the GPU: a task's sums do not depend on its batch, and a one-rank NCCL scan equals the plain scan."""

import datetime
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SCAN = dict(L=24, p=0.08, temperatures=[1.5, 2.1, 2.5], n_realizations=4, n_sweeps=60, n_therm=6, n_bins=3, seed=5)


def test_task_blocks_equal_full_batch(rb):
    plan = rb.plan_temperature_scan(**SCAN)
    full_i, full_f = rb.run_scan_tasks(plan)
    for blocks in ([(0, 5), (5, 12)], [(0, 1), (1, 2), (2, 12)]):
        for lo, hi in blocks:
            bi, bf = rb.run_scan_tasks(plan, range(lo, hi))
            assert np.array_equal(bi, full_i[lo:hi])
            assert np.array_equal(bf.view(np.int64), full_f[lo:hi].view(np.int64))
    # Plain engine, one task alone: the same sums again.
    pi, pf = rb.run_scan_tasks(plan, [7], engine="plain")
    assert np.array_equal(pi[0], full_i[7])
    assert np.array_equal(pf[0].view(np.int64), full_f[7].view(np.int64))


def test_one_rank_nccl_scan_equals_scan(rb):
    import torch
    import torch.distributed as dist

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60), device_id=torch.device("cuda", 0))
    try:
        got = rb.run_temperature_scan_sharded(**SCAN)
    finally:
        dist.destroy_process_group()
    want = rb.run_temperature_scan(**SCAN)
    for name, entry in want["observables"].items():
        for field, v in entry.items():
            np.testing.assert_array_equal(got["observables"][name][field], v, err_msg=f"{name} {field}")
    assert got["metadata"]["ranks"] == 1
