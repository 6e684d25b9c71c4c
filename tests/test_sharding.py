"""Sharded scans over gloo ranks on CPU: task blocks, the all-gather of bin sums and the assembled result.

Two (and three) processes each run their block of a scan's tasks with the
oracle's chain runner (the Philox chains the engine runs), gather the sums
with :func:`gather_task_sums` and assemble the jackknife result; every rank
must hold exactly the sums and observables of the unsharded scan.
"""

import os
import socket
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import shard_worker  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run_ranks(world, out, extra=()):
    port = _free_port()
    env = dict(os.environ, OMP_NUM_THREADS="1")
    procs = [subprocess.Popen([sys.executable, os.path.join(HERE, "shard_worker.py"), str(r), str(world), str(port),
                               str(out), *extra], env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
             for r in range(world)]
    logs = []
    for p in procs:
        try:
            logs.append(p.communicate(timeout=180)[0].decode(errors="replace"))
        except subprocess.TimeoutExpired:
            p.kill()
            logs.append(p.communicate()[0].decode(errors="replace"))
    for p, log in zip(procs, logs):
        assert p.returncode == 0, log[-3000:]
    return [dict(np.load(os.path.join(out, f"rank{r}.npz"))) for r in range(world)]


def test_shard_bounds_cover_tasks_once(rb):
    for n in (0, 1, 5, 64, 127):
        for world in (1, 2, 3, 8):
            blocks = [rb.shard_bounds(n, r, world) for r in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(blocks, blocks[1:]))
            sizes = [hi - lo for lo, hi in blocks]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        rb.shard_bounds(4, 2, 2)


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_scan_equals_unsharded(rb, orc, tmp_path, world):
    plan = rb.plan_temperature_scan(**shard_worker.SCAN)
    want_i, want_f = shard_worker.oracle_sums(rb, orc, plan, range(plan.n_tasks))
    want = rb.assemble_scan(plan, want_i, want_f)
    outs = _run_ranks(world, tmp_path)
    for r, got in enumerate(outs):
        assert (int(got["lo"]), int(got["hi"])) == rb.shard_bounds(plan.n_tasks, r, world)
        assert np.array_equal(got["full_i"], want_i)
        assert np.array_equal(got["full_f"].view(np.int64), want_f.view(np.int64))
        for name, entry in want["observables"].items():
            for field, v in entry.items():
                np.testing.assert_array_equal(got[f"{name}__{field}"], v, err_msg=f"{name} {field}")


def test_rank_with_no_tasks(rb, orc, tmp_path):
    """Two tasks over three ranks: the last rank holds none and still takes part in the gather."""
    scan = dict(shard_worker.SCAN, temperatures=shard_worker.SCAN["temperatures"][:2], n_realizations=1)
    plan = rb.plan_temperature_scan(**scan)
    want_i, want_f = shard_worker.oracle_sums(rb, orc, plan, range(plan.n_tasks))
    outs = _run_ranks(3, tmp_path, extra=("2",))
    assert int(outs[2]["hi"]) == int(outs[2]["lo"])
    for got in outs:
        assert np.array_equal(got["full_i"], want_i)
        assert np.array_equal(got["full_f"].view(np.int64), want_f.view(np.int64))
