"""The scan server: continuous batching gives every request exactly its stand-alone result.

Requests of different sizes arrive while others run (some admitted only when
memory frees up); each result must equal ``run_temperature_scan`` of the same
request alone -- values, errors and thermal errors bit for bit.
"""

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REQUESTS = [
    dict(L=16, p=0.05, temperatures=np.linspace(1.0, 3.0, 8), n_realizations=4, n_sweeps=300, n_bins=5, seed=1),
    dict(L=64, p=0.10, temperatures=np.linspace(1.5, 2.5, 6), n_realizations=5, n_sweeps=120, n_bins=4, seed=2),
    dict(L=33, p=0.0, temperatures=[2.269], n_realizations=3, n_sweeps=250, n_bins=5, seed=3, start="cold"),
    dict(L=256, p=0.08, temperatures=[1.6, 2.2], n_realizations=2, n_sweeps=60, n_bins=3, seed=4),
    dict(L=300, p=0.05, temperatures=[2.0], n_realizations=1, n_sweeps=30, n_bins=3, seed=5),
    dict(L=48, p=0.12, temperatures=np.linspace(1.0, 3.0, 4), n_realizations=6, n_sweeps=90, n_bins=3, seed=6,
         measure_percolation=False),
]


def _assert_same(got, want):
    np.testing.assert_array_equal(got["temperatures"], want["temperatures"])
    for name, entry in want["observables"].items():
        for field, v in entry.items():
            np.testing.assert_array_equal(got["observables"][name][field], v, err_msg=f"{name} {field}")
    assert got["metadata"]["n_realizations"] == want["metadata"]["n_realizations"]


def test_requests_in_the_mix_equal_alone(rb):
    alone = [rb.run_temperature_scan(**r) for r in REQUESTS]
    with rb.ScanServer(memory_bytes=64 << 20, quantum=37) as server:
        futures = []
        for i, r in enumerate(REQUESTS):
            futures.append(server.submit(rb.ScanRequest(**r)))
            if i % 2:
                time.sleep(0.05)  # later requests arrive while earlier ones run
        results = [f.result(timeout=600) for f in futures]
    for got, want in zip(results, alone):
        _assert_same(got, want)
    assert len(server.completed) == len(REQUESTS)
    assert server.words.used == 0 and server.rows.used == 0


def test_admission_waits_for_memory(rb):
    """A pool that holds one L=64 request at a time still serves three, one after the other."""
    r = dict(L=64, p=0.05, temperatures=[1.8, 2.4], n_realizations=4, n_sweeps=40, n_bins=2)
    fp = rb.request_footprint(64, 2, 4, 2)
    server = rb.ScanServer(memory_bytes=int(fp["words"] * 4 / 0.75) + 64, quantum=10)
    futs = [server.submit(rb.ScanRequest(**r, seed=s)) for s in (7, 8, 9)]
    server.run_until_idle()
    for s, f in zip((7, 8, 9), futs):
        _assert_same(f.result(timeout=1), rb.run_temperature_scan(**r, seed=s))
    admitted = sorted(c["admitted"] for c in server.completed)
    finished = sorted(c["finished"] for c in server.completed)
    assert admitted[1] >= finished[0] and admitted[2] >= finished[1]


def test_oversize_request_is_rejected(rb):
    server = rb.ScanServer(memory_bytes=1 << 20)
    with pytest.raises(ValueError):
        server.submit(rb.ScanRequest(L=256, p=0.1, temperatures=np.linspace(1, 3, 64), n_realizations=64))


def test_request_beyond_cluster_sizes_equals_alone(rb):
    """A request whose lattices exceed the cluster engine's sizes is served over the whole GPU (grid engine),
    inside the quanta of the mix, with the stand-alone result."""
    big = rb._native.cluster_max_l() + 40
    reqs = [dict(L=big, p=0.10, temperatures=[1.6, 2.3], n_realizations=1, n_sweeps=24, n_bins=3, seed=8),
            dict(L=32, p=0.05, temperatures=[2.0, 2.4], n_realizations=3, n_sweeps=60, n_bins=3, seed=9)]
    alone = [rb.run_temperature_scan(**r) for r in reqs]
    with rb.ScanServer(memory_bytes=256 << 20, quantum=10) as server:
        results = [f.result(timeout=600) for f in [server.submit(rb.ScanRequest(**r)) for r in reqs]]
    for got, want in zip(results, alone):
        _assert_same(got, want)
