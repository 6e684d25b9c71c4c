"""The cluster engine (256 < L <= rbim_cluster_max_l()): bit-exact chains against the oracle.

Each lattice is split over the CTAs of a thread-block cluster, so these cases
cover tiles that start inside a row (odd L), a last tile whose end is not a
word boundary, clusters that cross several tiles and the x seam from the last
tile to the first, merged clusters larger than one tile (more than 65536
sites), and every cluster size from 2 to 16.
"""

import numpy as np
import pytest

from test_gpu_sweeps import _chain, _couplings

pytestmark = pytest.mark.gpu


def test_cluster_limit(rb):
    assert rb._native.cluster_max_l() >= 512


@pytest.mark.parametrize("L", [257, 300, 333, 384, 512])
def test_cluster_chain_bit_exact(rb, orc, L):
    _chain(rb, orc, [L] * 3, "batched", n_therm=2, n_bins=2, spb=3)


@pytest.mark.parametrize("L", [600, 723, 725, 1000, 1024])
def test_cluster_large_sizes(rb, orc, L):
    if L > rb._native.cluster_max_l():
        pytest.skip(f"L = {L} exceeds this device's cluster limit")
    _chain(rb, orc, [L], "batched", n_therm=1, n_bins=1, spb=3, temps=(1.6,))
    _chain(rb, orc, [L], "batched", n_therm=0, n_bins=1, spb=2, temps=(2.27,))


def test_resident_and_cluster_in_one_call(rb, orc):
    _chain(rb, orc, [64, 300, 17, 512, 256, 257], "batched", n_therm=2, n_bins=2, spb=2)


def test_cluster_chunked_calls_and_records(rb, orc):
    L, n_therm, spb = 301, 2, 3
    cs, specs, J_host = _chain(rb, orc, [L] * 2, "batched", n_therm=n_therm, n_bins=2, spb=spb, records=True,
                               chunks=[1, 2, 4, 100])
    for i, s in enumerate(specs):
        recs = cs.chain_records(i)
        spins = orc.initial_spins(L * L, s.key, hot=True)
        for t in range(n_therm + 2 * spb):
            r = orc.sw_sweep(L, spins, J_host[i], s.key, rb.packing.threshold(s.beta), t, measure=t >= n_therm)
            if t >= n_therm:
                assert tuple(int(v) for v in recs[t - n_therm]) == tuple(int(v) for v in r), (i, t)


@pytest.mark.parametrize("L", [300, 512])
def test_cluster_one_giant_cluster(rb, L):
    """A cold ferromagnet at T -> 0: one cluster of all L^2 > 65536 sites, wrapping both ways."""
    J = np.ones(2 * L * L, dtype=np.int8)
    spec = rb.ChainSpec(L=L, realization=0, key=5, beta=50.0, n_therm=0, n_bins=1, sweeps_per_bin=4, records=True)
    cs = rb.ChainSet([spec], [rb.packing.pack_couplings(J, L)])
    cs.init_spins(hot=False)
    cs.run_batched(4)
    cs.check_status()
    rec = cs.chain_records(0)
    assert np.all(rec[:, 2] == 1) and np.all(rec[:, 3] == L * L) and np.all(rec[:, 5] == 0)
    assert np.all(rec[:, 6] == 0) and np.all(rec[:, 7] == 1) and np.all(rec[:, 8] == 1)
    assert np.all(np.abs(rec[:, 1]) == L * L) and np.all(np.abs(rec[:, 4]) == L * L)
    assert np.all(rec[:, 0] == -2 * L * L)


def test_cluster_scan_equals_plain_engine(rb):
    """The same scan on the cluster engine and on the plain engine gives identical results."""
    kw = dict(L=260, p=0.08, temperatures=[1.5, 2.3], n_realizations=2, n_sweeps=12, n_therm=3, n_bins=3, seed=9)
    a = rb.run_temperature_scan(**kw, engine="batched")
    b = rb.run_temperature_scan(**kw, engine="plain")
    for name, entry in a["observables"].items():
        for field, v in entry.items():
            np.testing.assert_array_equal(v, b["observables"][name][field], err_msg=f"{name} {field}")


def test_cluster_label_consistency_with_wrapping(rb, orc):
    """Frozen-temperature check of wraps at criticality: records agree with the oracle sweep by sweep."""
    L = 320
    J = _couplings(L, 0.0, 3)
    spins = orc.initial_spins(L * L, 11, hot=True)
    spec = rb.ChainSpec(L=L, realization=0, key=11, beta=0.5 * np.log(1 + np.sqrt(2)), n_therm=0, n_bins=1,
                        sweeps_per_bin=6, records=True)
    cs = rb.ChainSet([spec], [rb.packing.pack_couplings(J, L)])
    cs.init_spins(hot=True)
    cs.run_batched(6)
    cs.check_status()
    rec = cs.chain_records(0)
    thr = rb.packing.threshold(spec.beta)
    for t in range(6):
        r = orc.sw_sweep(L, spins, J, 11, thr, t, measure=True)
        assert tuple(int(v) for v in rec[t]) == tuple(int(v) for v in r), t
