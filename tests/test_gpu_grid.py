"""Grid engine (``rbim_sweeps_grid``): one lattice over a cooperative grid of CTAs, bit for bit against the oracle.

Each CTA keeps one tile of consecutive sites in shared memory; clusters that
cross tiles or the periodic seams are merged in a union-find in global memory
between grid-wide barriers.  Results must not depend on the plan (number of
tiles, CTA size): every case is compared with the oracle's restatement of the
reference's sweep (src/rbim/swendsen_wang.py:103-172) run as one chain of
src/rbim/simulation.py:196-242.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIND_CAP, UNION_CAP, BAD_CHAIN, GRID_WAIT = 1, 2, 4, 8


def _couplings(L, p, seed):
    rng = np.random.default_rng(seed)
    return np.where(rng.random(2 * L * L) < p, -1, 1).astype(np.int8)


def _chain_set(rb, L, T, p=0.1, seed=0, n_therm=3, n_bins=2, spb=3, records=False, hot=True):
    J = _couplings(L, p, 1000 + L + seed)
    spec = rb.ChainSpec(L=L, realization=0, key=(0x9E3779B97F4A7C15 * (L + 7 * seed + 1)) & (2**64 - 1), beta=1.0 / T,
                        n_therm=n_therm, n_bins=n_bins, sweeps_per_bin=spb, records=records)
    cs = rb.ChainSet([spec], [rb.packing.pack_couplings(J, L)])
    cs.init_spins(hot=hot)
    return cs, spec, J


def _assert_oracle(rb, orc, cs, spec, J, hot=True):
    ib, fb, spins = orc.run_chain(spec.L, J, spec.key, rb.packing.threshold(spec.beta), hot=hot, n_therm=spec.n_therm,
                                  n_bins=spec.n_bins, sweeps_per_bin=spec.sweeps_per_bin)
    gi, gf = cs.bins(0)
    assert np.array_equal(gi, ib), (spec.L, spec.beta)
    assert np.array_equal(gf.view(np.uint64), fb.view(np.uint64)), (spec.L, spec.beta)
    assert np.array_equal(cs.spins(0), spins.astype(np.int64)), (spec.L, spec.beta)


@pytest.mark.parametrize("L", [33, 40, 64, 100, 128, 200, 256, 300, 512])
@pytest.mark.parametrize("T", [1.6, 2.269, 4.0])
def test_grid_chain_bit_exact(rb, orc, L, T):
    """Default plan, the run split over three calls (the state between calls is the spin plane)."""
    cs, spec, J = _chain_set(rb, L, T)
    total = spec.n_therm + spec.n_bins * spec.sweeps_per_bin
    for n in (2, 4, total):
        cs.run_grid(n)
    cs.check_status()
    assert cs.device_sweeps()[0] == total
    _assert_oracle(rb, orc, cs, spec, J)


@pytest.mark.parametrize("L", [1024, 1500])
def test_grid_chain_bit_exact_large(rb, orc, L):
    """The single-lattice sizes the grid engine is for: p = 0.10 at T = 1.6 (a cluster spans the lattice) and the
    pure model's T_c."""
    for T in (1.6, 2.269):
        cs, spec, J = _chain_set(rb, L, T, n_therm=2, n_bins=2, spb=2)
        cs.run_grid(6)
        cs.check_status()
        _assert_oracle(rb, orc, cs, spec, J)


@pytest.mark.parametrize("plan", [(2, 1024), (3, 512), (7, 256), (16, 1024), (37, 512), (64, 256), (128, 256)])
def test_grid_plans_agree(rb, orc, plan):
    """Results do not depend on the number of tiles or the CTA size (tiles start on 128-site Philox chunks)."""
    L = 256
    cs, spec, J = _chain_set(rb, L, 2.269, seed=3)
    total = spec.n_therm + spec.n_bins * spec.sweeps_per_bin
    cs.run_grid(total, plan=plan)
    cs.check_status()
    _assert_oracle(rb, orc, cs, spec, J)


def test_grid_records_match_oracle(rb, orc):
    """Per-sweep records (E, M, clusters, S1, |M_C1|, S2, |M_C2|, wraps) equal the oracle's sweep by sweep."""
    L, n_therm = 300, 2
    cs, spec, J = _chain_set(rb, L, 2.269, seed=5, n_therm=n_therm, n_bins=2, spb=3, records=True)
    total = n_therm + 6
    cs.run_grid(total)
    cs.check_status()
    rec = cs.chain_records(0)
    spins = orc.initial_spins(L * L, spec.key, hot=True)
    thr = rb.packing.threshold(spec.beta)
    for t in range(total):
        r = orc.sw_sweep(L, spins, J, spec.key, thr, t, measure=t >= n_therm)
        if t >= n_therm:
            assert tuple(int(v) for v in rec[t - n_therm]) == tuple(int(v) for v in r), t


def test_grid_one_cluster_and_cold_start(rb, orc):
    """A cold ferromagnet at low temperature: one cluster spans every tile (one root, S1 = N, no second)."""
    L = 200
    cs, spec, J = _chain_set(rb, L, 0.5, p=0.0, n_therm=1, n_bins=2, spb=2, records=True, hot=False)
    cs.run_grid(5)
    cs.check_status()
    rec = cs.chain_records(0)
    assert np.all(rec[:, 2] == 1) and np.all(rec[:, 3] == L * L) and np.all(rec[:, 5] == 0)
    assert np.all(rec[:, 7] == 1) and np.all(rec[:, 8] == 1)
    _assert_oracle(rb, orc, cs, spec, J, hot=False)


def test_grid_matches_plain_engine(rb):
    """The grid and plain engines give identical bin sums and spins for the same chain."""
    out = []
    for engine in ("grid", "plain"):
        cs, spec, J = _chain_set(rb, 384, 2.2, seed=9, n_therm=4, n_bins=3, spb=4)
        cs.run_to_end(engine=engine)
        gi, gf = cs.bins(0)
        out.append((gi, gf.view(np.uint64), cs.spins(0)))
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def _status(cs):
    import torch

    torch.cuda.synchronize()
    return int(cs.status.item())


def test_grid_wait_bound_reports_and_returns(rb, orc):
    """A wait bound of one clock cycle makes the barriers give up: the call returns with RBIM_STATUS_GRID_WAIT set
    and nothing left waiting, and the device then runs a fresh chain bit for bit."""
    cs, spec, J = _chain_set(rb, 256, 2.269)
    cs.run_grid(4, wait_cycles=1)
    st = _status(cs)
    assert st & GRID_WAIT, st
    with pytest.raises(rb.RbimError, match="status word"):
        cs.check_status()
    cs2, spec2, J2 = _chain_set(rb, 256, 2.269, seed=1)
    total = spec2.n_therm + spec2.n_bins * spec2.sweeps_per_bin
    cs2.run_grid(total)
    cs2.check_status()
    _assert_oracle(rb, orc, cs2, spec2, J2)


@pytest.mark.parametrize("field,value", [("sweeps_per_bin", 0), ("L", 129)])
def test_grid_bad_descriptor_rejected(rb, field, value):
    """A malformed descriptor (sweeps_per_bin = 0), or one whose L is not the call's, is rejected by every CTA
    before any barrier: the call returns, the chain is left unchanged."""
    cs, spec, J = _chain_set(rb, 128, 2.0)
    before = cs.spin_pool.clone()
    cs.set_descriptor_field(0, field, value)
    cs.run_grid(3)
    assert _status(cs) == BAD_CHAIN
    assert cs.device_sweeps()[0] == 0
    assert bool((cs.spin_pool == before).all())


def test_grid_walk_bound_fires(rb):
    """walk_cap = 1 bounds every union-find walk to one step; on a cold ferromagnet the bound fires, the call
    returns and the status word says so."""
    cs, spec, J = _chain_set(rb, 256, 0.5, p=0.0, hot=False)
    cs.set_descriptor_field(0, "walk_cap", 1)
    cs.run_grid(3)
    st = _status(cs)
    assert st & (FIND_CAP | UNION_CAP), st
    assert not st & (BAD_CHAIN | GRID_WAIT)
    assert cs.device_sweeps()[0] == 3


def test_grid_without_boundary_hash(rb, orc):
    """L = 2800: tiles of about 53,000 sites leave no shared memory for the boundary-bond hash, so every bond the
    neighbouring-lane filter keeps is unioned globally; the chain is still bit-exact."""
    cs, spec, J = _chain_set(rb, 2800, 2.269, n_therm=1, n_bins=1, spb=2)
    assert rb._native.grid_plan(2800) is not None
    cs.run_grid(3)
    cs.check_status()
    _assert_oracle(rb, orc, cs, spec, J)
