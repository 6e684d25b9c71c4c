"""Bit-exact parity of activation, sweeps and whole chains against the oracle's Philox replay.

The engine and the oracle draw the same Philox4x32-10 stream, so for a fixed
key every occupation mask, flip, per-sweep record, per-bin sum and final spin
configuration must agree exactly; the integer sums are compared as integers
and the two double sums (M^4, |M_C1|/S1) bit for bit, since both sides add
the same values in the same order.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _thr(T):
    return int(np.floor(-np.expm1(-2.0 * (1.0 / T)) * 2**32))


def _couplings(L, p, seed):
    rng = np.random.default_rng(seed)
    return np.where(rng.random(2 * L * L) < p, -1, 1).astype(np.int8)


@pytest.mark.parametrize("L", [3, 5, 16, 33, 64, 100, 250])
def test_activation_matches_philox_replay(rb, orc, L):
    rng = np.random.default_rng(L)
    J = _couplings(L, 0.2, L)
    spins = np.where(rng.random(L * L) < 0.5, -1, 1).astype(np.int8)
    lattice = rb.build_lattice(L)
    for T, sweep in ((0.5, 0), (2.27, 7), (4.0, 2**33 + 5)):
        got = rb.activate_bonds(spins, lattice, J, 1.0 / T, key=0xABCDEF123 + L, sweep=sweep)
        want = orc.activate(L, spins, J, key=0xABCDEF123 + L, thr=rb.packing.threshold(1.0 / T), sweep=sweep)
        assert np.array_equal(got, want), (L, T)


def test_activation_refinement_branch(rb, orc):
    """Thresholds whose high half equals a bond's 16-bit draw force the second-stream draw."""
    L, key, sweep = 16, 0x5EED, 3
    lattice = rb.build_lattice(L)
    J = np.ones(2 * L * L, dtype=np.int8)
    spins = np.ones(L * L, dtype=np.int8)  # every bond satisfied
    lib = rb._native.lib()
    for k in (0, 7, 8, 101, 2 * L * L - 1):
        u = orc.bond_uniform(key, sweep, k) >> 16
        for lo in (0, 0x7FFF, 0xFFFF):
            thr = (u << 16) | lo
            want = orc.activate(L, spins, J, key=key, thr=thr, sweep=sweep)
            got = _activate_thr(rb, lib, L, spins, J, key, thr, sweep)
            assert np.array_equal(got, want), (k, lo)
            full = orc.bond_uniform(key, sweep, k)
            assert bool(want[k]) == (full < thr)


def _activate_thr(rb, lib, L, spins, J, key, thr, sweep):
    import ctypes
    import torch

    s = torch.from_numpy(rb.packing.pack_spins(spins, L).view(np.int32)).cuda()
    j = torch.from_numpy(rb.packing.pack_couplings(J, L).view(np.int32)).cuda()
    occ = torch.empty(2 * L * L, dtype=torch.uint8, device="cuda")
    ws = torch.empty(int(lib.rbim_activate_workspace_bytes(L)), dtype=torch.uint8, device="cuda")
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    rc = lib.rbim_activate(L, p(s), p(j), key, thr, sweep, p(occ), p(ws), ws.numel(),
                           ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    rb._native.check(rc, "rbim_activate")
    return occ.cpu().numpy().astype(bool)


def test_activation_limits(rb):
    """Reference ``tests/test_clusters.py:30-59``: beta = 0 activates nothing, beta = 50 everything satisfied."""
    L = 8
    lattice = rb.build_lattice(L)
    J = np.ones(2 * L * L, dtype=np.int8)
    spins = np.ones(L * L, dtype=np.int64)
    assert not rb.activate_bonds(spins, lattice, J, 0.0, key=1).any()
    full = rb.activate_bonds(spins, lattice, J, 50.0, key=1)
    assert full.all()
    n, _, wx, wy = rb.label_and_wrap(full, lattice)
    assert n == 1 and wx and wy


def _chain(rb, orc, Ls, engine, n_therm=5, n_bins=3, spb=7, p=0.1, temps=(1.0, 2.27, 4.0), records=False,
           chunks=None):
    specs, couplings, J_host = [], [], []
    for i, L in enumerate(Ls):
        J = _couplings(L, p, 100 + i)
        couplings.append(rb.packing.pack_couplings(J, L))
        J_host.append(J)
        T = temps[i % len(temps)]
        specs.append(rb.ChainSpec(L=L, realization=i, key=(0x1234567 * (i + 1)) & (2**64 - 1), beta=1.0 / T,
                                  n_therm=n_therm, n_bins=n_bins, sweeps_per_bin=spb, records=records))
    cs = rb.ChainSet(specs, couplings)
    cs.init_spins(hot=True)
    total = n_therm + n_bins * spb
    for n in chunks or [total]:
        if engine == "batched":
            cs.run_batched(n)
        else:
            cs.run_plain(n)
    cs.check_status()
    assert np.all(cs.device_sweeps() == total)
    for i, s in enumerate(specs):
        ib, fb, spins = orc.run_chain(s.L, J_host[i], s.key, rb.packing.threshold(s.beta), hot=True, n_therm=n_therm,
                                      n_bins=n_bins, sweeps_per_bin=spb)
        gi, gf = cs.bins(i)
        assert np.array_equal(gi, ib), (engine, s.L, i)
        assert np.array_equal(gf.view(np.uint64), fb.view(np.uint64)), (engine, s.L, i)
        assert np.array_equal(cs.spins(i), spins.astype(np.int64)), (engine, s.L, i)
    return cs, specs, J_host


@pytest.mark.parametrize("L", [3, 4, 8, 16, 32, 48, 64, 80, 100, 150, 180])
def test_batched_chain_bit_exact(rb, orc, L):
    _chain(rb, orc, [L] * 6, "batched")


@pytest.mark.parametrize("L", [3, 8, 32, 64, 128])
def test_plain_chain_bit_exact(rb, orc, L):
    _chain(rb, orc, [L] * 2, "plain")


@pytest.mark.parametrize("L", [300, 512, 1024, 1500])
def test_plain_chain_bit_exact_large(rb, orc, L):
    """The plain engine at the sizes engine="auto" sends to it: every single lattice with L > 128, and every
    lattice beyond the cluster engine (L > 1024).  p = 0.10 at T = 1.6 (one cluster spans the lattice) and at
    T_c of the pure model."""
    _chain(rb, orc, [L, L], "plain", n_therm=2, n_bins=2, spb=2, temps=(1.6, 2.269))


def test_plain_records_large(rb, orc):
    """Per-sweep records of the plain engine at L = 512, |M_C2| included, equal the oracle's sweep by sweep."""
    L, n_therm, spb = 512, 1, 2
    cs, specs, J_host = _chain(rb, orc, [L], "plain", n_therm=n_therm, n_bins=2, spb=spb, temps=(2.269,),
                               records=True)
    recs = cs.chain_records(0)
    s = specs[0]
    spins = orc.initial_spins(L * L, s.key, hot=True)
    for t in range(n_therm + 2 * spb):
        r = orc.sw_sweep(L, spins, J_host[0], s.key, rb.packing.threshold(s.beta), t, measure=t >= n_therm)
        if t >= n_therm:
            assert tuple(int(v) for v in recs[t - n_therm]) == tuple(int(v) for v in r), t


def test_batched_uneven_sizes_one_launch(rb, orc):
    _chain(rb, orc, [32, 48, 64, 96, 128, 5, 17, 200], "batched", n_therm=3, n_bins=2, spb=4)


def test_chunked_calls_equal_one_call(rb, orc):
    _chain(rb, orc, [24] * 4, "batched", n_therm=4, n_bins=3, spb=5, chunks=[1, 3, 2, 5, 4, 100])
    _chain(rb, orc, [24] * 2, "plain", n_therm=4, n_bins=3, spb=5, chunks=[2, 7, 100])


def test_records_match_oracle_sweeps(rb, orc):
    L, n_therm, spb = 20, 3, 6
    for engine in ("batched", "plain"):
        cs, specs, J_host = _chain(rb, orc, [L] * 3, engine, n_therm=n_therm, n_bins=2, spb=spb, records=True)
        for i, s in enumerate(specs):
            recs = cs.chain_records(i)
            spins = orc.initial_spins(L * L, s.key, hot=True)
            for t in range(n_therm + 2 * spb):
                r = orc.sw_sweep(L, spins, J_host[i], s.key, rb.packing.threshold(s.beta), t, measure=t >= n_therm)
                if t >= n_therm:
                    assert tuple(int(v) for v in recs[t - n_therm]) == tuple(int(v) for v in r), (engine, i, t)


def test_largest_lattice_on_chip_and_beyond(rb, orc):
    lmax = rb._native.resident_max_l()
    _chain(rb, orc, [lmax], "batched", n_therm=1, n_bins=1, spb=2, temps=(1.5,))
    _chain(rb, orc, [lmax + 1], "plain", n_therm=1, n_bins=1, spb=2, temps=(1.5,))


def test_cold_start_and_zero_temperature_limit(rb):
    """A cold ferromagnet at T -> 0 is one wrapping cluster every sweep."""
    L = 16
    J = np.ones(2 * L * L, dtype=np.int8)
    spec = rb.ChainSpec(L=L, realization=0, key=5, beta=50.0, n_therm=0, n_bins=1, sweeps_per_bin=10, records=True)
    cs = rb.ChainSet([spec], [rb.packing.pack_couplings(J, L)])
    cs.init_spins(hot=False)
    cs.run_batched(10)
    rec = cs.chain_records(0)
    assert np.all(rec[:, 2] == 1) and np.all(rec[:, 3] == L * L) and np.all(rec[:, 7] == 1) and np.all(rec[:, 8] == 1)
    assert np.all(rec[:, 5] == 0) and np.all(rec[:, 6] == 0)
    assert np.all(np.abs(rec[:, 1]) == L * L) and np.all(rec[:, 0] == -2 * L * L)


def test_sw_sweep_api_matches_oracle(rb, orc):
    L = 12
    lattice = rb.build_lattice(L)
    J = _couplings(L, 0.15, 9)
    spins = orc.initial_spins(L * L, 77, hot=True).astype(np.int64)
    ref = spins.astype(np.int8).copy()
    for t in range(4):
        res = rb.sw_sweep(spins, lattice, J, 1 / 1.8, key=77, sweep=t)
        r = orc.sw_sweep(L, ref, J, 77, rb.packing.threshold(1 / 1.8), t, measure=True)
        assert (res.energy, res.magnetization, res.n_clusters, res.largest_size, res.largest_abs_magnetization,
                res.second_size, res.second_abs_magnetization, res.wraps_x, res.wraps_y) == (
                    r[0], r[1], r[2], r[3], r[4], r[5], r[6], bool(r[7]), bool(r[8]))
        assert np.array_equal(spins, ref.astype(np.int64))


@pytest.mark.parametrize("L", [24, 48, 100, 160])
def test_single_realization_engines_agree(rb, L):
    """run_single_realization gives the same sums on every engine; engine="auto" takes one resident CTA (of the
    single-lattice size) for L <= SINGLE_CTA_MAX_L and the grid engine above."""
    J = _couplings(L, 0.08, L)
    engines = ("auto", "plain", "batched") + (("grid",) if L > 32 else ())
    out = {e: rb.run_single_realization(L, J, 2.1, n_sweeps=24, n_therm=4, n_bins=4, seed=11, engine=e)
           for e in engines}
    for e in engines[1:]:
        for k, v in out["auto"].primitives.items():
            assert np.array_equal(np.float64(v).view(np.uint64), np.float64(out[e].primitives[k]).view(np.uint64)), (e, k)
        for k, v in out["auto"].bin_primitives.items():
            assert np.array_equal(np.asarray(v, np.float64).view(np.uint64),
                                  np.asarray(out[e].bin_primitives[k], np.float64).view(np.uint64)), (e, k)


@pytest.mark.parametrize("L", [24, 200])
def test_plain_graph_replay_equals_direct_launches(rb, L):
    """run_plain replays a captured CUDA graph of its launch sequence; the state after any mix of replayed and
    directly launched calls equals the state after direct launches alone, bit for bit."""
    out = []
    for graph in (True, False):
        J = _couplings(L, 0.1, 5)
        spec = rb.ChainSpec(L=L, realization=0, key=42, beta=1 / 2.1, n_therm=3, n_bins=3, sweeps_per_bin=9,
                            records=True)
        cs = rb.ChainSet([spec], [rb.packing.pack_couplings(J, L)])
        cs.init_spins(hot=True)
        for n in (8, 8, 3, 8, 100):
            cs.run_plain(n, graph=graph)
        cs.check_status()
        assert (len(cs._graphs) == 2) == graph  # calls of 8 and of 100 sweeps
        out.append((cs.acc_int.cpu().numpy(), cs.acc_f64.cpu().numpy().view(np.int64), cs.spin_pool.cpu().numpy(),
                    cs.records.cpu().numpy(), cs.device_sweeps()))
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_sw_sweep_reused_state_does_not_leak(rb, orc):
    """sw_sweep keeps one device chain set per L; calls that alternate sizes, couplings, keys, temperatures and
    measured or unmeasured sweeps each still equal the oracle's sweep."""
    cases = []
    for L, seed in ((12, 1), (20, 2), (12, 3), (20, 4), (12, 1)):
        J = _couplings(L, 0.15, seed)
        spins = orc.initial_spins(L * L, 100 + seed, hot=True).astype(np.int64)
        cases.append((L, J, spins, 100 + seed))
    for step in range(3):
        for L, J, spins, key in cases:
            T = 1.6 + 0.3 * step
            measure = step != 1
            ref = spins.astype(np.int8).copy()
            res = rb.sw_sweep(spins, rb.build_lattice(L), J, 1 / T, key=key, sweep=step, measure=measure)
            r = orc.sw_sweep(L, ref, J, key, rb.packing.threshold(1 / T), step, measure=measure)
            assert np.array_equal(spins, ref.astype(np.int64)), (L, key, step)
            if measure:
                assert (res.energy, res.magnetization, res.n_clusters, res.largest_size, res.second_size,
                        res.second_abs_magnetization) == (r[0], r[1], r[2], r[3], r[5], r[6])
            else:
                assert res is None


def test_batched_set_beyond_cluster_sizes_runs_on_whole_gpu(rb, orc):
    """A batched set whose largest lattice exceeds the cluster engine's sizes runs that lattice over the whole
    GPU (grid engine) after the on-chip launches; every chain still equals the oracle's."""
    big = rb._native.cluster_max_l() + 40
    cs, specs, _ = _chain(rb, orc, [48, big, 96], "batched", n_therm=1, n_bins=1, spb=2, temps=(1.6, 2.269, 3.0))
    assert [specs[i].L for i in cs.plain_only] == [big] and cs.grid_ok(big)
