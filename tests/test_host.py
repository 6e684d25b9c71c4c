"""Host-side logic: geometry, disorder, packing, seeding, estimators and file formats (no GPU).

Mirrors the reference's ``tests/test_lattice.py`` and the parts of
``tests/test_physics.py`` that need no simulation, and pins the vectorised
jackknife against the reference's ``_combine_realizations`` output.
"""

import numpy as np
import pytest

from conftest import golden


@pytest.mark.parametrize("L", [3, 4, 8])
def test_bond_count_and_degree(rb, L):
    lattice = rb.build_lattice(L)
    assert lattice.n_sites == L * L and lattice.bonds.shape == (2 * L * L, 2)
    assert np.all(np.bincount(lattice.bonds.reshape(-1), minlength=lattice.n_sites) == 4)


@pytest.mark.parametrize("L", [3, 5, 8])
def test_wrap_masks(rb, L):
    lattice = rb.build_lattice(L)
    assert lattice.wraps_x.sum() == L and lattice.wraps_y.sum() == L
    assert not np.any(lattice.wraps_x & lattice.wraps_y)
    assert np.all(lattice.bonds[lattice.wraps_x, 0] // L == L - 1)
    assert np.all(lattice.bonds[lattice.wraps_y, 0] % L == L - 1)


def test_bond_ordering_matches_coupling_layout(rb):
    L = 4
    lattice = rb.build_lattice(L)
    J_h = np.arange(L * L, dtype=np.int8).reshape(L, L)
    J_v = -np.arange(L * L, dtype=np.int8).reshape(L, L)
    J = rb.couplings_from_disorder(J_h, J_v)
    for x in range(L):
        for y in range(L):
            n = rb.site_index(x, y, L)
            assert J[2 * n] == J_h[x, y] and J[2 * n + 1] == J_v[x, y]
            assert lattice.bonds[2 * n, 0] == n and lattice.bonds[2 * n + 1, 0] == n


def test_small_lattice_rejected(rb):
    with pytest.raises(ValueError):
        rb.build_lattice(2)


def test_frustration(rb):
    L = 6
    ones = np.ones((L, L), np.int8)
    assert rb.frustration_density(ones, ones) == 0.0
    J_h = ones.copy()
    J_h[2, 3] = -1
    fr = rb.frustrated_plaquettes(J_h, ones)
    assert fr.sum() == 2 and fr[2, 3] and fr[2, 2]
    rng = np.random.default_rng(12345)
    J_h, J_v = rb.generate_disorder(128, 0.3, rng)
    expected = 4 * 0.3 * 0.7 * (0.7**2 + 0.3**2)
    assert abs(rb.frustration_density(J_h, J_v) - expected) < 0.01


def test_disorder_generation_draws_like_the_reference(rb):
    """Same numpy calls as the reference (``disorder.py:59-60``): J_h then J_v from one generator."""
    rng = np.random.default_rng(9)
    J_h, J_v = rb.generate_disorder(5, 0.4, rng)
    rng2 = np.random.default_rng(9)
    u1, u2 = rng2.random((5, 5)), rng2.random((5, 5))
    assert np.array_equal(J_h, np.where(u1 < 0.4, -1, 1)) and np.array_equal(J_v, np.where(u2 < 0.4, -1, 1))
    assert J_h.dtype == np.int8
    with pytest.raises(ValueError):
        rb.generate_disorder(4, 1.5, rng)


@pytest.mark.parametrize("L,p,n", [(3, 0.05, 4), (17, 0.5, 3), (64, 1e-9, 2), (256, 0.1, 20), (9, 0.0, 2),
                                   (9, 1.0, 2)])
def test_batched_disorder_equals_the_reference_calls(rb, L, p, n):
    """generate_disorders (integer compares on the raw PCG64 draws, drawn in parallel chunks when many) gives the
    couplings of n reference calls ``rng.random((L, L)) < p`` (J_h, then J_v) in a row, and leaves the generator
    where those calls leave it."""
    a, b = np.random.default_rng(1000 + L), np.random.default_rng(1000 + L)
    got = rb.disorder.generate_disorders(L, p, a, n)
    for J_h, J_v in got:
        u1, u2 = b.random((L, L)), b.random((L, L))
        assert J_h.dtype == np.int8 and J_h.shape == (L, L)
        assert np.array_equal(J_h, np.where(u1 < p, -1, 1)) and np.array_equal(J_v, np.where(u2 < p, -1, 1))
    assert a.bit_generator.state == b.bit_generator.state


def test_batched_disorder_in_groups(rb, monkeypatch):
    """Large batches are drawn in groups of realizations, one after the other: same couplings, same end state."""
    monkeypatch.setattr(rb.disorder, "_GROUP_DRAWS", 3000)
    a, b = np.random.default_rng(7), np.random.default_rng(7)
    got = rb.disorder.generate_disorders(20, 0.2, a, 9)
    for J_h, J_v in got:
        u1, u2 = b.random((20, 20)), b.random((20, 20))
        assert np.array_equal(J_h, np.where(u1 < 0.2, -1, 1)) and np.array_equal(J_v, np.where(u2 < 0.2, -1, 1))
    assert a.bit_generator.state == b.bit_generator.state


def test_child_keys_equal_spawned_children(rb):
    """Vectorised SeedSequence children: the same keys as spawn() + chain_key for many parents."""
    seeding = rb.seeding
    for seed in (0, 1, 12345, 2**32 + 7, 2**70 + 3, 2**127 + 11, [1, 2, 3], [2**40, 5]):
        for depth in (0, 1):
            a = np.random.SeedSequence(seed)
            b = np.random.SeedSequence(seed)
            if depth:
                a, b = a.spawn(5)[3], b.spawn(5)[3]
            a, b = a.spawn(2)[1], b.spawn(2)[1]
            want = np.array([rb.chain_key(c) for c in a.spawn(257)], dtype=np.uint64)
            assert np.array_equal(seeding.child_keys(b, 257), want), (seed, depth)
            b.spawn(257)
            more = np.array([rb.chain_key(c) for c in a.spawn(5)], dtype=np.uint64)
            assert np.array_equal(seeding.child_keys(b, 5), more), (seed, depth)
    assert seeding.child_keys(np.random.SeedSequence(3), 0).size == 0


def test_disorder_file_round_trip(rb, tmp_path):
    J_h, J_v = rb.generate_disorder(7, 0.2, np.random.default_rng(1))
    path = tmp_path / rb.default_disorder_filename(7, 0.2, 3)
    assert path.name == "disorder_L=7_p=0.200_r=0003.npz"
    rb.save_disorder(str(path), J_h, J_v, p=0.2, seed=5)
    a, b = rb.load_disorder(str(path))
    assert np.array_equal(a, J_h) and np.array_equal(b, J_v)
    bad = tmp_path / "bad.npz"
    np.savez(bad, foo=np.zeros(3))
    with pytest.raises(KeyError):
        rb.load_disorder(str(bad))


@pytest.mark.parametrize("L", [3, 5, 16, 33, 48])
def test_packing_round_trips(rb, L):
    rng = np.random.default_rng(L)
    spins = np.where(rng.random(L * L) < 0.5, -1, 1)
    w = rb.packing.pack_spins(spins, L)
    assert w.size == rb.packing.words_for(L) and w.size % 4 == 0
    assert np.array_equal(rb.packing.unpack_spins(w, L), spins)
    # Bits past L*L stay zero.
    bits = np.unpackbits(w.view(np.uint8), bitorder="little")
    assert not bits[L * L:].any()
    J = np.where(rng.random(2 * L * L) < 0.3, -1, 1).astype(np.int8)
    assert np.array_equal(rb.packing.unpack_couplings(rb.packing.pack_couplings(J, L), L), J)


def test_plane_words_match_the_library(rb):
    for L in (3, 7, 32, 48, 100, 256, 1024):
        assert rb.packing.words_for(L) == rb._native.plane_words(L)


def test_threshold(rb):
    assert rb.packing.threshold(0.0) == 0
    assert rb.packing.threshold(50.0) == 2**32
    assert rb.packing.threshold(0.5) == int(np.floor((1 - np.exp(-1.0)) * 2**32))
    assert rb.bond_activation_probability(0.0) == pytest.approx(0.0)
    assert rb.bond_activation_probability(100.0) == pytest.approx(1.0)


def test_auto_engine_choice(rb):
    """engine="auto", one lattice: one resident CTA for L <= SINGLE_CTA_MAX_L (512 threads up to L = 32, 1024
    above), else the grid engine where it has a plan, else the plain engine; batched for every other set."""
    eng = rb.engine
    spec = lambda L: rb.ChainSpec(L=L, realization=0, key=1, beta=0.5, n_therm=0, n_bins=1, sweeps_per_bin=1)
    m = eng.SINGLE_CTA_MAX_L
    plan = lambda L: (148, 1024) if 32 < L <= 3000 else None
    assert eng.auto_engine([spec(m + 1)], plan) == "grid" and eng.auto_engine([spec(1024)], plan) == "grid"
    assert eng.auto_engine([spec(m)], plan) == "batched" and eng.auto_engine([spec(16)], plan) == "batched"
    assert eng.auto_engine([spec(4096)], plan) == "plain"
    assert eng.auto_engine([spec(m + 1)], lambda L: None) == "plain"
    assert eng.auto_engine([spec(1024), spec(1024)], plan) == "batched"
    assert [eng.single_cta_threads(L) for L in (3, 32, 33, 64)] == [512, 512, 1024, 1024]


def test_chain_keys_follow_seed_sequences(rb):
    ss = np.random.SeedSequence(0)
    _, run = ss.spawn(2)
    kids = run.spawn(3)
    keys = [rb.chain_key(k) for k in kids]
    assert len(set(keys)) == 3
    w = kids[1].generate_state(2, np.uint32)
    assert keys[1] == int(w[0]) | (int(w[1]) << 32)
    assert rb.chain_key(5) == rb.chain_key(np.random.SeedSequence(5))


def _results_from_fixture(rb, d, ci):
    n_r, n_bins, T, N = d[f"c{ci}_meta"]
    prim, bins = d[f"c{ci}_prim"], d[f"c{ci}_bins"]
    out = []
    for r in range(int(n_r)):
        out.append(rb.RealizationResult(
            primitives={n: float(prim[r, k]) for k, n in enumerate(rb.PRIMITIVES)},
            bin_primitives={n: bins[r, k].copy() for k, n in enumerate(rb.PRIMITIVES)}))
    return out, float(T), int(N)


@pytest.mark.parametrize("ci", [0, 1, 2])
def test_jackknife_matches_reference(rb, ci):
    d = golden("combine.npz")
    results, T, N = _results_from_fixture(rb, d, ci)
    combined = rb.combine_realizations(results, T, N)
    names = list(d["observables"])
    assert names == list(rb.OBSERVABLES)
    for key, arr in (("value", d[f"c{ci}_value"]), ("error", d[f"c{ci}_error"]),
                     ("thermal_error", d[f"c{ci}_thermal"])):
        got = np.array([combined[n][key] for n in names])
        np.testing.assert_allclose(got, arr, rtol=1e-11, atol=1e-14, equal_nan=True)


def test_realization_from_sums(rb):
    ib = np.zeros((2, 12), np.int64)
    fb = np.zeros((2, 2))
    ib[0, 0], ib[1, 0] = -30, -50          # energy sums of two bins of 5 sweeps
    ib[0, 9], ib[1, 9] = 5, 0              # wrap_x
    fb[:, 0] = [10.0, 20.0]
    r = rb.realization_from_sums(ib, fb, 5)
    assert r.primitives["energy"] == -8.0
    assert np.array_equal(r.bin_primitives["energy"], [-6.0, -10.0])
    assert r.primitives["wrap_x"] == 0.5 and r.primitives["magnetization_4"] == 3.0
    r2 = rb.realization_from_sums(ib, fb, 5, measure_percolation=False)
    assert np.isnan(r2.primitives["wrap_x"]) and np.all(np.isnan(r2.bin_primitives["wrap_any"]))


def test_derive_observables_conventions(rb):
    prim = {n: 1.0 for n in rb.PRIMITIVES}
    prim.update(energy=-10.0, energy_sq=104.0, magnetization_sq=0.0, magnetization_4=0.0)
    d = rb.derive_observables(prim, 2.0, 4)
    assert d["specific_heat"] == pytest.approx(4.0 / (4.0 * 4))
    assert d["binder"] == 0.0


def test_results_file_format(rb, tmp_path):
    ref = rb.load_results(str(golden("results_format.npz").fid.name))
    assert set(ref["observables"]) == set(rb.OBSERVABLES)
    assert ref["metadata"]["L"] == 16
    path = tmp_path / "out" / "scan.npz"
    rb.save_results(str(path), ref)
    back = rb.load_results(str(path))
    for name in rb.OBSERVABLES:
        for key in ("value", "error", "thermal_error"):
            np.testing.assert_array_equal(back["observables"][name][key], ref["observables"][name][key])
    assert back["metadata"] == ref["metadata"]


def test_scan_argument_errors_before_any_device_work(rb):
    with pytest.raises(ValueError):
        rb.run_temperature_scan(8, 0.1, [2.0], n_sweeps=5, n_bins=10)
    with pytest.raises(ValueError):
        rb.run_temperature_scan(8, 0.1, [2.0], n_sweeps=100, n_bins=0)
    with pytest.raises(ValueError):
        rb.run_temperature_scan(8, 0.1, [2.0], start="warm")
    with pytest.raises(ValueError):
        rb.run_temperature_scan(8, 0.1, [2.0], n_realizations=3, disorder=[rb.generate_disorder(8, 0.1)])
    with pytest.raises(ValueError):
        rb.run_temperature_scan(2, 0.1, [2.0])
    with pytest.raises(ValueError):
        rb.run_single_realization(8, np.ones(128, np.int8), 2.0, n_sweeps=10, n_therm=1, n_bins=20)


def test_engine_refuses_to_run_without_cuda(rb):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(rb.RbimError):
        rb.run_temperature_scan(8, 0.1, [2.0], n_sweeps=20, n_bins=2)


def _per_temperature_assembly(rb, plan, int_sums, f_sums):
    """The per-temperature path: realization_from_sums and combine_realizations, one temperature at a time."""
    n_r = plan.n_realizations
    raw = [rb.realization_from_sums(int_sums[k], f_sums[k], plan.sweeps_per_bin, plan.measure_percolation)
           for k in range(plan.n_tasks)]
    out = {}
    for t, T in enumerate(plan.temperatures):
        out[t] = rb.combine_realizations(raw[t * n_r:(t + 1) * n_r], T, plan.L * plan.L)
    return out


@pytest.mark.parametrize("n_r,n_bins,measure", [(5, 4, True), (1, 6, True), (3, 1, False), (7, 10, True)])
def test_vectorised_assembly_matches_per_temperature(rb, n_r, n_bins, measure):
    rng = np.random.default_rng(n_r * 100 + n_bins)
    L, spb = 12, 9
    temps = [1.3, 2.1, 2.6, 3.4]
    plan = rb.ScanPlan(L=L, p=0.1, temperatures=temps, couplings=[np.ones(2 * L * L, np.int8)] * n_r,
                       keys=np.arange(len(temps) * n_r, dtype=np.uint64), n_sweeps=n_bins * spb, n_therm=3,
                       n_bins=n_bins, sweeps_per_bin=spb, seed=1, hot=True, start="hot", measure_percolation=measure)
    N = L * L
    n = plan.n_tasks
    E = rng.integers(-2 * N, 0, size=(n, n_bins, spb))
    M = rng.integers(-N, N + 1, size=(n, n_bins, spb))
    S1 = rng.integers(1, N + 1, size=(n, n_bins, spb))
    MC = rng.integers(0, N + 1, size=(n, n_bins, spb))
    S2 = rng.integers(0, N // 2, size=(n, n_bins, spb))
    NC = rng.integers(1, N, size=(n, n_bins, spb))
    WX = rng.integers(0, 2, size=(n, n_bins, spb))
    WY = rng.integers(0, 2, size=(n, n_bins, spb))
    ii = np.stack([E.sum(-1), (E * E).sum(-1), M.sum(-1), np.abs(M).sum(-1), (M * M).sum(-1), S1.sum(-1), MC.sum(-1),
                   S2.sum(-1), NC.sum(-1), WX.sum(-1), WY.sum(-1), (WX | WY).sum(-1)], axis=-1).astype(np.int64)
    ff = np.stack([((M * M).astype(float) ** 2).sum(-1), (MC / S1).sum(-1)], axis=-1)
    got = rb.assemble_scan(plan, ii, ff)["observables"]
    want = _per_temperature_assembly(rb, plan, ii, ff)
    for name in rb.OBSERVABLES:
        for field in ("value", "error", "thermal_error"):
            w = np.array([want[t][name][field] for t in range(len(temps))])
            np.testing.assert_allclose(got[name][field], w, rtol=1e-12, atol=1e-15, err_msg=f"{name} {field}")


def test_occupancy_threads(rb):
    """The resident CTA size doubles while every lattice of a launch still fits the GPU at twice the threads."""
    occ = rb.engine.occupancy_threads
    assert occ(32, 1280, 148) == 64  # the reference's L = 32 scan
    assert occ(32, 524288, 148) == 32  # a full GPU keeps one-warp CTAs
    assert occ(128, 16384, 148) == 128
    assert occ(128, 10, 148) == 1024 and occ(1024, 1, 148) == 1024
    assert occ(32, 2368, 148) == 64 and occ(32, 2369, 148) == 32
