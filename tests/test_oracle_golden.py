"""The CPU oracle pinned against golden vectors produced by the reference itself.

Fixtures come from ``tests/golden/make_golden.py`` (reference union-find,
``_unionfind.py:91-136``; spanning-forest oracle, ``tests/test_wrapping.py:22-64``;
``cluster_statistics``/``_two_largest``/``energy``/``magnetization``).  The
Philox known-answer vectors are the published Random123 ones.
"""

import numpy as np
import pytest

from conftest import golden


def test_philox_known_answers(orc):
    kat = [
        ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]
    for ctr, key, want in kat:
        assert tuple(int(v) for v in orc.philox4x32_10(ctr, key)) == want


def test_union_find_matches_reference(orc, label_kat):
    for i in range(len(label_kat)):
        c = label_kat.case(i)
        n, labels, wx, wy = orc.label_and_wrap(c["active"], c["L"])
        assert n == c["n_clusters"], i
        assert np.array_equal(labels, c["labels"]), i
        assert (wx, wy) == c["wraps"], i


def test_spanning_forest_oracle_matches_reference(orc, label_kat):
    checked = wrapping = 0
    for i in range(len(label_kat)):
        c = label_kat.case(i)
        if not c["has_bf"]:
            continue
        got = orc.spanning_forest_winding(c["active"], c["L"])
        assert got == c["bf"] == c["wraps"], i
        checked += 1
        wrapping += any(got)
    assert checked > 100 and wrapping > 20


def test_statistics_match_reference(orc):
    d = golden("stats.npz")
    for i in range(d["L"].size):
        L = int(d["L"][i])
        spins = d["spins"][d["spin_offsets"][i]: d["spin_offsets"][i + 1]]
        J = d["J"][d["J_offsets"][i]: d["J_offsets"][i + 1]]
        m = d["masks"][d["mask_offsets"][i]: d["mask_offsets"][i + 1]]
        active = np.unpackbits(m, bitorder="little")[: 2 * L * L].astype(bool)
        n, labels, _, _ = orc.label_and_wrap(active, L)
        sizes, mags = orc.cluster_statistics(labels, spins, n)
        first, second = orc.two_largest(sizes)
        assert n == d["n_clusters"][i]
        assert sizes[first] == d["s1"][i]
        assert (0 if second is None else sizes[second]) == d["s2"][i]
        if not d["top_tied"][i]:
            # With a tie for the largest size the reference's choice is
            # numpy.argpartition's; the oracle takes the smallest label.
            assert abs(mags[first]) == d["mc1"][i]
        assert orc.energy(L, spins, J) == d["energy"][i]
        assert orc.magnetization(spins) == d["magnetization"][i]


def test_activation_only_satisfied_and_limits(orc):
    rng = np.random.default_rng(7)
    L = 12
    J = np.where(rng.random(2 * L * L) < 0.3, -1, 1).astype(np.int8)
    spins = np.where(rng.random(L * L) < 0.5, -1, 1).astype(np.int8)
    thr = int(np.floor(-np.expm1(-1.2) * 2**32))
    occ = orc.activate(L, spins, J, key=123, thr=thr, sweep=5)
    a = np.arange(2 * L * L) >> 1
    x, y = a // L, a % L
    b = np.where(np.arange(2 * L * L) % 2 == 0, ((x + 1) % L) * L + y, x * L + (y + 1) % L)
    sat = J * spins[a] * spins[b] > 0
    assert not np.any(occ & ~sat)
    assert occ.sum() > 0
    assert not orc.activate(L, spins, J, key=1, thr=0, sweep=0).any()
    assert np.array_equal(orc.activate(L, spins, J, key=1, thr=2**32, sweep=0), sat)


def test_lazy_activation_equals_full_uniform_comparison(orc):
    """The oracle's eight-bonds-per-block activation equals comparing each bond's 32-bit uniform with thr."""
    L, key, sweep = 9, 4242, 11
    rng = np.random.default_rng(3)
    J = np.where(rng.random(2 * L * L) < 0.3, -1, 1).astype(np.int8)
    spins = np.where(rng.random(L * L) < 0.5, -1, 1).astype(np.int8)
    a = np.arange(2 * L * L) >> 1
    x, y = a // L, a % L
    b = np.where(np.arange(2 * L * L) % 2 == 0, ((x + 1) % L) * L + y, x * L + (y + 1) % L)
    sat = J * spins[a] * spins[b] > 0
    uni = np.array([orc.bond_uniform(key, sweep, k) for k in range(2 * L * L)], dtype=np.uint64)
    thrs = [0, 1, 2**31, 2**32 - 1, 2**32]
    thrs += [int(uni[k] >> 16 << 16) | lo for k in (0, 5, 77) for lo in (0, 0x8000, 0xFFFF)]
    for thr in thrs:
        want = sat & (uni < thr)
        assert np.array_equal(orc.activate(L, spins, J, key=key, thr=thr, sweep=sweep), want), thr


def test_chain_is_deterministic_and_binning_invariant(orc):
    L = 8
    J = np.ones(2 * L * L, dtype=np.int8)
    thr = int(np.floor(-np.expm1(-2 / 2.3) * 2**32))
    a = orc.run_chain(L, J, 99, thr, n_therm=20, n_bins=4, sweeps_per_bin=25)
    b = orc.run_chain(L, J, 99, thr, n_therm=20, n_bins=4, sweeps_per_bin=25)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    c = orc.run_chain(L, J, 99, thr, n_therm=20, n_bins=10, sweeps_per_bin=10)
    assert np.array_equal(a[0].sum(axis=0), c[0].sum(axis=0))
    assert np.allclose(a[1].sum(axis=0), c[1].sum(axis=0), rtol=1e-12)


@pytest.mark.parametrize("L", [3, 6, 10])
def test_oracle_sweeps_against_spanning_forest(orc, L):
    """Wrap flags of sampled sweeps agree with the independent forest oracle."""
    rng = np.random.default_rng(L)
    J = np.where(rng.random(2 * L * L) < 0.1, -1, 1).astype(np.int8)
    spins = orc.initial_spins(L * L, key=L, hot=True)
    seen = 0
    for T in (1.0, 2.27, 4.0):
        thr = int(np.floor(-np.expm1(-2 / T) * 2**32))
        for t in range(8):
            occ = orc.activate(L, spins, J, key=L, thr=thr, sweep=t)
            _, _, wx, wy = orc.label_and_wrap(occ, L)
            assert (wx, wy) == orc.spanning_forest_winding(occ, L)
            seen += wx or wy
            orc.sw_sweep(L, spins, J, key=L, thr=thr, sweep=t, measure=False)
    assert seen > 0
