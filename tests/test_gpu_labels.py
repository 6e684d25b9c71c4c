"""Bit-exact labelling parity of the CUDA engine (C ABI ``rbim_label_wrap``).

Canonical labels, cluster counts and both wrap flags must equal the
reference's union-find (``_unionfind.py:91-136``) on every frozen mask; the
resident engine covers L <= rbim_resident_max_l() and the plain engine the
larger lattices.
"""

import hashlib

import numpy as np
import pytest

from conftest import big_mask, golden

pytestmark = pytest.mark.gpu


def test_reference_masks(rb, label_kat):
    by_L = {}
    for i in range(len(label_kat)):
        by_L.setdefault(label_kat.case(i)["L"], []).append(i)
    for L, idx in sorted(by_L.items()):
        cases = [label_kat.case(i) for i in idx]
        ncl, labels, wraps = rb.label_and_wrap_many(np.stack([c["active"] for c in cases]), L)
        for k, c in enumerate(cases):
            assert ncl[k] == c["n_clusters"], (L, idx[k])
            assert np.array_equal(labels[k], c["labels"]), (L, idx[k])
            assert tuple(bool(v) for v in wraps[k]) == c["wraps"], (L, idx[k])


@pytest.mark.parametrize("L", [3, 4, 7, 31, 32, 33, 47, 64, 100, 128, 200])
def test_random_masks_against_oracle(rb, orc, L):
    rng = np.random.default_rng(L)
    masks = np.stack([rng.random(2 * L * L) < q for q in (0.0, 0.2, 0.45, 0.5, 0.55, 0.8, 1.0)])
    ncl, labels, wraps = rb.label_and_wrap_many(masks, L)
    for k in range(masks.shape[0]):
        n, lab, wx, wy = orc.label_and_wrap(masks[k], L)
        assert ncl[k] == n and np.array_equal(labels[k], lab) and tuple(wraps[k]) == (wx, wy), (L, k)


def test_resident_boundary_sizes(rb, orc):
    """The largest resident L and the smallest plain-engine L."""
    lmax = rb._native.resident_max_l()
    for L in (lmax, lmax + 1):
        rng = np.random.default_rng(L)
        masks = np.stack([rng.random(2 * L * L) < q for q in (0.5, 0.7)])
        ncl, labels, wraps = rb.label_and_wrap_many(masks, L)
        for k in range(2):
            n, lab, wx, wy = orc.label_and_wrap(masks[k], L)
            assert ncl[k] == n and np.array_equal(labels[k], lab) and tuple(wraps[k]) == (wx, wy), (L, k)


def _check_big(rb, d, rows):
    for i in rows:
        L, seed = int(d["L"][i]), int(d["seed"][i])
        ncl, labels, wraps = rb.label_and_wrap_many(big_mask(L, seed)[None, :], L)
        lab = labels[0]
        assert ncl[0] == d["n_clusters"][i], (L, seed)
        assert tuple(bool(v) for v in wraps[0]) == tuple(bool(v) for v in d["wraps"][i]), (L, seed)
        sizes = np.bincount(lab, minlength=int(ncl[0]))
        top = np.sort(sizes)[::-1]
        assert top[0] == d["s1"][i] and (top[1] if top.size > 1 else 0) == d["s2"][i], (L, seed)
        assert hashlib.sha1(lab.astype("<i4").tobytes()).hexdigest() == str(d["sha1"][i]), (L, seed)


def test_critical_masks_large_lattices(rb):
    """Bond probability 1/2 at L = 256, 512, 1024: a subset of the golden KAT."""
    d = golden("label_kat_big.npz")
    rows = []
    for L, k in ((256, 10), (512, 5), (1024, 8)):
        rows += list(np.flatnonzero(d["L"] == L)[:k])
    _check_big(rb, d, rows)


@pytest.mark.slow
def test_critical_masks_L1024_all(rb):
    """All 1000 L = 1024 masks of the labelling KAT."""
    d = golden("label_kat_big.npz")
    _check_big(rb, d, np.flatnonzero(d["L"] == 1024))


def test_handles_many_lattices_in_one_call(rb, orc):
    L = 24
    rng = np.random.default_rng(3)
    masks = rng.random((300, 2 * L * L)) < 0.5
    ncl, labels, wraps = rb.label_and_wrap_many(masks, L)
    for k in range(0, 300, 37):
        n, lab, wx, wy = orc.label_and_wrap(masks[k], L)
        assert ncl[k] == n and np.array_equal(labels[k], lab) and tuple(wraps[k]) == (wx, wy)


def test_spanning_differs_from_wrapping(rb):
    """Reference ``tests/test_clusters.py:94-111`` on the GPU labeller."""
    L = 6
    lattice = rb.build_lattice(L)
    active = np.zeros(lattice.n_bonds, dtype=bool)
    for y in range(L - 1):
        active[2 * y + 1] = True
    assert rb.spans_along(active, lattice, "y")
    assert not rb.wraps_along(active, lattice, "y")
    active[2 * (L - 1) + 1] = True
    assert rb.wraps_along(active, lattice, "y")
