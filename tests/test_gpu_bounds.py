"""Device loop bounds and descriptor checks report through the status word, and every call returns.

Every loop of the sweep kernels has an iteration bound; hitting one sets a bit
of the device status word, which the host turns into ``RbimError``.  Nothing
waits on anything: a bound that fires ends its loop and the kernel carries on
to its end.  Two host-side ways make the bounds fire without any fault:

* a chain descriptor's ``walk_cap`` (a test hook of ``rbim_chain_t``) lowers
  the bound on one union-find walk to a few steps, so that a small lattice at
  low temperature (one large cluster, long walks) exceeds it;
* a malformed descriptor (``sweeps_per_bin = 0``, or an ``L`` the call was not
  made for) is rejected by the kernels with ``RBIM_STATUS_BAD_CHAIN`` and left
  unchanged, while the other chains of the same call still run correctly.

After each case the device is used again and checked against the oracle.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIND_CAP, UNION_CAP, BAD_CHAIN = 1, 2, 4


def _set(rb, Ls, beta=2.0, p=0.0, hot=False, n_bins=1, spb=4):
    specs, couplings, J_host = [], [], []
    for i, L in enumerate(Ls):
        rng = np.random.default_rng(50 + i)
        J = np.where(rng.random(2 * L * L) < p, -1, 1).astype(np.int8)
        specs.append(rb.ChainSpec(L=L, realization=i, key=0xB0B + 17 * i, beta=beta, n_therm=1, n_bins=n_bins,
                                  sweeps_per_bin=spb))
        couplings.append(rb.packing.pack_couplings(J, L))
        J_host.append(J)
    cs = rb.ChainSet(specs, couplings)
    cs.init_spins(hot=hot)
    return cs, specs, J_host


def _run(cs, engine, n):
    if engine == "plain":
        cs.run_plain(n)
    else:
        cs.run_batched(n)


def _status(cs):
    import torch

    torch.cuda.synchronize()
    return int(cs.status.item())


def _device_still_exact(rb, orc):
    """A fresh chain set on the same device matches the oracle bit for bit."""
    cs, specs, J_host = _set(rb, [24, 24], beta=1 / 2.2, p=0.1, hot=True, n_bins=2, spb=3)
    cs.run_batched(7)
    cs.check_status()
    for i, s in enumerate(specs):
        ib, fb, spins = orc.run_chain(s.L, J_host[i], s.key, rb.packing.threshold(s.beta), hot=True, n_therm=1,
                                      n_bins=2, sweeps_per_bin=3)
        gi, gf = cs.bins(i)
        assert np.array_equal(gi, ib) and np.array_equal(gf.view(np.uint64), fb.view(np.uint64))
        assert np.array_equal(cs.spins(i), spins.astype(np.int64))


@pytest.mark.parametrize("engine,L", [("batched", 64), ("batched", 200), ("plain", 64), ("plain", 300)])
def test_walk_bound_fires_and_call_returns(rb, orc, engine, L):
    # A cold ferromagnet at T = 0.5: one cluster covers the lattice, so walks run long.
    cs, _, _ = _set(rb, [L])
    cs.set_descriptor_field(0, "walk_cap", 1)
    _run(cs, engine, 5)
    st = _status(cs)
    assert st & (FIND_CAP | UNION_CAP), st
    assert not st & BAD_CHAIN
    with pytest.raises(rb.RbimError, match="status word"):
        cs.check_status()
    # The run itself completed: the sweep counter reached the end.
    assert cs.device_sweeps()[0] == 5
    _device_still_exact(rb, orc)


def test_default_bound_does_not_fire(rb):
    """The same lattices with walk_cap = 0 (the default bounds) report nothing."""
    for engine, L in (("batched", 64), ("plain", 64), ("batched", 300)):
        cs, _, _ = _set(rb, [L])
        _run(cs, engine, 5)
        assert _status(cs) == 0, (engine, L)


@pytest.mark.parametrize("engine,Ls", [("batched", [16, 16, 16]), ("batched", [300, 300, 300]),
                                       ("plain", [16, 16, 16])])
def test_bad_descriptor_is_rejected_and_others_run(rb, orc, engine, Ls):
    cs, specs, J_host = _set(rb, Ls, beta=1 / 2.0, p=0.1, hot=True, n_bins=2, spb=2)
    cs.set_descriptor_field(1, "sweeps_per_bin", 0)
    _run(cs, engine, 5)
    st = _status(cs)
    assert st == BAD_CHAIN, st
    with pytest.raises(rb.RbimError, match="status word"):
        cs.check_status()
    sweeps = cs.device_sweeps()
    assert sweeps[1] == 0  # the rejected chain is left unchanged
    gi, gf = cs.bins(1)
    assert not gi.any() and not gf.any()
    for i in (0, 2):
        assert sweeps[i] == 5
        s = specs[i]
        ib, fb, spins = orc.run_chain(s.L, J_host[i], s.key, rb.packing.threshold(s.beta), hot=True, n_therm=1,
                                      n_bins=2, sweeps_per_bin=2)
        gi, gf = cs.bins(i)
        assert np.array_equal(gi, ib) and np.array_equal(gf.view(np.uint64), fb.view(np.uint64)), (engine, i)
        assert np.array_equal(cs.spins(i), spins.astype(np.int64)), (engine, i)
    _device_still_exact(rb, orc)


@pytest.mark.parametrize("engine", ["batched", "plain"])
def test_descriptor_size_mismatch_is_rejected(rb, orc, engine):
    """A descriptor whose L exceeds what the call was made for (the resident launch's l_max, or the plain call's L
    and workspace) is rejected before any site is touched."""
    cs, _, _ = _set(rb, [16, 16], beta=1 / 2.0, p=0.1, hot=True)
    before = cs.spin_pool.clone()
    cs.set_descriptor_field(0, "L", 17 if engine == "plain" else 300)
    _run(cs, engine, 3)
    assert _status(cs) == BAD_CHAIN
    assert cs.device_sweeps()[0] == 0
    w = rb.packing.words_for(16)
    assert bool((cs.spin_pool[:w] == before[:w]).all())
    _device_still_exact(rb, orc)
