"""``rbim_sweeps_plain_noalloc``: plain sweeps on the library's static device scratch.

The entry point must give exactly what ``rbim_sweeps_plain`` gives with a
caller workspace -- spins, bin sums (the doubles bit for bit), records,
sweep counters and status -- over two calls in a row, for lattices of
different sizes sharing the one scratch (a large L before a small one, so
stale scratch from the large lattice is present), and reject L above its
limit with a message naming the limit.  The comparison does not depend on
what ran before: the first lattice (L = 512) fills the scratch and the
smaller ones that follow meet its stale contents, whether the file runs
alone in a fresh process or after the rest of the suite.
"""

import ctypes

import numpy as np
import pytest

SIZES = (512, 37, 3, 256, 100)


def _twin_sets(rb):
    """Two identical chain sets (hot start) over SIZES, with records."""
    specs, couplings = [], []
    for r, L in enumerate(SIZES):
        rng = np.random.default_rng(1000 + L)
        J = np.where(rng.random(2 * L * L) < 0.1, -1, 1).astype(np.int8)
        couplings.append(rb.packing.pack_couplings(J, L))
        T = (1.6, 2.27, 3.0)[r % 3]
        specs.append(rb.ChainSpec(L=L, realization=r, key=0x1234 + 7 * L, beta=1.0 / T, n_therm=2, n_bins=3,
                                  sweeps_per_bin=3, records=True))
    sets = []
    for _ in range(2):
        cs = rb.ChainSet(specs, couplings)
        cs.init_spins(hot=True)
        sets.append(cs)
    return sets


@pytest.mark.gpu
def test_noalloc_matches_workspace_entry_on_two_calls(rb):
    import torch

    ref, got = _twin_sets(rb)
    for n in (4, 7):  # two calls in a row; the second crosses into the measured bins
        ref.run_plain(n)
        got.run_plain_noalloc(n)
        torch.cuda.synchronize()
        assert int(got.status.item()) == 0
        assert int(ref.status.item()) == 0
        assert torch.equal(ref.spin_pool, got.spin_pool)
        assert torch.equal(ref.acc_int, got.acc_int)
        assert torch.equal(ref.acc_f64.view(torch.int64), got.acc_f64.view(torch.int64))
        assert torch.equal(ref.records, got.records)
        assert np.array_equal(ref.device_sweeps(), got.device_sweeps())
    # The chains really moved: every one ran 11 sweeps and has measured sums.
    assert np.all(got.device_sweeps() == 11)
    assert int(got.acc_int[:, 5].min().item()) > 0


def test_noalloc_limits(rb):
    """Size checks run on the host before any CUDA call."""
    lib = rb._native.lib()
    assert lib.rbim_noalloc_max_l() == 512
    dummy = ctypes.c_void_p(256)
    for L, code in ((513, -3), (4096, -3), (2, -1)):
        rc = lib.rbim_sweeps_plain_noalloc(L, dummy, dummy, dummy, dummy, dummy, None, 1, dummy, None)
        assert rc == code, L
        msg = lib.rbim_last_error().decode()
        if code == -3:
            assert "512" in msg and "rbim_sweeps_plain" in msg
    assert lib.rbim_sweeps_plain_noalloc(64, None, None, None, None, None, None, 1, None, None) == -1
    assert lib.rbim_sweeps_plain_noalloc(64, None, None, None, None, None, None, 0, None, None) == 0
