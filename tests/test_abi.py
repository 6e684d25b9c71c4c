"""The C ABI library loads and exports every symbol of ``include/rbim_sm100.h`` (no GPU needed).

Only calls that do no device work are made here: size queries, the resident
limit, and argument checks that must fail before touching CUDA.
"""

import ctypes
import os
import re

import numpy as np

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "rbim_sm100.h")


def _declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rbim_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree(rb):
    assert _declared_functions() == sorted(rb._native.EXPORTED_SYMBOLS)


def test_library_exports_every_declared_symbol(rb):
    lib = rb._native.lib()
    for name in _declared_functions():
        assert hasattr(lib, name), name


def test_chain_struct_layout_matches_header(rb):
    text = open(HEADER).read()
    body = re.search(r"typedef struct rbim_chain_t \{(.*?)\} rbim_chain_t;", text, re.S).group(1)
    fields = re.findall(r"(u?int64_t)\s+([A-Za-z_]+);", body)
    assert [f for _, f in fields] == list(rb._native.CHAIN_DTYPE.names)
    for (ctype, name) in fields:
        kind = rb._native.CHAIN_DTYPE[name]
        assert kind.itemsize == 8 and (kind.kind == "u") == ctype.startswith("u"), name


def test_host_only_queries(rb):
    lib = rb._native.lib()
    assert lib.rbim_abi_version() == 2
    assert lib.rbim_plane_words(3) == 4 and lib.rbim_plane_words(64) == 128
    lmax = lib.rbim_resident_max_l()
    assert 128 <= lmax <= 256
    assert lib.rbim_label_wrap_workspace_bytes(lmax) == 0
    assert lib.rbim_label_wrap_workspace_bytes(lmax + 1) == lib.rbim_plain_workspace_bytes(lmax + 1) > 0
    assert lib.rbim_plain_workspace_bytes(1024) >= 8 * 1024 * 1024
    assert lib.rbim_activate_workspace_bytes(2) == 0
    assert lib.rbim_batched_workspace_bytes() >= 4
    # Default CTA size of the resident engine: a supported size, never
    # shrinking as L grows, 0 outside the engine's range.
    sizes = [lib.rbim_resident_threads(L) for L in range(3, lmax + 1)]
    assert set(sizes) <= {32, 64, 128, 256, 512, 1024}
    assert sizes == sorted(sizes)
    assert lib.rbim_resident_threads(2) == 0 and lib.rbim_resident_threads(lmax + 1) == 0
    # Cluster plans: CTA size 512 (half-size tiles) or 1024 wherever a cluster size exists.
    for L in range(lmax + 1, 1025):
        c, t = lib.rbim_cluster_size(L), lib.rbim_cluster_threads(L)
        assert (c == 0) == (t == 0) and t in (0, 512, 1024), L
    assert lib.rbim_cluster_threads(lmax) == 0
    assert {lib.rbim_cluster_threads(L) for L in (300, 420)} == {512, 1024}
    assert lib.rbim_cluster_size(300) == lib.rbim_cluster_size(420)


def test_argument_errors_are_reported_without_device_work(rb):
    lib = rb._native.lib()
    p = ctypes.c_void_p
    rc = lib.rbim_sweeps_batched(None, 4, 32, None, None, None, None, None, 10, 0, None, None, 0, None)
    assert rc == -1 and b"null pointer" in lib.rbim_last_error()
    dummy = p(16)
    rc = lib.rbim_sweeps_batched(dummy, 4, 100000, dummy, dummy, dummy, dummy, None, 10, 0, dummy, dummy, 256, None)
    assert rc == -3
    rc = lib.rbim_sweeps_batched(dummy, 4, 32, dummy, dummy, dummy, dummy, None, 10, 384, dummy, dummy, 256, None)
    assert rc == -1 and b"threads" in lib.rbim_last_error()
    rc = lib.rbim_sweeps_batched(dummy, 4, 2, dummy, dummy, dummy, dummy, None, 10, 0, dummy, dummy, 256, None)
    assert rc == -1 and b"at least 3" in lib.rbim_last_error()
    rc = lib.rbim_sweeps_plain(64, dummy, dummy, dummy, dummy, dummy, None, 5, dummy, dummy, 10, None)
    assert rc == -1 and b"workspace too small" in lib.rbim_last_error()
    rc = lib.rbim_label_wrap(8, -1, dummy, dummy, dummy, dummy, dummy, None, 0, None)
    assert rc == -1
    rc = lib.rbim_activate(8, dummy, dummy, 1, 2**32 + 1, 0, dummy, dummy, 1 << 20, None)
    assert rc == -1 and b"thr" in lib.rbim_last_error()
    # Grid engine: sizes, plans and workspace are checked on the host.
    rc = lib.rbim_sweeps_grid(32, dummy, dummy, dummy, dummy, dummy, None, 5, dummy, 0, 0, 0, dummy, 1 << 30, None)
    assert rc == -3 and b"33..65535" in lib.rbim_last_error()
    rc = lib.rbim_sweeps_grid(64, None, None, None, None, None, None, 5, None, 0, 0, 0, None, 0, None)
    assert rc == -1 and b"null pointer" in lib.rbim_last_error()
    rc = lib.rbim_sweeps_grid(64, dummy, dummy, dummy, dummy, dummy, None, 5, dummy, 1000, 1024, 0, dummy, 1 << 30, None)
    assert rc == -1 and b"cannot run" in lib.rbim_last_error()
    rc = lib.rbim_sweeps_grid(1024, dummy, dummy, dummy, dummy, dummy, None, 5, dummy, 128, 1024, 0, dummy, 4096, None)
    assert rc == -1 and b"workspace too small" in lib.rbim_last_error()
    assert lib.rbim_grid_workspace_bytes(1024, 128) >= 8 * 1024 * 1024
    assert lib.rbim_grid_workspace_bytes(32, 4) == 0
    # Zero-work calls succeed without touching the device.
    assert lib.rbim_sweeps_grid(64, None, None, None, None, None, None, 0, None, 0, 0, 0, None, 0, None) == 0
    assert lib.rbim_sweeps_batched(None, 0, 32, None, None, None, None, None, 10, 0, None, None, 0, None) == 0
    assert lib.rbim_label_wrap(8, 0, None, None, None, None, None, None, 0, None) == 0


def test_grid_workspace_covers_its_arrays(rb):
    """Grid workspace: one 64-bit node word per site, C x L tile-root ids and a
    flip bit per site at least, 256-byte granular, growing with L; 0 outside
    the engine's range."""
    lib = rb._native.lib()
    prev = 0
    for L in (33, 64, 100, 257, 1024, 2048, 3100):
        for C in (2, 64, 148):
            b = lib.rbim_grid_workspace_bytes(L, C)
            assert b % 256 == 0 and b >= 8 * L * L + 4 * C * L + L * L // 8, (L, C)
        cur = lib.rbim_grid_workspace_bytes(L, 148)
        assert cur > prev, L
        prev = cur
    assert lib.rbim_grid_workspace_bytes(70000, 4) == 0
    assert lib.rbim_grid_workspace_bytes(64, -1) == 0


def test_packing_matches_the_documented_layout(rb):
    # Site n is bit n & 31 of word n >> 5; a set spin bit means s = -1.
    L = 6
    spins = np.ones(L * L, dtype=np.int64)
    spins[[0, 5, 31, 32, 35]] = -1
    w = rb.packing.pack_spins(spins, L)
    assert w[0] == (1 << 0) | (1 << 5) | (1 << 31) and w[1] == (1 << 0) | (1 << 3)


def test_engine_buckets_split_modes(rb):
    """Launch buckets: resident lattices by default CTA size, cluster lattices by (CTAs per cluster, CTA size),
    the rest plain; resident buckets sort before cluster buckets, cluster before plain."""
    nat = rb._native
    r_max = nat.lib().rbim_resident_max_l()
    Ls = [16, 32, 48, 200, 300, 420, 2000]
    keys = nat.engine_buckets(Ls, r_max, 1024)
    assert keys[0] == keys[1] == (0, 32) and keys[2] == (0, 128) and keys[3][0] == 0
    assert keys[4][:2] == keys[5][:2] and keys[4] != keys[5]  # same cluster size, different CTA size
    assert keys[6] == (2, 0)
    assert max(k for k in keys if k[0] == 0) < min(k for k in keys if k[0] == 1) < (2, 0)
