"""Shared pytest configuration.

``-m "not gpu"`` runs the CPU suite (oracle against golden vectors, host
logic, the C ABI's exports); ``-m gpu`` runs the parity tests of the CUDA
engine, which call through the C ABI and compare with the oracle.
"""

from __future__ import annotations

import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA engine")
    config.addinivalue_line("markers", "slow: long-running statistical check")


def load_package():
    return importlib.import_module("rbim-fk-percolation_b200")


@pytest.fixture(scope="session")
def rb():
    """The engine package (``rbim-fk-percolation_b200``)."""
    return load_package()


@pytest.fixture(scope="session")
def orc():
    """The CPU oracle (test infrastructure)."""
    import oracle

    oracle.load()
    return oracle


def golden(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.skip(f"golden fixture {name} has not been generated")
    return np.load(path, allow_pickle=False)


class LabelKat:
    """Accessor of ``label_kat.npz``: masks with the reference union-find's answers."""

    def __init__(self):
        d = golden("label_kat.npz")
        self.d = {k: d[k] for k in d.files}
        self.n = self.d["L"].size

    def __len__(self):
        return self.n

    def case(self, i):
        d = self.d
        L = int(d["L"][i])
        m = d["masks"][d["mask_offsets"][i]: d["mask_offsets"][i + 1]]
        active = np.unpackbits(m, bitorder="little")[: 2 * L * L].astype(bool)
        labels = d["labels"][d["label_offsets"][i]: d["label_offsets"][i + 1]].astype(np.int64)
        return dict(L=L, active=active, labels=labels, n_clusters=int(d["n_clusters"][i]),
                    wraps=tuple(bool(v) for v in d["wraps"][i]), has_bf=bool(d["has_bf"][i]),
                    bf=tuple(bool(v) for v in d["bf_wraps"][i]))


@pytest.fixture(scope="session")
def label_kat():
    return LabelKat()


def big_mask(L, seed):
    """Mask of the large-lattice KAT (same generator as ``make_golden.big_mask``)."""
    return np.random.default_rng(seed).random(2 * L * L) < 0.5
