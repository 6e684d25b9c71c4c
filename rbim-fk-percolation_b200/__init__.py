"""B200-native Swendsen-Wang engine for the 2D +-J random-bond Ising model.

Drop-in for the Python API of Amirhossein-Manouchehri/rbim-fk-percolation
(``rbim``): the same ``run_temperature_scan`` / ``run_single_realization``
signatures and return values, the same disorder and result ``.npz`` formats,
the same observables with jackknife ``error`` and ``thermal_error``.  The
sweep itself (bond activation, FK labelling with exact wrapping, cluster
flip, measurement) runs in hand-written sm_100a CUDA kernels behind the C ABI
of ``include/rbim_sm100.h`` (``librbim_sm100.so``); there is no CPU fallback.

The directory name is not a Python identifier, so load the package with
``importlib.import_module("rbim-fk-percolation_b200")``; it also registers
itself as ``rbim_b200`` in ``sys.modules``.
"""

import sys as _sys

from . import _native, autotune, seeding
from ._native import RbimError
from .clusters import (
    activate_bonds,
    bond_activation_probability,
    cluster_statistics,
    label_and_wrap,
    label_and_wrap_many,
    label_clusters,
    spans_along,
    wraps_along,
)
from .disorder import (
    default_disorder_filename,
    frustrated_plaquettes,
    frustration_density,
    generate_disorder,
    generate_disorders,
    load_disorder,
    save_disorder,
)
from .engine import ChainSet, ChainSpec, chain_key
from .lattice import Lattice, build_lattice, couplings_from_disorder, site_index
from .simulation import (
    OBSERVABLES,
    PRIMITIVES,
    RealizationResult,
    ScanPlan,
    assemble_scan,
    combine_realizations,
    derive_observables,
    load_results,
    realization_from_sums,
    plan_temperature_scan,
    run_scan_tasks,
    run_single_realization,
    run_temperature_scan,
    save_results,
)
from .serving import RangeAllocator, ScanRequest, ScanServer, request_footprint
from .sharding import gather_task_sums, run_temperature_scan_sharded, shard_bounds
from .timeseries import collect_series, integrated_autocorrelation
from .swendsen_wang import SweepResult, aligned_spins, energy, initial_spins, magnetization, random_spins, sw_sweep

__version__ = "0.1.0"

__all__ = [
    "RbimError",
    "Lattice",
    "build_lattice",
    "site_index",
    "couplings_from_disorder",
    "generate_disorder",
    "generate_disorders",
    "load_disorder",
    "save_disorder",
    "frustrated_plaquettes",
    "frustration_density",
    "default_disorder_filename",
    "bond_activation_probability",
    "activate_bonds",
    "label_clusters",
    "label_and_wrap",
    "label_and_wrap_many",
    "cluster_statistics",
    "wraps_along",
    "spans_along",
    "SweepResult",
    "sw_sweep",
    "energy",
    "magnetization",
    "random_spins",
    "aligned_spins",
    "initial_spins",
    "RealizationResult",
    "PRIMITIVES",
    "OBSERVABLES",
    "derive_observables",
    "realization_from_sums",
    "combine_realizations",
    "run_single_realization",
    "run_temperature_scan",
    "ScanPlan",
    "plan_temperature_scan",
    "run_scan_tasks",
    "assemble_scan",
    "shard_bounds",
    "gather_task_sums",
    "run_temperature_scan_sharded",
    "ScanRequest",
    "ScanServer",
    "RangeAllocator",
    "request_footprint",
    "collect_series",
    "integrated_autocorrelation",
    "save_results",
    "load_results",
    "ChainSet",
    "ChainSpec",
    "chain_key",
]

_sys.modules.setdefault("rbim_b200", _sys.modules[__name__])
