"""Launch-shape autotuner: size classes, the persisted cache, and (GPU) CTA-size invariance of the results."""

import json

import numpy as np
import pytest


def test_size_classes(rb):
    at = rb.autotune
    assert [at.size_class(L) for L in (3, 16, 17, 32, 33, 200, 256)] == [16, 16, 32, 32, 64, 256, 256]


def test_cache_round_trip(rb, tmp_path, monkeypatch):
    at = rb.autotune
    path = tmp_path / "tune.json"
    path.write_text(json.dumps({"GPU X|64": 512, "GPU X|128": 999}))
    monkeypatch.setenv("RBIM_TUNE_CACHE", str(path))
    monkeypatch.setattr(at, "_loaded", False)
    monkeypatch.setattr(at, "_cache", {})
    c = at.cache()
    assert c == {"GPU X|64": 512}  # values that are not CTA sizes are dropped
    at._cache["GPU X|256"] = 1024
    at._save()
    assert json.loads(path.read_text()) == {"GPU X|256": 1024, "GPU X|64": 512}


def test_disabled_by_default_returns_rule(rb, monkeypatch):
    at = rb.autotune
    monkeypatch.setattr(at, "_enabled", False)
    assert at.tuned_threads(64, None) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("L", [24, 64])
def test_results_do_not_depend_on_cta_size(rb, L):
    rng = np.random.default_rng(L)
    J = [rb.packing.pack_couplings(np.where(rng.random(2 * L * L) < 0.1, -1, 1).astype(np.int8), L) for _ in range(3)]
    specs = [rb.ChainSpec(L=L, realization=k % 3, key=11 * k + 1, beta=1.0 / (1.5 + 0.2 * k), n_therm=2, n_bins=2,
                          sweeps_per_bin=4, records=True) for k in range(6)]
    out = []
    for threads in rb.autotune.CANDIDATES:
        cs = rb.ChainSet(specs, J)
        cs.init_spins(hot=True)
        cs.run_batched(10, threads=threads)
        cs.check_status()
        ai, af = cs.all_bins()
        out.append((ai, af.view(np.int64), cs.spin_pool.cpu().numpy(), cs.records.cpu().numpy()))
    for o in out[1:]:
        for a, b in zip(out[0], o):
            assert np.array_equal(a, b)


@pytest.mark.gpu
def test_tune_picks_a_candidate_and_run_batched_uses_it(rb, monkeypatch, tmp_path):
    at = rb.autotune
    monkeypatch.setenv("RBIM_TUNE_CACHE", str(tmp_path / "t.json"))
    monkeypatch.setattr(at, "_loaded", False)
    monkeypatch.setattr(at, "_cache", {})
    best = at.tune(32, n_chains=64, sweeps=2)
    assert best in at.CANDIDATES
    assert any(k.endswith("|32") and v == best for k, v in at.cache().items())
    monkeypatch.setattr(at, "_enabled", True)
    kw = dict(L=20, p=0.1, temperatures=[1.5, 2.5], n_realizations=2, n_sweeps=40, n_bins=2, seed=3)
    tuned = rb.run_temperature_scan(**kw)
    monkeypatch.setattr(at, "_enabled", False)
    plain = rb.run_temperature_scan(**kw)
    for name, entry in plain["observables"].items():
        for field, v in entry.items():
            np.testing.assert_array_equal(tuned["observables"][name][field], v)


def test_cluster_plan_cache_entries(rb, tmp_path, monkeypatch):
    at = rb.autotune
    path = tmp_path / "tune.json"
    path.write_text(json.dumps({"GPU X|cluster|512": [4, 1024], "GPU X|cluster|300": [3, 333],
                                "GPU X|cluster|724": [1, 1024], "GPU X|64": 128}))
    monkeypatch.setenv("RBIM_TUNE_CACHE", str(path))
    monkeypatch.setattr(at, "_loaded", False)
    monkeypatch.setattr(at, "_cache", {})
    assert at.cache() == {"GPU X|cluster|512": [4, 1024], "GPU X|64": 128}
    monkeypatch.setattr(at, "_enabled", False)
    assert at.tuned_cluster_plan(512, [512], None) is None


def test_cluster_plans_host_query(rb):
    """The plan list is empty outside the cluster engine's range, and the CTA counts are cluster sizes."""
    lib = rb._native.lib()
    assert lib.rbim_cluster_plans(rb._native.resident_max_l(), None, None, 0) == 0
    assert lib.rbim_cluster_plans(70000, None, None, 0) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("L", [300, 512])
def test_results_do_not_depend_on_cluster_plan(rb, L):
    """Every plan rbim_cluster_plans lists gives the default plan's spins, bin sums and records bit for bit (tile
    boundaries fall elsewhere, the Philox numbers do not)."""
    plans = rb._native.cluster_plans(L)
    assert plans and plans[0] == (rb._native.lib().rbim_cluster_size(L), rb._native.lib().rbim_cluster_threads(L))
    rng = np.random.default_rng(L)
    J = [rb.packing.pack_couplings(np.where(rng.random(2 * L * L) < 0.1, -1, 1).astype(np.int8), L) for _ in range(2)]
    specs = [rb.ChainSpec(L=L, realization=k % 2, key=31 * k + 7, beta=1.0 / (1.6 + 0.3 * k), n_therm=1, n_bins=2,
                          sweeps_per_bin=2, records=True) for k in range(3)]
    out = []
    for plan in plans:
        cs = rb.ChainSet(specs, J)
        cs.init_spins(hot=True)
        cs._run_batched_fixed(5, 0, cluster_plan=plan)
        cs.check_status()
        ai, af = cs.all_bins()
        out.append((plan, ai, af.view(np.int64), cs.spin_pool.cpu().numpy(), cs.records.cpu().numpy()))
    for o in out[1:]:
        for a, b in zip(out[0][1:], o[1:]):
            assert np.array_equal(a, b), o[0]


@pytest.mark.gpu
def test_tune_cluster_picks_a_listed_plan(rb, monkeypatch, tmp_path):
    at = rb.autotune
    monkeypatch.setenv("RBIM_TUNE_CACHE", str(tmp_path / "t.json"))
    monkeypatch.setattr(at, "_loaded", False)
    monkeypatch.setattr(at, "_cache", {})
    L = 320
    best = at.tune_cluster(L, n_chains=12, sweeps=1)
    assert best in rb._native.cluster_plans(L)
    monkeypatch.setattr(at, "_enabled", True)
    kw = dict(L=L, p=0.08, temperatures=[1.6, 2.4], n_realizations=2, n_sweeps=6, n_therm=2, n_bins=2, seed=5)
    tuned = rb.run_temperature_scan(**kw, engine="batched")
    monkeypatch.setattr(at, "_enabled", False)
    default = rb.run_temperature_scan(**kw, engine="batched")
    for name, entry in default["observables"].items():
        for field, v in entry.items():
            np.testing.assert_array_equal(tuned["observables"][name][field], v)
