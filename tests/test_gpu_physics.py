"""Statistical parity of whole scans with the reference, and exact p = 0 physics.

Full chains use Philox instead of numpy's PCG64, so scans are compared with
the reference's own scans (``tests/golden/scan_*.npz``, produced by
``run_temperature_scan`` of the reference at the same seeds, hence on the same
disorder realizations) in units of the combined jackknife error,
``z = (a - b) / sqrt(err_a^2 + err_b^2)``.

For an observable whose error is dominated by thermal noise (rare wrapping
events at high T, for instance) ``z`` is close to a standard normal even for
a correct engine, so over K comparisons a rule "every |z| <= 2" would fail
with probability 1 - 0.954^K (99% for K = 100).  The acceptance rule is
therefore: the number of |z| > 2 stays within the 99.9% quantile of
Binomial(K, 0.0455), no |z| exceeds 4, and the mean of z^2 stays below 2.
An observable exactly constant in both runs (zero error on both sides) must
agree to 1e-12.
"""

import numpy as np
import pytest
from scipy import stats as _stats

from conftest import golden
from oracle import onsager

pytestmark = pytest.mark.gpu


def _ref_scan(name):
    d = golden(name)
    params = {k[len("param__"):]: d[k][()] for k in d.files if k.startswith("param__")}
    obs = {}
    for k in d.files:
        if "__" in k and not k.startswith("param__"):
            o, f = k.split("__", 1)
            obs.setdefault(o, {})[f] = d[k]
    return d["temperatures"], obs, params


def _compare(ref_obs, got_obs, temps):
    """Failures of the acceptance rule in the module docstring (empty list = pass)."""
    z_all, over2, bad = [], [], []
    for name, ref in ref_obs.items():
        got = got_obs[name]
        for i in range(len(temps)):
            a, b = got["value"][i], ref["value"][i]
            sa, sb = got["error"][i], ref["error"][i]
            if not (np.isfinite(a) and np.isfinite(b)):
                if np.isfinite(a) != np.isfinite(b):
                    bad.append(("nonfinite", name, float(temps[i]), a, b))
                continue
            sigma = np.sqrt(sa**2 + sb**2)
            if sigma == 0:
                if abs(a - b) > 1e-12:
                    bad.append(("constant", name, float(temps[i]), float(a), float(b)))
                continue
            z = (a - b) / sigma
            z_all.append(z)
            if abs(z) > 2:
                over2.append((name, float(temps[i]), round(float(z), 2)))
            if abs(z) > 4:
                bad.append(("|z|>4", name, float(temps[i]), float(a), float(b), float(z)))
    k = len(z_all)
    allowed = int(_stats.binom.ppf(0.999, k, 0.0455)) if k else 0
    if len(over2) > allowed:
        bad.append(("too many |z|>2", len(over2), "allowed", allowed, "of", k, over2))
    if k and float(np.mean(np.square(z_all))) > 2.0:
        bad.append(("mean z^2", float(np.mean(np.square(z_all)))))
    return bad


def _run_like(rb, params, temps, **kw):
    return rb.run_temperature_scan(int(params["L"]), float(params["p"]), temps,
                                   n_realizations=int(params["n_realizations"]), n_sweeps=int(params["n_sweeps"]),
                                   n_therm=int(params["n_therm"]), n_bins=int(params["n_bins"]),
                                   seed=int(params["seed"]), **kw)


def test_scan_matches_reference_within_two_sigma(rb):
    temps, ref, params = _ref_scan("scan_small.npz")
    res = _run_like(rb, params, temps)
    assert list(res["observables"]) == list(rb.OBSERVABLES)
    bad = _compare(ref, res["observables"], temps)
    assert not bad, bad


def test_plain_engine_scan_matches_reference(rb):
    temps, ref, params = _ref_scan("scan_small.npz")
    params = dict(params, n_realizations=4)
    res = _run_like(rb, params, temps[:2], engine="plain")
    res_b = _run_like(rb, params, temps[:2], engine="batched")
    # Same Philox streams: the two engines give identical scans.
    for name in rb.OBSERVABLES:
        for key in ("value", "error", "thermal_error"):
            np.testing.assert_array_equal(res["observables"][name][key], res_b["observables"][name][key])


def test_pure_model_energy_is_exact_and_m_equals_p_infinity(rb):
    temps, ref, params = _ref_scan("scan_pure.npz")
    res = _run_like(rb, params, temps)
    obs = res["observables"]
    L = int(params["L"])
    for i, T in enumerate(temps):
        exact = onsager.energy_per_site_torus(float(T), L)
        e, err = obs["energy"]["value"][i], obs["energy"]["error"][i]
        assert abs(e - exact) <= 3 * err + 1e-4, (T, e, exact, err)
    bad = _compare(ref, obs, temps)
    assert not bad, bad
    # Coniglio-Klein at p = 0 (reference tests/test_physics.py:110-124).
    i = int(np.argmin(abs(temps - 2.0)))
    assert obs["p_infinity"]["value"][i] == pytest.approx(obs["abs_magnetization"]["value"][i], abs=0.05)
    assert obs["cluster_magnetization_ratio"]["value"][i] > 0.9


def test_binder_limits(rb):
    """Reference ``tests/test_physics.py:127-139``."""
    ordered = rb.run_temperature_scan(12, 0.0, [1.2], n_sweeps=3000, n_therm=600, n_bins=10, seed=4)
    disordered = rb.run_temperature_scan(12, 0.0, [5.0], n_sweeps=3000, n_therm=600, n_bins=10, seed=4)
    assert ordered["observables"]["binder"]["value"][0] == pytest.approx(2.0 / 3.0, abs=0.03)
    assert abs(disordered["observables"]["binder"]["value"][0]) < 0.1


def test_onsager_magnetization(rb):
    """Reference ``tests/test_physics.py:92-101`` on the GPU engine."""
    J = rb.couplings_from_disorder(np.ones((16, 16), np.int8), np.ones((16, 16), np.int8))
    r = rb.run_single_realization(16, J, 2.0, n_sweeps=4000, n_therm=1000, n_bins=10, seed=2024)
    d = rb.derive_observables(r.primitives, 2.0, 256)
    assert d["abs_magnetization"] == pytest.approx(onsager.onsager_magnetization(2.0), abs=0.04)
    assert -2.0 <= d["energy"] <= 0.0


@pytest.mark.slow
def test_c1_scan_matches_reference(rb):
    """L = 32, p = 0.05, 32 realizations x 40 temperatures, 20k + 2k sweeps."""
    temps, ref, params = _ref_scan("scan_c1.npz")
    res = _run_like(rb, params, temps)
    bad = _compare(ref, res["observables"], temps)
    assert not bad, bad


def test_large_lattice_critical_energy(rb):
    """The single-lattice configuration's second run: L = 1024, p = 0 at T_c, 2,000 measured sweeps.

    * E/N within the run's error of Kaufman's exact finite-torus value;
    * Coniglio-Klein, the reference's P_inf = |m| check (``tests/test_physics.py:110-124``): at T_c both scale
      as L^(-1/8) and the reference's own scans give P_inf / |m| = 0.998 at L = 32 and 0.997 at L = 64
      (20,000 and 8,000 sweeps), so they agree to within 0.02 at any L;
    * |m| L^(1/8) = 1.010 (L = 32) and 1.014 (L = 64) in those reference scans, so finite-size scaling puts
      |m| at L = 1024 near 1.012 * 1024^(-1/8) = 0.425.
    """
    L = 1024
    J = rb.couplings_from_disorder(np.ones((L, L), np.int8), np.ones((L, L), np.int8))
    r = rb.run_single_realization(L, J, onsager.TC_EXACT, n_sweeps=2000, n_therm=200, n_bins=20, seed=7,
                                  start="cold")
    e = r.primitives["energy"] / (L * L)
    bins = r.bin_primitives["energy"] / (L * L)
    err = bins.std(ddof=1) / np.sqrt(bins.size)
    exact = onsager.energy_per_site_torus(onsager.TC_EXACT, L)
    assert abs(e - exact) <= 4 * err + 1e-4, (e, exact, err)
    d = rb.derive_observables(r.primitives, onsager.TC_EXACT, L * L)
    assert d["p_infinity"] == pytest.approx(d["abs_magnetization"], abs=0.02), d
    assert d["abs_magnetization"] == pytest.approx(1.012 * L ** (-0.125), abs=0.03), d


def test_large_lattice_ordered_phase(rb):
    """L = 1024, p = 0 at T = 2.0 (reference ``tests/test_physics.py:92-124`` at the single-lattice size):
    |m| on Onsager's curve (no visible finite-size offset at this L), P_inf = |m|, and the percolating
    cluster's spins aligned."""
    L = 1024
    J = rb.couplings_from_disorder(np.ones((L, L), np.int8), np.ones((L, L), np.int8))
    r = rb.run_single_realization(L, J, 2.0, n_sweeps=1000, n_therm=200, n_bins=10, seed=2024, start="cold")
    d = rb.derive_observables(r.primitives, 2.0, L * L)
    assert d["abs_magnetization"] == pytest.approx(onsager.onsager_magnetization(2.0), abs=0.005), d
    assert d["p_infinity"] == pytest.approx(d["abs_magnetization"], abs=0.01), d
    assert d["cluster_magnetization_ratio"] > 0.9
