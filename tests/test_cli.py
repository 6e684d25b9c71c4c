"""The command-line front end: argument surface of the reference's scripts, host-only subcommands, GPU runs."""

import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "rbim-fk-percolation_b200", "cli.py")


def _cli():
    import importlib.util

    spec = importlib.util.spec_from_file_location("rbim_cli", CLI)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_run_sweep_options_match_the_reference_script():
    ap = _cli().build_parser()
    args = ap.parse_args(["run-sweep", "--L", "32", "--p", "0.05", "--t-min", "1.0", "--t-max", "3.0", "--n-temps",
                          "40", "--realizations", "32", "--sweeps", "20000", "--out", "x.npz", "--backend", "cuda",
                          "--no-percolation", "--start", "cold", "--workers", "4", "--therm", "7", "--bins", "20"])
    assert (args.L, args.p, args.n_temps, args.realizations, args.sweeps, args.therm, args.bins) == (
        32, 0.05, 40, 32, 20000, 7, 20)
    assert args.no_percolation and args.start == "cold" and args.backend == "cuda"
    with pytest.raises(SystemExit):
        ap.parse_args(["run-sweep", "--L", "8", "--p", "0.1", "--out", "x.npz", "--backend", "numba"])


def test_crossing_interpolation():
    cli = _cli()
    T = np.array([1.0, 2.0, 3.0])
    assert cli.crossing(T, np.array([0.0, 1.0, 2.0]), np.array([0.5, 0.5, 0.5])) == pytest.approx(1.5)
    assert cli.crossing(T, np.array([1.0, 2.0, 3.0]), np.array([0.0, 0.0, 0.0])) is None
    found = cli.pairwise_crossings(T, {8: np.array([0.0, 1.0, 2.0]), 16: np.array([0.5, 0.5, 0.5])})
    assert found == [(8, 16, pytest.approx(1.5))]


def test_generate_disorder_writes_the_reference_files(rb, tmp_path):
    out = tmp_path / "dis"
    r = subprocess.run([sys.executable, CLI, "generate-disorder", "--L", "8", "--p", "0.1", "--realizations", "3",
                        "--out", str(out), "--seed", "5"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    files = sorted(os.listdir(out))
    assert files == [rb.default_disorder_filename(8, 0.1, i) for i in range(3)]
    # Same realizations as SeedSequence(5).spawn(3) through generate_disorder.
    for i, child in enumerate(np.random.SeedSequence(5).spawn(3)):
        J_h, J_v = rb.generate_disorder(8, 0.1, np.random.default_rng(child))
        h, v = rb.load_disorder(str(out / files[i]))
        assert np.array_equal(h, J_h) and np.array_equal(v, J_v)


def test_integrated_autocorrelation_known_cases(rb):
    assert rb.integrated_autocorrelation(np.ones(100)) == (0.5, 0)
    rng = np.random.default_rng(1)
    tau, _ = rb.integrated_autocorrelation(rng.standard_normal(20000))
    assert abs(tau - 0.5) < 0.1
    # AR(1) with coefficient a: tau_int = (1 + a) / (2 (1 - a)).
    a, n = 0.8, 200000
    x = np.empty(n)
    x[0] = 0.0
    e = rng.standard_normal(n)
    for i in range(1, n):
        x[i] = a * x[i - 1] + e[i]
    tau, _ = rb.integrated_autocorrelation(x)
    assert tau == pytest.approx((1 + a) / (2 * (1 - a)), rel=0.1)


@pytest.mark.gpu
def test_run_sweep_writes_what_the_scan_returns(rb, tmp_path):
    out = tmp_path / "scan.npz"
    r = subprocess.run([sys.executable, CLI, "run-sweep", "--L", "12", "--p", "0.1", "--n-temps", "4",
                        "--realizations", "3", "--sweeps", "200", "--bins", "4", "--seed", "3", "--out", str(out)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    got = rb.load_results(str(out))
    want = rb.run_temperature_scan(12, 0.1, np.linspace(1.0, 3.0, 4), n_realizations=3, n_sweeps=200, n_bins=4,
                                   seed=3)
    for name, entry in want["observables"].items():
        for field, v in entry.items():
            np.testing.assert_array_equal(got["observables"][name][field], v)


@pytest.mark.gpu
def test_time_series_match_oracle_records(rb, orc):
    L, temps, n_sweeps, n_therm, n_r = 10, [1.5, 2.5], 30, 5, 2
    series = rb.collect_series(L, 0.1, temps, n_sweeps=n_sweeps, n_therm=n_therm, n_realizations=n_r, seed=4)
    plan = rb.plan_temperature_scan(L, 0.1, temps, n_realizations=n_r, n_sweeps=n_sweeps, n_therm=n_therm, n_bins=1,
                                    seed=4)
    for k in range(plan.n_tasks):
        t, r = divmod(k, n_r)
        J = plan.couplings[r]
        spins = orc.initial_spins(L * L, int(plan.keys[k]), hot=True)
        thr = rb.packing.threshold(1.0 / temps[t])
        for s in range(n_therm + n_sweeps):
            rec = orc.sw_sweep(L, spins, J, int(plan.keys[k]), thr, s, measure=s >= n_therm)
            if s >= n_therm:
                i = s - n_therm
                assert series["energy"][t, r, i] == rec[0]
                assert series["largest_size"][t, r, i] == rec[3]
                assert series["largest_abs_mag"][t, r, i] == rec[4]
                assert series["second_size"][t, r, i] == rec[5]
                assert series["second_abs_mag"][t, r, i] == rec[6]
                assert series["wrap_y"][t, r, i] == rec[8]
                assert series["mag_ratio"][t, r, i] == pytest.approx(rec[4] / rec[3])


@pytest.mark.gpu
def test_validate_pure_ising_finds_tc(rb):
    import argparse

    cli = _cli()
    args = argparse.Namespace(sizes=[16, 32], t_min=2.1, t_max=2.45, n_temps=8, sweeps=3000, bins=10, seed=0,
                              workers=None, chunk=500)
    b, w = cli.validate_pure_ising(args)
    tc = 2.0 / np.log(1.0 + np.sqrt(2.0))
    assert b is not None and abs(b - tc) < 0.08
    assert w is not None and abs(w - tc) < 0.08


@pytest.mark.gpu
def test_pure_ising_crossings_drift_to_tc(rb):
    """The reference's validation (``scripts/validate_pure_ising.py``, ``README.md:146-158``) on the GPU.

    * At the reference's own settings (L = 8, 16, 24; 11 temperatures in [2.15, 2.40]; 8,000 sweeps of one
      chain per temperature) every Binder and wrap_y crossing lies within 0.025 of the exact T_c: the
      reference's README table spans 2.2491 ... 2.2683, and one 8,000-sweep chain per point puts about 0.01
      of noise on a crossing.
    * With 100,000 sweeps the Binder crossings of L-doubling pairs rise toward T_c as L grows (8/16 < 16/32 <
      32/64 < T_c, as the README's 2.2491 -> 2.2627 do), the largest pair lands within 0.006 of T_c, every
      wrap_y crossing within 0.004, and the two estimates of the largest pair agree (Coniglio-Klein at p = 0).
      The chains are seeded, so the numbers are the same on every run.
    """
    cli = _cli()
    temps = np.linspace(2.15, 2.40, 11)
    tc = 2.0 / np.log(1.0 + np.sqrt(2.0))
    table = {}
    for sizes, sweeps in (((8, 16, 24), 8000), ((8, 16, 32, 64), 100000)):
        b, w = cli.pure_ising_curves(sizes, temps, sweeps, 10, 0, chunk=5000)
        table[sizes] = ({(la, lb): t for la, lb, t in cli.pairwise_crossings(temps, b)},
                        {(la, lb): t for la, lb, t in cli.pairwise_crossings(temps, w)})
        print(f"crossings {sizes} {sweeps} sweeps: binder {table[sizes][0]} wrap {table[sizes][1]}")
    bs, ws = table[(8, 16, 24)]
    assert set(bs) == set(ws) == {(8, 16), (8, 24), (16, 24)}
    assert all(abs(t - tc) < 0.025 for t in list(bs.values()) + list(ws.values())), (bs, ws)
    bl, wl = table[(8, 16, 32, 64)]
    assert bl[(8, 16)] < bl[(16, 32)] < bl[(32, 64)] < tc, bl
    assert abs(bl[(32, 64)] - tc) < 0.006, bl
    assert all(abs(t - tc) < 0.004 for t in wl.values()), wl
    assert abs(bl[(32, 64)] - wl[(32, 64)]) < 0.005
