"""Ensemble comparison statistics (dms_stats) on synthetic accumulators (CPU)."""
import numpy as np

from engine_fixtures import dms_b200  # noqa: F401  (puts the package on sys.path)
import dms_stats


def fake_results(n, captured, per_traj, events, seed):
    rng = np.random.default_rng(seed)
    h = np.zeros((8, 2000))
    x = rng.exponential(per_traj, size=(captured, 200))
    h[0, :200] = x.sum(axis=0)
    h[4, :200] = (x ** 2).sum(axis=0)
    counters = {"trajectories": n, "captured": captured, "total_scatterings": 10 * n}
    ev = np.zeros(events, dtype=[("trajectory_id", np.uint64), ("lifetime_unbinding", np.float64)])
    return {"counters": counters, "histograms": h, "events": ev}


def test_identical_runs_agree_exactly():
    a = fake_results(10000, 500, 2.0, 50, seed=1)
    c = dms_stats.compare_runs(a, a)
    assert c["capture_fraction_sigmas"] == 0.0
    assert c["radial_chi2"] == 0.0 and c["radial_p_value"] == 1.0
    assert c["evaporation_rate_rel_error"] == 0.0


def test_independent_samples_pass_and_shift_fails():
    a = fake_results(10000, 500, 2.0, 50, seed=1)
    b = fake_results(10000, 500, 2.0, 50, seed=2)
    c = dms_stats.compare_runs(a, b)
    assert c["radial_dof"] == 200
    assert c["radial_p_value"] > 0.001
    shifted = fake_results(10000, 500, 2.6, 50, seed=2)
    assert dms_stats.compare_runs(a, shifted)["radial_p_value"] < 1e-6


def test_capture_fraction_sigmas():
    a = fake_results(10000, 500, 2.0, 50, seed=1)
    b = fake_results(10000, 560, 2.0, 50, seed=1)
    c = dms_stats.compare_runs(a, b)
    sigma = np.sqrt(0.05 * 0.95 / 10000 + 0.056 * 0.944 / 10000)
    assert abs(c["capture_fraction_sigmas"] - 0.006 / sigma) < 1e-9
    assert abs(c["capture_fraction_rel_error"] - 0.12) < 1e-12


def test_reference_gates_pass_for_same_distribution_and_fail_for_shift():
    a = fake_results(100000, 5000, 2.0, 2000, seed=1)
    rng = np.random.default_rng(5)
    a["events"]["lifetime_unbinding"] = rng.exponential(1e6, 2000)
    b = fake_results(100000, 5040, 2.0, 2010, seed=2)
    b["events"]["lifetime_unbinding"] = rng.exponential(1e6, 2010)
    g = dms_stats.reference_gates(a, b)
    assert all(ok for ok, _ in g.values()), g
    c = fake_results(100000, 8000, 2.0, 2000, seed=2)
    c["counters"]["total_scatterings"] = 13 * 100000
    g = dms_stats.reference_gates(a, c)
    assert not g["capture_95pct_intervals_overlap"][0]
    assert not g["average_scatterings_relative_difference"][0]


def test_wilson_interval_contains_rate():
    lo, hi = dms_stats.wilson_interval(50, 1000)
    assert lo < 0.05 < hi and abs((hi - lo) - 0.0276) < 2e-3
