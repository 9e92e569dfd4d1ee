"""CUDA engine against the C oracle, through the C ABI (B200 required).

Tolerances: tables and replayed trajectories are compared for exact equality (the FP64 build
computes every state-feeding operation in the same IEEE order as the oracle, and the shared
elementary functions of include/dms_math.h); the device-built rate grid, which uses CUDA's
erf/exp, is compared to 1e-13 relative; accumulated histograms to 1e-12 relative (atomic
summation order)."""
import math

import numpy as np
import pytest

from dms_ctypes import C_KMS, NUM_TARGETS, RSUN_KM, point_params as oracle_point_params, records_to_dicts
from engine_fixtures import REPLAY_POINT, dms_b200, outcome, state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    e = dms_b200.Engine(0)
    yield e
    e.close()


@pytest.fixture(scope="module")
def replay(engine, oracle):
    p = REPLAY_POINT
    oracle.set_point(oracle_point_params(p["mass_gev"], p["sigma_p_cm2"], interpolation_points=p["interpolation_points"]))
    pid = engine.add_point(dms_b200.point_params(p["mass_gev"], p["sigma_p_cm2"], interpolation_points=p["interpolation_points"]))
    device_grid = engine.rate_grid(pid, p["interpolation_points"])
    engine.set_rate_grid(pid, oracle.rate_grid())
    return pid, device_grid


def test_tables_bit_identical(engine, oracle):
    t = oracle.tables()
    for which, name in [(0, "r"), (1, "gm"), (2, "temperature_gev"), (3, "vesc2"), (4, "n_e")]:
        assert np.array_equal(engine.solar_table(which), t[name]), name
    assert np.array_equal(engine.solar_table(5).reshape(-1, NUM_TARGETS), t["n_targets"])


def test_device_rate_grid_matches_oracle(replay, oracle):
    _, device_grid = replay
    og = oracle.rate_grid()
    scale = np.maximum(np.abs(og), 1e-300)
    assert np.max(np.abs(device_grid - og) / scale) < 1e-13


def test_rate_queries(engine, replay, oracle):
    pid, _ = replay
    rng = np.random.default_rng(3)
    r = np.concatenate([rng.uniform(0, RSUN_KM, 300), [0.0, RSUN_KM, 1.5 * RSUN_KM]])
    v = np.concatenate([rng.uniform(0, 3000, 300), [100.0, 100.0, 100.0]])
    got = engine.rate(pid, r, v, interpolated=True)
    want = np.array([oracle.query(5, a, b) for a, b in zip(r, v)])
    assert np.array_equal(got, want)
    got_c = engine.rate(pid, r, v, interpolated=False)
    want_c = np.array([oracle.query(6, a, b) for a, b in zip(r, v)])
    assert np.max(np.abs(got_c - want_c) / np.maximum(np.abs(want_c), 1e-300)) < 1e-13


@pytest.mark.parametrize("capture_mode", [False, True])
def test_replay_matches_oracle(engine, replay, oracle, capture_mode):
    pid, _ = replay
    n = 400
    opts = dms_b200.run_opts(seed=7, capture_mode=capture_mode, max_scatterings=10 ** 6, time_limit_s=120.0)
    mine = engine.run_records(pid, 0, n, opts, histograms=not capture_mode)
    ref = oracle.run_records(7, pid, 0, n, capture_mode=capture_mode, max_scatterings=10 ** 6, histograms=not capture_mode)
    a, b = mine["records"], ref["records"]
    mism = [i for i in range(n) if outcome(a[i]) != outcome(b[i])]
    assert not mism, [(i, outcome(a[i]), outcome(b[i])) for i in mism[:5]]
    worst = 0.0
    for i in range(n):
        x, y = np.array(state(a[i])), np.array(state(b[i]))
        worst = max(worst, float(np.max(np.abs(x - y) / np.maximum(np.abs(y), 1e-300))))
        assert a[i].t_capture == b[i].t_capture or (math.isnan(a[i].t_capture) and math.isnan(b[i].t_capture))
        assert a[i].lifetime_unbinding == b[i].lifetime_unbinding
    assert worst <= 1e-10, worst
    if not capture_mode:
        assert np.max(np.abs(mine["hist_dt"] - ref["hist_dt"])) <= 1e-10 * max(np.max(ref["hist_dt"]), 1e-300)


def test_accumulated_results_match_records(engine, replay):
    pid, _ = replay
    n = 2000
    opts = dms_b200.run_opts(seed=11, capture_mode=False, max_scatterings=10 ** 6, time_limit_s=300.0)
    recs = engine.run_records(pid, 0, n, opts, histograms=True)
    engine.reset_results(pid)
    engine.run([(pid, 0, n)], opts)
    res = engine.results(pid)
    c = res["counters"]
    r = recs["records"]
    captured = [i for i in range(n) if r[i].flags & 0x2]
    escaped = [i for i in range(n) if not (r[i].flags & 0x2) and r[i].termination_reason == 1]
    assert c["trajectories"] == n
    assert c["captured"] == len(captured)
    assert c["completed_outward_escapes"] == len(escaped)
    assert c["total_scatterings"] == sum(r[i].number_of_scatterings for i in range(n))
    assert c["free"] == sum(1 for i in escaped if r[i].flags & 0x20)
    assert c["reflected"] == sum(1 for i in escaped if r[i].flags & 0x40)
    h = res["histograms"]
    for slot, idx in ((0, captured), (2, escaped)):
        want = recs["hist_dt"][idx].sum(axis=0)
        want_sq = (recs["hist_dt"][idx] ** 2).sum(axis=0)
        assert np.allclose(h[slot], want, rtol=1e-12, atol=0)
        assert np.allclose(h[slot + 4], want_sq, rtol=1e-12, atol=0)
    lifetimes = sorted(r[i].lifetime_unbinding for i in captured if r[i].lifetime_unbinding >= 0)
    assert sorted(res["events"]["lifetime_unbinding"].tolist()) == lifetimes


def test_errors_leave_context_usable(engine, replay):
    pid, _ = replay
    with pytest.raises(dms_b200.EngineError):
        engine.run([(pid + 1000, 0, 10)], dms_b200.run_opts())
    with pytest.raises(dms_b200.EngineError):
        engine.run([(pid, 0, 10)], dms_b200.run_opts(boundary_rsun=0.0))
    with pytest.raises(dms_b200.EngineError):
        engine.add_point(dms_b200.point_params(-1.0, 1e-36))
    # a wall-clock limit far below the run length cancels the launch; the context stays usable
    with pytest.raises(dms_b200.EngineError, match="cancelled"):
        engine.run([(pid, 0, 10 ** 7)], dms_b200.run_opts(seed=5, time_limit_s=0.05))
    out = engine.run_records(pid, 0, 4, dms_b200.run_opts(seed=7, time_limit_s=60.0))
    assert all(out["records"][i].termination_reason in range(11) for i in range(4))


def test_direct_rate_point_matches_oracle(engine, oracle):
    """interpolation_points = 0 builds no grid: every lookup sums the 64 channels on the fly
    (src/Solar_Model.cpp:397-405, 324-342).  The device uses CUDA's erf/exp and the oracle the C
    library's, so rates agree to 1e-13 relative, not bit for bit; replayed Capture-mode
    trajectories then agree in outcome and, where the outcome agrees, to 1e-8 relative."""
    pid = engine.add_point(dms_b200.point_params(0.3, 1e-36, interpolation_points=0))
    oracle.set_point(oracle_point_params(0.3, 1e-36, interpolation_points=0))
    with pytest.raises(dms_b200.EngineError):
        engine.rate_grid(pid, 2)
    rng = np.random.default_rng(5)
    r = rng.uniform(0, RSUN_KM, 200)
    v = rng.uniform(0, 3000, 200)
    got = engine.rate(pid, r, v, interpolated=True)
    want = np.array([oracle.query(5, a, b) for a, b in zip(r, v)])
    assert np.max(np.abs(got - want) / np.maximum(np.abs(want), 1e-300)) < 1e-13
    n = 64
    opts = dms_b200.run_opts(seed=7, capture_mode=True, max_scatterings=10 ** 5, time_limit_s=120.0)
    a = engine.run_records(pid, 0, n, opts)["records"]
    b = oracle.run_records(7, pid, 0, n, capture_mode=True, max_scatterings=10 ** 5)["records"]
    same = [i for i in range(n) if outcome(a[i]) == outcome(b[i])]
    assert len(same) >= 0.9 * n, [(i, outcome(a[i]), outcome(b[i])) for i in range(n) if i not in same][:5]
    for i in same:
        x, y = np.array(state(a[i])), np.array(state(b[i]))
        assert np.max(np.abs(x - y) / np.maximum(np.abs(y), 1e-300)) < 1e-8


def test_reflected_particles_recorded(engine):
    """Reflected particles carried to 1 AU are recorded with their speed (the reflection-spectrum
    sample, src/Data_Generation.cpp:824-846); their number equals the reflected count minus the
    failed final Kepler shifts, and the spectrum's rates follow from it."""
    pid = engine.add_point(dms_b200.point_params(0.3, 1e-36, interpolation_points=1000))
    n = 1 << 14
    engine.run([(pid, 0, n)], dms_b200.run_opts(seed=7, max_scatterings=10 ** 6, time_limit_s=300.0))
    res = engine.results(pid, events_capacity=1, reflections_capacity=1 << 16)
    c = res["counters"]
    refl = res["reflections"]
    assert len(refl) == c["reflected"] - c["final_reflection_shift_failures"] > 0
    assert np.all(refl["speed_kms"] > 0.0) and np.all(np.abs(refl["cos_sun_velocity"]) <= 1.0)
    assert len(set(refl["trajectory_id"].tolist())) == len(refl)
    s = engine.reflection_spectrum(pid, rings=1, ring=0, dm_density_gev_cm3=0.4)
    assert s["reflections"] == len(refl) and s["trajectories"] == n
    assert s["reflection_rate_per_s"] == pytest.approx(s["entering_rate_per_s"] * len(refl) / n, rel=1e-12)
    assert s["speed_max_kms"] == pytest.approx(1.05 * refl["speed_kms"].max(), rel=1e-12)
    # equal-area rings split the sample
    parts = [engine.reflection_spectrum(pid, rings=4, ring=k)["reflections"] for k in range(4)]
    assert sum(parts) == len(refl)
    u = np.linspace(0.0, s["speed_max_kms"], 2001)
    pdf = engine.reflection_pdf(pid, u)
    assert np.all(pdf >= 0.0) and abs(np.trapezoid(pdf, u) - 1.0) < 0.05
