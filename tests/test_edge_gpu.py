"""Edge cases of the launch interface and the other benchmark points, through the C ABI
(B200 required).

* empty and ragged launches: no ranges is an error, zero-length ranges are no-ops, several
  points and odd range sizes in one launch, and the same ids split differently over ranges,
  give the counters of the per-trajectory records (results are keyed by trajectory id, not
  by launch layout);
* the scattering cap (`maximum_number_of_scatterings`): trajectories that reach it end with
  the reference's MaxScatterings reason, replayed bit for bit against the oracle;
* the Capture-mode point m = 1 GeV, sigma_n = 1e-35 cm^2 and the heavy-scattering point
  m = 0.1 GeV, sigma_n = 1e-33 cm^2, replayed against the oracle on the oracle's grid
  (identical outcomes and draw counts, states to 1e-10 relative)."""
import numpy as np
import pytest

from dms_ctypes import point_params as oracle_point_params
from engine_fixtures import dms_b200, outcome, state

pytestmark = pytest.mark.gpu

REASON_WALL_TIME_LIMIT = 3   # TrajectoryTerminationReason::WallTimeLimit, include/dms.h
REASON_MAX_SCATTERINGS = 5   # TrajectoryTerminationReason::MaxScatterings


@pytest.fixture(scope="module")
def engine():
    e = dms_b200.Engine(0)
    yield e
    e.close()


def _replay(engine, oracle, mass, sigma, capture_mode, n, max_scatterings, seed=3):
    oracle.set_point(oracle_point_params(mass, sigma, interpolation_points=300))
    pid = engine.add_point(dms_b200.point_params(mass, sigma, interpolation_points=300))
    engine.set_rate_grid(pid, oracle.rate_grid())
    opts = dms_b200.run_opts(seed=seed, capture_mode=capture_mode, max_scatterings=max_scatterings, time_limit_s=120.0)
    a = engine.run_records(pid, 0, n, opts)["records"]
    b = oracle.run_records(seed, pid, 0, n, capture_mode=capture_mode, max_scatterings=max_scatterings)["records"]
    mism = [i for i in range(n) if outcome(a[i]) != outcome(b[i])]
    assert not mism, [(i, outcome(a[i]), outcome(b[i])) for i in mism[:5]]
    for i in range(n):
        x, y = np.array(state(a[i])), np.array(state(b[i]))
        assert np.max(np.abs(x - y) / np.maximum(np.abs(y), 1e-300)) <= 1e-10
    return pid, a


def test_capture_mode_point_of_the_capture_benchmark(engine, oracle):
    _, a = _replay(engine, oracle, 1.0, 1e-35, True, 256, 10 ** 5)
    assert sum(1 for i in range(256) if a[i].flags & 0x2) > 64


def test_heavy_scattering_point(engine, oracle):
    _, a = _replay(engine, oracle, 0.1, 1e-33, True, 96, 10 ** 4)
    assert max(a[i].number_of_scatterings for i in range(96)) > 10


def test_scattering_cap_ends_trajectories_with_max_scatterings(engine, oracle):
    pid, a = _replay(engine, oracle, 0.3, 1e-36, False, 200, 3)
    capped = [i for i in range(200) if a[i].termination_reason == REASON_MAX_SCATTERINGS]
    assert capped and all(a[i].number_of_scatterings == 3 for i in capped)
    engine.reset_results(pid)
    engine.run([(pid, 0, 200)], dms_b200.run_opts(seed=3, max_scatterings=3, time_limit_s=120.0))
    c = engine.results(pid, events_capacity=1)["counters"]
    assert c["reasons"][REASON_MAX_SCATTERINGS] == len(capped)
    assert c["computational_truncations"] >= len(capped)


def test_empty_and_ragged_launches(engine):
    params = dms_b200.point_params(0.3, 1e-36, interpolation_points=300)
    p0, p1 = engine.add_point(params), engine.add_point(dms_b200.point_params(1.0, 1e-35, interpolation_points=300))
    opts = dms_b200.run_opts(seed=9, capture_mode=True, max_scatterings=10 ** 5, time_limit_s=300.0)
    for p in (p0, p1):
        engine.reset_results(p)
    with pytest.raises(dms_b200.EngineError, match="no work ranges"):
        engine.run([], opts)
    engine.run([(p0, 5, 0)], opts)                      # an empty range is a no-op
    assert engine.results(p0, events_capacity=1)["counters"]["trajectories"] == 0
    # odd sizes, two points, interleaved ranges, one launch
    layout = [(p0, 0, 1), (p1, 0, 33), (p0, 1, 1000), (p1, 33, 7), (p0, 1001, 0), (p0, 1001, 55)]
    engine.run(layout, opts)
    for p, n in ((p0, 1056), (p1, 40)):
        want = engine.run_records(p, 0, n, opts)["records"]
        c = engine.results(p, events_capacity=1)["counters"]
        assert c["trajectories"] == n
        assert c["total_scatterings"] == sum(want[i].number_of_scatterings for i in range(n))
        assert c["captured"] == sum(1 for i in range(n) if want[i].flags & 0x2)
        reasons = [0] * 11
        for i in range(n):
            reasons[want[i].termination_reason] += 1
        assert c["reasons"] == reasons


def test_results_do_not_depend_on_the_range_split(engine):
    pid = engine.add_point(dms_b200.point_params(0.3, 1e-36, interpolation_points=300))
    opts = dms_b200.run_opts(seed=13, max_scatterings=10 ** 5, time_limit_s=300.0)
    n = 1200
    out = []
    for layout in ([(pid, 0, n)], [(pid, 700, n - 700), (pid, 0, 700)], [(pid, k, 100) for k in range(0, n, 100)]):
        engine.reset_results(pid)
        engine.run(layout, opts)
        out.append(engine.results(pid, events_capacity=1 << 12))
    for r in out[1:]:
        assert r["counters"] == out[0]["counters"]
        assert np.allclose(r["histograms"], out[0]["histograms"], rtol=1e-12, atol=0)
        assert sorted(r["events"]["trajectory_id"].tolist()) == sorted(out[0]["events"]["trajectory_id"].tolist())


def test_trajectory_wall_time_limit(engine, oracle):
    """max_trajectory_wall_time_sec (src/Simulation_Trajectory.cpp:824-840, 873-874, 953-954): a
    trajectory whose wall time on its lane passes the limit ends with WallTimeLimit; every other
    trajectory is untouched and replays the oracle (which has no limit) exactly."""
    oracle.set_point(oracle_point_params(0.3, 1e-36, interpolation_points=300))
    pid = engine.add_point(dms_b200.point_params(0.3, 1e-36, interpolation_points=300))
    engine.set_rate_grid(pid, oracle.rate_grid())
    n = 4096
    opts = dms_b200.run_opts(seed=5, max_scatterings=10 ** 6, time_limit_s=120.0, max_trajectory_wall_time_s=0.002)
    a = engine.run_records(pid, 0, n, opts)["records"]
    b = oracle.run_records(5, pid, 0, n, max_scatterings=10 ** 6)["records"]
    limited = [i for i in range(n) if a[i].termination_reason == REASON_WALL_TIME_LIMIT]
    assert 0 < len(limited) < n
    for i in range(n):
        if i in limited:
            assert a[i].number_of_draws <= b[i].number_of_draws
            assert a[i].number_of_scatterings <= b[i].number_of_scatterings
        else:
            assert outcome(a[i]) == outcome(b[i]), i
    engine.reset_results(pid)
    engine.run([(pid, 0, n)], opts)
    c = engine.results(pid, events_capacity=1)["counters"]
    assert c["reasons"][REASON_WALL_TIME_LIMIT] > 0
    assert c["computational_truncations"] >= c["reasons"][REASON_WALL_TIME_LIMIT]
    with pytest.raises(dms_b200.EngineError, match="max_trajectory_wall_time_sec"):
        engine.run([(pid, 0, 4)], dms_b200.run_opts(max_trajectory_wall_time_s=-1.0))
