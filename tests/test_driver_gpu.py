"""The run driver (dms_generate_data, dms_write_outputs) against the contracts of the
reference's own Generate_Data tests (B200 required).

Each test restates one test of tests/test_Data_Generation.cpp with the same particle
(m = 0.01 GeV, sigma_p = sigma_e = 1e-100 pb, low-mass SI), the same Configure() arguments
(initial_and_final_radius, maximum scatterings, maximum free steps), sample size, trajectory
budget and seed, and checks the same counts and bincount.txt lines."""
import os

import pytest

from engine_fixtures import dms_b200

pytestmark = pytest.mark.gpu

SIGMA_CM2 = 1.0e-100 * 1.0e-36   # 1e-100 pb
MASS_GEV = 0.01


@pytest.fixture(scope="module")
def engine():
    e = dms_b200.Engine(0)
    yield e
    e.close()


def _point(engine, n=1000):
    return engine.add_point(dms_b200.point_params(MASS_GEV, SIGMA_CM2, sigma_e_cm2=SIGMA_CM2, interpolation_points=n))


def _bincount(engine, pid, gen, tmp_path):
    d = str(tmp_path / "out")
    engine.write_outputs(pid, gen, MASS_GEV, SIGMA_CM2, d)
    return open(os.path.join(d, "bincount.txt")).read()


def _valid(c):
    return c["captured"] + c["completed_outward_escapes"]


def test_initial_shift_failure_is_reported(engine, tmp_path):
    """TestInitialShiftFailureIsReported (tests/test_Data_Generation.cpp:276-303): a boundary
    inside the Sun makes every initial Kepler shift fail; the run stops on the shift-failure fuse."""
    pid = _point(engine)
    gen = engine.generate(pid, sample_size=1, max_trajectories=1, boundary_rsun=0.5, max_scatterings=1, max_free_steps=10,
                          sigma_p_cm2=SIGMA_CM2)
    c = gen["counters"]
    assert _valid(c) == 0
    assert c["numerical_failures"] == c["trajectories"] == 1
    assert c["initial_shift_failures"] == 1
    assert "# EARLY_STOP: initial_shift_failure_fraction_exceeded" in _bincount(engine, pid, gen, tmp_path)


def test_computationally_truncated_non_capture_is_excluded_from_capture_rate(engine, tmp_path):
    """TestComputationallyTruncatedNonCaptureIsExcludedFromCaptureRate (:305-335)."""
    pid = _point(engine)
    gen = engine.generate(pid, sample_size=1, max_trajectories=1, seed=20260710, boundary_rsun=2.0, max_scatterings=0,
                          max_free_steps=10, sigma_p_cm2=SIGMA_CM2)
    c = gen["counters"]
    assert _valid(c) == 0 and c["numerical_failures"] == 0
    text = _bincount(engine, pid, gen, tmp_path)
    for line in ("# valid_trajectories = 0", "# unresolved_not_captured_trajectories = 1", "# computational_truncations = 1",
                 "# capture_rate_valid = 0.00000000", "# capture_rate_valid_CI_95_lower = 0.00000000",
                 "# EARLY_STOP: max_trajectories_reached"):
        assert line in text, line


def test_unlimited_budget_stops_when_every_trajectory_is_invalid(engine, tmp_path):
    """TestUnlimitedBudgetStopsWhenEveryTrajectoryIsInvalid (:337-357): capture mode, no
    trajectory budget, every trajectory truncated: the invalid-fraction fuse ends the run."""
    pid = _point(engine)
    gen = engine.generate(pid, sample_size=1, max_trajectories=0, seed=20260710, capture_mode=True, boundary_rsun=2.0,
                          max_scatterings=0, max_free_steps=10, sigma_p_cm2=SIGMA_CM2, time_limit_s=60.0)
    assert gen["early_stop"] == "invalid_trajectory_fraction_exceeded"
    assert "# EARLY_STOP: invalid_trajectory_fraction_exceeded" in _bincount(engine, pid, gen, tmp_path)


def test_capture_mode_completed_escape_is_included_in_capture_rate(engine):
    """TestCaptureModeCompletedEscapeIsIncludedInCaptureRate (:359-378): a 10 x 10 rate grid, a
    boundary at 1.1 R_sun, up to 500 scatterings: the particle crosses the Sun unscattered and
    escapes, a valid non-capture."""
    pid = _point(engine, n=10)
    gen = engine.generate(pid, sample_size=1, max_trajectories=1, seed=20260710, capture_mode=True, boundary_rsun=1.1,
                          max_scatterings=500, sigma_p_cm2=SIGMA_CM2)
    c = gen["counters"]
    assert _valid(c) == 1
    assert c["captured"] == 0 and c["numerical_failures"] == 0
