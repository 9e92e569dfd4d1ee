"""The launch autotuner (dms_autotune) and the lane-scheduling options it sets: block size,
blocks per SM, queue chunk and the warp batching of scatterings and terminations (B200
required).

Every draw is keyed by (seed, point, trajectory id), so these options may change throughput but
never results: the same ids under the tuned and the default settings, and under deliberately
odd ones, give the same counters, the same evaporation events and histograms equal up to the
order of the floating-point atomic additions.  The tuner's trial launches run on fresh ids into
a scratch accumulator and leave the points' own results untouched."""
import numpy as np
import pytest

from engine_fixtures import REPLAY_POINT, dms_b200

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    e = dms_b200.Engine(0)
    p = REPLAY_POINT
    pid = e.add_point(dms_b200.point_params(p["mass_gev"], p["sigma_p_cm2"], interpolation_points=p["interpolation_points"]))
    yield e, pid
    e.close()


def _run(e, pid, opts, n=8192):
    e.reset_results(pid)
    e.run([(pid, 0, n)], opts)
    return e.results(pid)


def _same(a, b):
    ca, cb = dict(a["counters"]), dict(b["counters"])
    assert ca == cb
    assert np.allclose(a["histograms"], b["histograms"], rtol=1e-12, atol=0.0)
    ea, eb = np.sort(a["events"], order="trajectory_id"), np.sort(b["events"], order="trajectory_id")
    assert np.array_equal(ea, eb)


def test_autotune_picks_settings_that_leave_results_unchanged(engine):
    e, pid = engine
    base = dms_b200.run_opts(seed=7, max_scatterings=10 ** 6, time_limit_s=300.0)
    e.reset_results(pid)
    e.run([(pid, 0, 64)], base)
    before = e.results(pid)
    tuned, trials = e.autotune([(pid, 0, 8192)], base, trial_seconds=0.1)
    assert trials >= 8
    chosen = dms_b200.lane_options(tuned)
    print({"tuned": chosen, "trials": trials})
    assert chosen["threads_per_block"] in (0, 64, 96, 128) and chosen["queue_chunk"] in (0, 1, 2, 4)
    assert tuned.seed == base.seed and tuned.max_scatterings == base.max_scatterings
    # the trials touched only a scratch accumulator
    _same(before, e.results(pid))
    _same(_run(e, pid, base), _run(e, pid, tuned))


def test_odd_lane_options_leave_results_unchanged(engine):
    e, pid = engine
    base = dms_b200.run_opts(seed=3, max_scatterings=10 ** 6, time_limit_s=300.0)
    odd = dms_b200.run_opts(seed=3, max_scatterings=10 ** 6, time_limit_s=300.0, threads_per_block=96, blocks_per_sm=2,
                            queue_chunk=7, scatter_batch=1, scatter_wait=1, final_batch=32, final_wait=1024)
    _same(_run(e, pid, base, 5000), _run(e, pid, odd, 5000))


def test_lane_options_are_validated(engine):
    e, pid = engine
    for kw in (dict(queue_chunk=1025), dict(scatter_batch=33), dict(final_wait=1025)):
        with pytest.raises(dms_b200.EngineError):
            e.run([(pid, 0, 4)], dms_b200.run_opts(seed=1, **kw))
