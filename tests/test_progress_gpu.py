"""Live progress of a launch in flight (dms_set_progress_callback, dms_peek_progress,
dms_peek_results) through the C ABI (B200 required).

The hook runs on the thread that waits for the launch, so a peek that waited for the kernel
would show up as one late call instead of many; the published evaporation events of every peek
must be a prefix of the final event list, slot for slot."""
import time

import numpy as np
import pytest

from engine_fixtures import REPLAY_POINT, dms_b200

pytestmark = pytest.mark.gpu

QUEUE = 1 << 24   # far more trajectories than the time limit lets finish


@pytest.fixture(scope="module")
def engine():
    e = dms_b200.Engine(0)
    p = REPLAY_POINT
    pid = e.add_point(dms_b200.point_params(p["mass_gev"], p["sigma_p_cm2"], interpolation_points=p["interpolation_points"]))
    yield e, pid
    e.close()


def test_progress_hook_reads_the_launch_in_flight(engine):
    e, pid = engine
    e.reset_results(pid)
    seen = []

    def hook(eng):
        t0 = time.perf_counter()
        pr = eng.peek_progress()
        r = eng.peek_results(pid, events_capacity=1 << 16)
        seen.append({"progress": pr, "trajectories": r["counters"]["trajectories"],
                     "scatterings": r["counters"]["total_scatterings"], "events": r["events"].copy(),
                     "seconds": time.perf_counter() - t0})
        return False

    e.set_progress_callback(hook, 0.05)
    try:
        with pytest.raises(dms_b200.EngineError, match="wall-clock limit"):
            e.run([(pid, 0, QUEUE)], dms_b200.run_opts(seed=11, max_scatterings=10 ** 6, time_limit_s=1.5))
    finally:
        e.set_progress_callback(None)
    final = e.results(pid, events_capacity=1 << 16)

    assert len(seen) >= 10, len(seen)
    assert all(s["progress"]["running"] and s["progress"]["total"] == QUEUE for s in seen)
    assert max(s["seconds"] for s in seen) < 0.25
    dispatched = [s["progress"]["dispatched"] for s in seen]
    done = [s["trajectories"] for s in seen]
    scat = [s["scatterings"] for s in seen]
    assert dispatched == sorted(dispatched) and dispatched[-1] > 0
    assert done == sorted(done) and scat == sorted(scat) and done[-1] > 0
    assert all(d <= q for d, q in zip(done, dispatched))
    assert final["counters"]["trajectories"] >= done[-1]
    assert len(final["events"]) > 0
    for s in seen:
        k = len(s["events"])
        assert np.array_equal(s["events"], final["events"][:k])
    assert e.peek_progress()["running"] is False


def test_calls_that_change_the_launch_are_refused_in_the_hook(engine):
    e, pid = engine
    e.reset_results(pid)
    refused = []

    def hook(eng):
        for call in (lambda: eng.add_point(dms_b200.point_params(0.3, 1e-36, interpolation_points=50)),
                     lambda: eng.reset_results(pid),
                     lambda: eng.run([(pid, 0, 4)], dms_b200.run_opts(seed=1)),
                     lambda: eng.run_records_noalloc(pid, 0, 4, dms_b200.run_opts(seed=1), None)):
            try:
                call()
            except dms_b200.EngineError as err:
                refused.append("in flight" in str(err))
        return True

    e.set_progress_callback(hook, 0.05)
    try:
        with pytest.raises(dms_b200.EngineError, match="progress callback"):
            e.run([(pid, 0, QUEUE)], dms_b200.run_opts(seed=3, max_scatterings=10 ** 6, time_limit_s=60.0))
    finally:
        e.set_progress_callback(None)
    assert refused == [True, True, True, True]
    n = e.lib.dms_num_points(e.h)
    assert n == 1   # the refused add_point left no point behind


def test_progress_hook_can_cancel(engine):
    e, pid = engine
    e.reset_results(pid)
    e.set_progress_callback(lambda eng: True, 0.05)
    try:
        t0 = time.perf_counter()
        with pytest.raises(dms_b200.EngineError, match="progress callback"):
            e.run([(pid, 0, QUEUE)], dms_b200.run_opts(seed=3, max_scatterings=10 ** 6, time_limit_s=60.0))
        assert time.perf_counter() - t0 < 30.0
    finally:
        e.set_progress_callback(None)


def test_peek_after_run_matches_results(engine):
    e, pid = engine
    e.reset_results(pid)
    e.run([(pid, 0, 4096)], dms_b200.run_opts(seed=5, max_scatterings=10 ** 6))
    got, want = e.peek_results(pid), e.results(pid)
    assert got["counters"] == want["counters"]
    assert np.array_equal(got["histograms"], want["histograms"])
    assert np.array_equal(got["events"], want["events"])
