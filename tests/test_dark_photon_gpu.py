"""The dark photon interaction (src/Dark_Photon.cpp) on the CUDA engine against the C oracle,
through the C ABI (B200 required).

The points are those of tests/golden/reference_dark_photon.json, where the oracle is pinned to
the reference's own dark photon.  Tolerances as in test_engine_gpu.py: the device-built rate
grid (CUDA's erf/exp) to 1e-13 relative; replayed FP64 trajectories on the oracle's grid in
identical outcome and draw count, states to 1e-10 relative.  The mixed-precision form is a
different arithmetic, so it is held to the ensemble: its capture fraction within 4 combined
binomial standard deviations of the FP64 form's."""
import json
import math
import os

import numpy as np
import pytest

from dms_ctypes import point_params as oracle_point_params
from engine_fixtures import dms_b200, outcome, state

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_dark_photon.json")
with open(GOLDEN) as _f:
    POINTS = json.load(_f)["points"]


@pytest.fixture(scope="module")
def engine():
    e = dms_b200.Engine(0)
    yield e
    e.close()


def _params(module, p, n=200):
    return module(p["mass_gev"], 0.0, sigma_e_cm2=p["sigma_e_cm2"], interpolation_points=n,
                  interaction=p["interaction"], mediator_mass_mev=p["mediator_mass_mev"])


@pytest.mark.parametrize("which", range(len(POINTS)))
def test_dark_photon_replay_matches_oracle(engine, oracle, which):
    p = POINTS[which]
    oracle.set_point(_params(oracle_point_params, p))
    pid = engine.add_point(_params(dms_b200.point_params, p))
    og = oracle.rate_grid()
    dg = engine.rate_grid(pid, 200)
    assert np.max(np.abs(dg - og) / np.maximum(np.abs(og), 1e-300)) < 1e-13
    engine.set_rate_grid(pid, og)
    n = 300
    opts = dms_b200.run_opts(seed=7, capture_mode=False, max_scatterings=10 ** 6, time_limit_s=120.0)
    a = engine.run_records(pid, 0, n, opts)["records"]
    b = oracle.run_records(7, pid, 0, n, capture_mode=False, max_scatterings=10 ** 6)["records"]
    mism = [i for i in range(n) if outcome(a[i]) != outcome(b[i])]
    assert not mism, [(i, outcome(a[i]), outcome(b[i])) for i in mism[:5]]
    worst = 0.0
    for i in range(n):
        x, y = np.array(state(a[i])), np.array(state(b[i]))
        worst = max(worst, float(np.max(np.abs(x - y) / np.maximum(np.abs(y), 1e-300))))
        assert a[i].lifetime_unbinding == b[i].lifetime_unbinding
    assert worst <= 1e-10, worst
    assert sum(a[i].number_of_scatterings for i in range(n)) > n


def test_dark_photon_general_mixed_form_capture_fraction(engine):
    p = POINTS[2]
    pid = engine.add_point(_params(dms_b200.point_params, p, n=1000))
    n = 1 << 16
    frac = {}
    for name, prec in (("fp64", dms_b200.PRECISION_FP64), ("mixed", dms_b200.PRECISION_MIXED)):
        engine.reset_results(pid)
        engine.run([(pid, 0, n)], dms_b200.run_opts(seed=21, capture_mode=True, max_scatterings=10 ** 6,
                                                   time_limit_s=300.0, precision=prec))
        c = engine.results(pid, events_capacity=1)["counters"]
        assert c["trajectories"] == n
        frac[name] = c["captured"] / n
    sigma = math.sqrt(frac["fp64"] * (1 - frac["fp64"]) / n + frac["mixed"] * (1 - frac["mixed"]) / n)
    assert frac["fp64"] > 0.01
    assert abs(frac["mixed"] - frac["fp64"]) <= 4.0 * sigma, (frac, sigma)
