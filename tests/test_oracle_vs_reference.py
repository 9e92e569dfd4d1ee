"""The C oracle against the reference's own sources (golden fixtures written by
tests/golden/make_golden.py from oracle/_ref, the reference compiled against the shims).

Bit-level agreement is not expected between the two: the reference computes in natural units
and the oracle in km/s, and the surface approach of Propagate_Freely has a knife edge (a step
that lands exactly on R_sun versus one ulp outside takes a different step-size branch,
src/Simulation_Trajectory.cpp:886-899).  What must hold: identical tables, identical draw
consumption and classification for single-segment trajectories, first scatterings within 1e-7
relative (median below 1e-10), and >= 98 % identical outcomes for long evaporating ones."""
import json
import math
import os

import numpy as np
import pytest

from dms_ctypes import point_params

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_records.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def oracle_golden_point(oracle, golden):
    p = golden["point"]
    oracle.set_point(point_params(p["mass_gev"], p["sigma_p_cm2"], interpolation_points=p["interpolation_points"]))
    return oracle


def test_tables_match_reference(oracle, golden):
    t = golden["tables"]
    for code, name, tol in [(0, "gm", 1e-14), (1, "temperature_K", 1e-13), (2, "vesc", 1e-14), (3, "n_e", 1e-9)]:
        for r, expect in zip(t["radii_km"], t[name]):
            got = oracle.query(code, r)
            assert got == pytest.approx(expect, rel=tol, abs=0.0), (name, r)
    for r, expect in zip(t["radii_km"], t["n_h1"]):
        assert oracle.query(4, r, 0) == pytest.approx(expect, rel=1e-9, abs=0.0)


def _outcome(d):
    return (d["nscat"], d["reason"], d["flags"], d["draws"])


def test_capture_mode_outcomes_identical(oracle_golden_point, golden):
    ref = golden["modes"]["capture"]["records"]
    res = oracle_golden_point.run_records(golden["seed"], 0, 0, len(ref), capture_mode=True)
    from dms_ctypes import records_to_dicts
    mine = records_to_dicts(res["records"])
    for a, b in zip(ref, mine):
        assert _outcome(a) == _outcome(b), a["id"]
        x, y = np.array(a["initial"][1]), np.array(b["initial"][1])
        assert np.max(np.abs(x - y)) <= 1e-9 * np.linalg.norm(x)


def test_parameter_point_outcomes_agree(oracle_golden_point, golden):
    ref = golden["modes"]["normal"]["records"]
    res = oracle_golden_point.run_records(golden["seed"], 0, 0, len(ref), capture_mode=False)
    from dms_ctypes import records_to_dicts
    mine = records_to_dicts(res["records"])
    same = sum(_outcome(a) == _outcome(b) for a, b in zip(ref, mine))
    assert same >= int(math.ceil(0.98 * len(ref)))
    captured_ref = sum(1 for a in ref if a["flags"] & 2)
    captured_mine = sum(1 for b in mine if b["flags"] & 2)
    assert captured_ref == captured_mine


@pytest.mark.parametrize("mode", ["normal", "capture"])
def test_first_scattering_agrees(oracle_golden_point, golden, mode):
    errs = []
    for t, ref_tr in enumerate(golden["modes"][mode]["first_scatter"]):
        tr = oracle_golden_point.run_records(golden["seed"], 0, t, 1, capture_mode=(mode == "capture"), trace_capacity=1)["trace"]
        assert (ref_tr is None) == (len(tr) == 0)
        if ref_tr is None:
            continue
        assert tr[0][2] == ref_tr[2]  # same draw index at the scattering
        errs.append(max(abs(tr[0][0] - ref_tr[0]) / ref_tr[0], abs(tr[0][1] - ref_tr[1]) / ref_tr[1]))
    assert errs and max(errs) < 1e-7 and float(np.median(errs)) < 1e-10


@pytest.mark.parametrize("mode", ["normal", "capture"])
def test_replay_from_the_reference_initial_states(oracle_golden_point, golden, mode):
    """The path after the initial conditions, pinned separately.  The map from the halo sample at
    1000 AU to the event at 2 R_sun (Initial_Conditions + Hyperbolic_Kepler_Shift,
    src/Simulation_Utilities.cpp:176-321) amplifies last-bit differences about 1e7-fold, so the
    oracle's own initial states (km units, the shared series for sin/cos/acos) differ from the
    reference's (natural units, glibc) by about 1e-9 relative.  Started from the reference's own
    shifted states (the fixture's "initial"), the oracle reproduces the outcomes of (nearly)
    every trajectory, and the first scatterings agree to 1e-10 for most of them; the rest differ
    because the RK45 step-size control divides the tolerance by |r5 - r4|, a cancellation whose
    last bits differ between unit systems, so step sequences carry rounding noise
    (src/Simulation_Trajectory.cpp:477-502, 1540-1545)."""
    from dms_ctypes import records_to_dicts
    import numpy as np
    ref = golden["modes"][mode]["records"]
    starts = np.array([[r["initial"][0]] + list(r["initial"][1]) + list(r["initial"][2]) for r in ref])
    capture = mode == "capture"
    mine = records_to_dicts(oracle_golden_point.run_from_starts(golden["seed"], 0, 0, starts, capture_mode=capture)["records"])
    same = sum(_outcome(a) == _outcome(b) for a, b in zip(ref, mine))
    assert same >= (len(ref) if capture else int(math.ceil(0.99 * len(ref))))
    errs = []
    for t, ref_tr in enumerate(golden["modes"][mode]["first_scatter"]):
        if ref_tr is None:
            continue
        tr = oracle_golden_point.run_from_starts(golden["seed"], 0, t, starts[t:t + 1], capture_mode=capture,
                                                 trace_capacity=1)["trace"]
        assert tr[0][2] == ref_tr[2]
        errs.append(max(abs(tr[0][0] - ref_tr[0]) / ref_tr[0], abs(tr[0][1] - ref_tr[1]) / ref_tr[1]))
    errs = np.array(errs)
    assert np.median(errs) < 2e-11 and np.mean(errs <= 1e-10) >= 0.85 and errs.max() < 1e-8


DP_GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_dark_photon.json")


@pytest.fixture(scope="module")
def dp_golden():
    with open(DP_GOLDEN) as f:
        return json.load(f)


def _dp_point(p):
    return point_params(p["mass_gev"], 0.0, sigma_e_cm2=p["sigma_e_cm2"], interpolation_points=200,
                        interaction=p["interaction"], mediator_mass_mev=p["mediator_mass_mev"])


@pytest.mark.parametrize("which", [0, 1, 2])
def test_dark_photon_rates_match_reference(oracle, dp_golden, which):
    """Channel and total rates of the dark photon (src/Dark_Photon.cpp:167-229 through
    src/Solar_Model.cpp:263-342): the kinetic-mixing cross sections and the General form factor."""
    p = dp_golden["points"][which]
    oracle.set_point(_dp_point(p))
    for i, r in enumerate(dp_golden["radii_km"]):
        for j, v in enumerate(dp_golden["speeds_kms"]):
            want = p["rates"][i][j]
            got = [oracle.query(12, r, k, v) for k in dp_golden["channels"]] + [oracle.query(6, r, v)]
            for a, b in zip(got, want):
                assert a == pytest.approx(b, rel=1e-9, abs=0.0), (p["name"], r, v)
    assert p["rates"][1][2][-1] > 0.0


@pytest.mark.parametrize("which", [0, 1, 2])
def test_dark_photon_outcomes_agree(oracle, dp_golden, which):
    """Trajectory outcomes with the dark photon's scattering angles (isotropic for Contact, the
    closed-form General sampler, src/Dark_Photon.cpp:286-325)."""
    from dms_ctypes import records_to_dicts
    p = dp_golden["points"][which]
    oracle.set_point(_dp_point(p))
    ref = p["records"]
    mine = records_to_dicts(oracle.run_records(dp_golden["seed"], 0, 0, len(ref))["records"])
    same = sum(_outcome(a) == _outcome(b) for a, b in zip(ref, mine))
    assert same >= int(math.ceil(0.98 * len(ref))), (p["name"], same)
    assert sum(1 for a in ref if a["flags"] & 2) == sum(1 for b in mine if b["flags"] & 2)
    assert sum(a["nscat"] for a in ref) > len(ref)
