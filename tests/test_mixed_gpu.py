"""Mixed-precision (batched FP32) kernel against the FP64 kernel on the same trajectories.

The two forms draw from the same Philox streams but round differently, so trajectories part
ways after a few steps and agreement is statistical.  Acceptance, per point: capture fraction
within 1 binomial standard error of the FP64 run, and every ensemble gate of the reference's
validation script (capture intervals overlap, evaporation fraction z <= 3, mean scatterings
within 10 %, captured radial total variation <= 0.10, evaporation median within 20 % and
90th percentile within 30 %).  The per-bin chi-squared of the captured radial histogram is
reported with the comparison (B200 required)."""
import json

import pytest

from engine_fixtures import dms_b200
import dms_stats

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    e = dms_b200.Engine(0)
    yield e
    e.close()


def run_both(engine, mass, sigma, capture_mode, seed, n, max_scatterings=10 ** 6):
    pid = engine.add_point(dms_b200.point_params(mass, sigma, interpolation_points=1000))
    out = []
    for precision in (dms_b200.PRECISION_FP64, dms_b200.PRECISION_MIXED):
        engine.reset_results(pid)
        engine.run([(pid, 0, n)], dms_b200.run_opts(seed=seed, capture_mode=capture_mode, max_scatterings=max_scatterings,
                                                    time_limit_s=300.0, precision=precision))
        out.append(engine.results(pid))
    return out


def check(ref, mixed):
    cmp = dms_stats.compare_runs(ref, mixed)
    gates = dms_stats.reference_gates(ref, mixed)
    report = json.dumps({"compare": cmp, "gates": gates}, default=str)
    print(report)
    assert ref["counters"]["captured"] > 100, report
    assert cmp["capture_fraction_sigmas"] <= 1.0, report
    failed = [k for k, (ok, _) in gates.items() if not ok]
    assert not failed, report
    return cmp


def test_parameter_point_mixed_agrees_with_fp64(engine):
    ref, mixed = run_both(engine, 0.3, 1e-36, capture_mode=False, seed=7, n=1 << 18)
    check(ref, mixed)
    assert mixed["counters"]["trajectories"] == 1 << 18
    assert len(mixed["events"]) >= 30


def test_capture_mode_mixed_agrees_with_fp64(engine):
    ref, mixed = run_both(engine, 1.0, 1e-35, capture_mode=True, seed=1, n=1 << 16, max_scatterings=10 ** 5)
    check(ref, mixed)


def test_mixed_records_mode_runs(engine):
    pid = engine.add_point(dms_b200.point_params(0.3, 1e-36, interpolation_points=1000))
    opts = dms_b200.run_opts(seed=7, max_scatterings=10 ** 6, time_limit_s=120.0, precision=dms_b200.PRECISION_MIXED)
    out = engine.run_records(pid, 0, 256, opts, histograms=True)
    recs = out["records"]
    assert all(recs[i].termination_reason in range(11) for i in range(256))
    assert all(recs[i].trajectory_id == i for i in range(256))
