"""Faults injected on the host, each of which must end in an error status or a termination
reason and leave the context usable (B200 required): a solar model file cut in the middle of
a row, one with text or NaN where numbers belong, an empty one; a rate grid poisoned with NaN;
a point without any cross section.  Nothing here faults the GPU: the bad inputs are caught by
the host, or by the kernel's own finiteness checks."""
import numpy as np
import pytest

from engine_fixtures import dms_b200

pytestmark = pytest.mark.gpu

REASON_OUTWARD_ESCAPE = 1
REASON_NUMERICAL_FAILURE = 8


@pytest.fixture(scope="module")
def engine():
    e = dms_b200.Engine(0)
    yield e
    e.close()


def _lines():
    with open(dms_b200.SOLAR_MODEL) as f:
        return f.read().splitlines(keepends=True)


@pytest.mark.parametrize("kind", ["cut_mid_row", "text", "nan_radius", "empty"])
def test_bad_solar_model_files_are_rejected(engine, tmp_path, kind):
    lines = _lines()
    if kind == "cut_mid_row":
        text = "".join(lines[:400]) + lines[400][: len(lines[400]) // 2]
    elif kind == "text":
        text = "".join(lines[:300]) + lines[300].replace(lines[300].split()[3], "abc", 1) + "".join(lines[301:])
    elif kind == "nan_radius":
        fields = lines[300].split()
        text = "".join(lines[:300]) + lines[300].replace(fields[1], "nan", 1) + "".join(lines[301:])
    else:
        text = ""
    bad = tmp_path / "model.dat"
    bad.write_text(text)
    with pytest.raises(dms_b200.EngineError):
        engine._check(engine.lib.dms_load_solar_model(engine.h, str(bad).encode()))
    # the context keeps working with the real model
    engine._check(engine.lib.dms_load_solar_model(engine.h, dms_b200.SOLAR_MODEL.encode()))
    pid = engine.add_point(dms_b200.point_params(0.3, 1e-36, interpolation_points=50))
    out = engine.run_records(pid, 0, 8, dms_b200.run_opts(seed=1, capture_mode=True, time_limit_s=60.0))
    assert all(0 <= out["records"][i].termination_reason < 11 for i in range(8))


def test_nan_poisoned_rate_grid_ends_trajectories_as_numerical_failures(engine):
    pid = engine.add_point(dms_b200.point_params(0.3, 1e-36, interpolation_points=100))
    engine.set_rate_grid(pid, np.full((100, 100), np.nan))
    n = 256
    opts = dms_b200.run_opts(seed=2, capture_mode=True, max_scatterings=10 ** 4, time_limit_s=60.0)
    recs = engine.run_records(pid, 0, n, opts)["records"]
    reasons = [recs[i].termination_reason for i in range(n)]
    # every trajectory that enters the Sun reads a NaN rate; the rest pass by and escape
    assert REASON_NUMERICAL_FAILURE in reasons
    assert set(reasons) <= {REASON_NUMERICAL_FAILURE, REASON_OUTWARD_ESCAPE}
    assert all(recs[i].number_of_scatterings == 0 for i in range(n))
    engine.reset_results(pid)
    engine.run([(pid, 0, n)], opts)
    c = engine.results(pid, events_capacity=1)["counters"]
    assert c["trajectories"] == n and c["numerical_failures"] == reasons.count(REASON_NUMERICAL_FAILURE)


def test_point_without_cross_section_never_scatters(engine):
    pid = engine.add_point(dms_b200.point_params(0.3, 0.0, sigma_e_cm2=0.0, interpolation_points=100))
    n = 512
    recs = engine.run_records(pid, 0, n, dms_b200.run_opts(seed=4, max_scatterings=10 ** 4, time_limit_s=60.0))["records"]
    assert all(recs[i].number_of_scatterings == 0 for i in range(n))
    assert all(recs[i].termination_reason == REASON_OUTWARD_ESCAPE for i in range(n))
    assert not any(recs[i].flags & 0x2 for i in range(n))
