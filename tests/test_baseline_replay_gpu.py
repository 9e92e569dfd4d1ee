"""Deterministic replay of the engine against the CPU oracle at the benchmark configurations,
with the engine's own device-built 1000 x 1000 rate grid (B200 required).

The device builds the grid with CUDA's erf/exp and the oracle with the C library's, so the two
grids differ in the last bits (within 1e-13 relative).  Each replay therefore runs twice:

* the oracle on the engine's grid (dms_oracle_set_rate_grid): every outcome (scatter count,
  termination reason, flags, draw count) identical and the final FP64 state within 1e-10
  relative, trajectory by trajectory;
* the oracle on its own CPU-built grid: the number of trajectories whose outcome differs is
  reported and must stay below 3 % (a last-bit rate difference moves a scattering point by
  about 1e-13 and chaotic random walks amplify it).

Configurations: Capture mode m = 1 GeV, sigma_n = 1e-35 cm^2, seed 1, max 1e5 scatterings,
ids 0..4095; Parameter point m = 0.3 GeV, sigma_n = 1e-36 cm^2, seed 7, max 1e6 scatterings,
ids 0..2047; heavy scattering m = 0.1 GeV, sigma_n = 1e-33 cm^2, seed 11, max 1e7 scatterings,
ids 0..511 (Parameter-point mode, under a 300 s launch limit)."""
import json

import numpy as np
import pytest

from engine_fixtures import dms_b200, outcome, state
import cpu_pool

pytestmark = pytest.mark.gpu

CASES = {
    "capture_1GeV_1e-35": dict(params=dict(mass_gev=1.0, sigma_p_cm2=1e-35, interpolation_points=1000), seed=1,
                               capture_mode=True, max_scatterings=10 ** 5, count=4096),
    "parameter_point_0.3GeV_1e-36": dict(params=dict(mass_gev=0.3, sigma_p_cm2=1e-36, interpolation_points=1000), seed=7,
                                         capture_mode=False, max_scatterings=10 ** 6, count=2048),
    "heavy_0.1GeV_1e-33": dict(params=dict(mass_gev=0.1, sigma_p_cm2=1e-33, interpolation_points=1000), seed=11,
                               capture_mode=False, max_scatterings=10 ** 7, count=512),
}


@pytest.fixture(scope="module")
def engine():
    e = dms_b200.Engine(0)
    yield e
    e.close()


def _outcomes(recs, n):
    return [outcome(recs[i]) for i in range(n)]


@pytest.mark.parametrize("name", list(CASES))
def test_replay_on_the_device_built_grid(engine, name):
    cfg = CASES[name]
    p, n = cfg["params"], cfg["count"]
    pid = engine.add_point(dms_b200.point_params(p["mass_gev"], p["sigma_p_cm2"],
                                                 interpolation_points=p["interpolation_points"]))
    grid = engine.rate_grid(pid, p["interpolation_points"])
    opts = dms_b200.run_opts(seed=cfg["seed"], capture_mode=cfg["capture_mode"], max_scatterings=cfg["max_scatterings"],
                             time_limit_s=300.0)
    mine = engine.run_records(pid, 0, n, opts)["records"]
    kw = dict(capture_mode=cfg["capture_mode"], max_scatterings=cfg["max_scatterings"], point=pid)
    on_device_grid = cpu_pool.run_ensemble("oracle", p, cfg["seed"], 0, n, grid=grid, **kw)["outcomes"]
    on_own_grid = cpu_pool.run_ensemble("oracle", p, cfg["seed"], 0, n, **kw)["outcomes"]

    def table(o):
        return [(int(o["nscat"][i]), int(o["reason"][i]), int(o["flags"][i]), int(o["draws"][i])) for i in range(n)]

    a = _outcomes(mine, n)
    b, c = table(on_device_grid), table(on_own_grid)
    bad_device = [i for i in range(n) if a[i] != b[i]]
    bad_own = [i for i in range(n) if a[i] != c[i]]
    s_mine = np.array([state(mine[i]) for i in range(n)])
    s_oracle = on_device_grid["final_state"]
    rel = np.abs(s_mine - s_oracle) / np.maximum(np.abs(s_oracle), 1e-300)
    report = {"case": name, "trajectories": n, "captured": sum(1 for i in range(n) if mine[i].flags & 0x2),
              "scatterings": int(sum(x[0] for x in a)),
              "mismatches_on_device_grid": len(bad_device), "mismatches_on_oracle_grid": len(bad_own),
              "first_mismatches_on_oracle_grid": bad_own[:10], "max_final_state_rel_error": float(np.max(rel))}
    print(json.dumps(report))
    assert not bad_device, report
    assert float(np.max(rel)) <= 1e-10, report
    assert len(bad_own) <= 0.03 * n, report
