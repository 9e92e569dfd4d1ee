"""Generates the golden fixtures of tests/golden from the reference's OWN hot-path sources
(compiled by oracle/Makefile into oracle/_ref/libdms_ref.so against the shims in oracle/shim).

reference_records.json: table values at fixed radii, and per-trajectory outcomes for
trajectories 0..N-1 of the point m = 0.3 GeV, sigma_p = 1e-36 cm^2 (SHM of the reference test
configs, 200 x 200 rate grid), seed 7, in Parameter-point and Capture mode, plus the first
scattering (r, v, draw index) of the first trajectories.

reference_dark_photon.json: the reference's dark photon (src/Dark_Photon.cpp) in low-mass mode,
"Contact" and "General" with two mediator masses: channel and total rates on a grid of (r, v),
and per-trajectory outcomes of trajectories 0..N_DP-1 in Parameter-point mode.
Run:  python tests/golden/make_golden.py
"""
import json
import math
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from dms_ctypes import RSUN_KM, Reference, point_params, records_to_dicts  # noqa: E402

N_TRAJ = 300
N_TRACE = 60
SEED = 7
POINT = dict(mass_gev=0.3, sigma_p_cm2=1e-36, interpolation_points=200)


def clean(x):
    if isinstance(x, float) and math.isnan(x):
        return "nan"
    if isinstance(x, (list, tuple)):
        return [clean(v) for v in x]
    return x


N_DP = 120
DP_POINTS = [dict(name="contact", mass_gev=0.3, sigma_e_cm2=5e-42, interaction=1, mediator_mass_mev=0.0),
             dict(name="general_1MeV", mass_gev=0.3, sigma_e_cm2=1e-40, interaction=2, mediator_mass_mev=1.0),
             dict(name="general_0.2MeV", mass_gev=1.0, sigma_e_cm2=2e-39, interaction=2, mediator_mass_mev=0.2)]
DP_RADII = [1.0e4, 1.0e5, 3.0e5, 6.0e5]
DP_SPEEDS = [5.0, 80.0, 400.0, 1500.0]
DP_CHANNELS = [-1, 0, 1, 4, 12, 40, 62]


def dark_photon(ref):
    out = {"seed": SEED, "radii_km": DP_RADII, "speeds_kms": DP_SPEEDS, "channels": DP_CHANNELS, "points": []}
    for p in DP_POINTS:
        ref.set_point(point_params(p["mass_gev"], 0.0, sigma_e_cm2=p["sigma_e_cm2"], interpolation_points=200,
                                   interaction=p["interaction"], mediator_mass_mev=p["mediator_mass_mev"]))
        rates = [[[ref.query(12, r, k, v) for k in DP_CHANNELS] + [ref.query(6, r, v)] for v in DP_SPEEDS] for r in DP_RADII]
        res = ref.run_records(SEED, 0, 0, N_DP, capture_mode=False)
        recs = [{k: clean(d[k]) for k in ("id", "nscat", "draws", "reason", "flags", "final", "lifetime")}
                for d in records_to_dicts(res["records"])]
        out["points"].append(dict(p, rates=rates, records=recs))
    with open(os.path.join(HERE, "reference_dark_photon.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))


def main():
    ref = Reference()
    if "--dark-photon-only" in sys.argv:
        dark_photon(ref)
        return
    radii = [0.0, 0.0015 * RSUN_KM, 0.1 * RSUN_KM, 0.5 * RSUN_KM, 0.9695 * RSUN_KM, RSUN_KM, 1.5 * RSUN_KM]
    tables = {name: [ref.query(code, r) for r in radii] for code, name in [(0, "gm"), (1, "temperature_K"), (2, "vesc"), (3, "n_e")]}
    tables["n_h1"] = [ref.query(4, r, 0) for r in radii]
    tables["radii_km"] = radii
    ref.set_point(point_params(POINT["mass_gev"], POINT["sigma_p_cm2"], interpolation_points=POINT["interpolation_points"]))
    out = {"point": POINT, "seed": SEED, "tables": tables, "modes": {}}
    for mode in ("normal", "capture"):
        res = ref.run_records(SEED, 0, 0, N_TRAJ, capture_mode=(mode == "capture"))
        recs = []
        for d in records_to_dicts(res["records"]):
            recs.append({k: clean(d[k]) for k in ("id", "nscat", "draws", "reason", "flags", "initial", "final",
                                                  "t_capture", "lifetime")})
        traces = []
        for t in range(N_TRACE):
            tr = ref.run_records(SEED, 0, t, 1, capture_mode=(mode == "capture"), trace_capacity=1)["trace"]
            traces.append([float(v) for v in tr[0]] if len(tr) else None)
        out["modes"][mode] = {"records": recs, "first_scatter": traces}
    with open(os.path.join(HERE, "reference_records.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
    dark_photon(ref)


if __name__ == "__main__":
    main()
