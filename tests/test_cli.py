"""The `dms_sun` command-line drop-in: configuration errors (CPU, the file is read before any
CUDA call) and complete Parameter-point and Capture runs with their summary and output files
(B200 required)."""
import math
import os
import subprocess

import numpy as np

import pytest

from dms_ctypes import PACKAGE_DIR

DMS_SUN = os.path.join(PACKAGE_DIR, "dms_sun")

BASE = {
    "ID": '"cli_test"',
    "run_mode": '"Parameter point"',
    "sample_size": "16",
    "fixed_seed": "7",
    "max_trajectories": "4096",
    "interpolation_points": "200",
    "maximum_number_of_scatterings": "100000",
    "DM_mass": "0.3",
    "DM_spin": "0.5",
    "DM_fraction": "1.0",
    "DM_light": "true",
    "DM_interaction": '"SI"',
    "DM_isospin_conserved": "true",
    "DM_cross_section_nucleon": "1.0e-36",
    "DM_cross_section_electron": "0.0",
    "DM_form_factor": '"Contact"',
    "DM_distribution": '"SHM"',
    "DM_local_density": "0.4",
    "SHM_v0": "220.0",
    "SHM_vEscape": "544.0",
    "SHM_vObserver": "[11.1, 232.2, 7.3]",
}


def write_config(path, **over):
    keys = dict(BASE)
    keys.update(over)
    with open(path, "w") as f:
        f.write("// run configuration written by the test\n")
        for k, v in keys.items():
            if v is not None:
                f.write("%s = %s;\n" % (k, v))
    return path


def run(cfg, cwd, timeout=600):
    return subprocess.run([DMS_SUN, cfg], cwd=cwd, capture_output=True, text=True, timeout=timeout)


needs_cli = pytest.mark.skipif(not os.path.exists(DMS_SUN), reason="dms_sun not built (run __graft_entry__.build())")


@needs_cli
def test_usage_without_arguments():
    p = subprocess.run([DMS_SUN], capture_output=True, text=True, timeout=60)
    assert p.returncode == 1 and "Usage" in p.stderr


@needs_cli
@pytest.mark.parametrize("over, message", [
    ({"run_mode": '"Parameter scan"'}, "is not provided by this engine"),
    ({"run_mode": '"Spectrum"'}, "Run mode Spectrum not recognized."),
    ({"interpolation_points": "-1"}, "'interpolation_points' must be non-negative."),
    ({"sample_size": None}, "No 'sample_size' setting in configuration file."),
    ({"DM_interaction": '"SD"'}, "is not provided by this engine (SI and Dark photon are)."),
    ({"DM_light": "false"}, "DM_light = false"),
    ({"maximum_number_of_scatterings": "1.5"}, "'maximum_number_of_scatterings' must be a non-negative integer."),
    ({"snapshot_enabled": "true", "snapshot_interval": "0.5"}, "'snapshot_interval' must be a positive integer number of seconds."),
    ({"DM_interaction": '"Dark photon"', "DM_form_factor": None}, "No 'DM_form_factor' setting in configuration file."),
    ({"DM_interaction": '"Dark photon"', "DM_form_factor": '"General"'}, "No 'DM_mediator_mass' setting in configuration file."),
    ({"DM_interaction": '"Dark photon"', "DM_form_factor": '"General"', "DM_mediator_mass": "-1.0"},
     "'DM_mediator_mass' must be finite and positive for the General form factor."),
    ({"DM_interaction": '"Dark photon"', "DM_form_factor": '"Long-Range"'}, "Divergence in the IR."),
    ({"DM_interaction": '"Dark photon"', "DM_form_factor": '"Anapole"'}, "Form factor Anapole not recognized."),
    ({"DM_interaction": '"Dark photon"', "DM_cross_section_electron": None},
     "No 'DM_cross_section_electron' setting in configuration file."),
    ({"snapshot_enabled": "true", "snapshot_interval": '"often"'}, "'snapshot_interval' must be a numeric value."),
])
def test_configuration_errors(tmp_path, over, message):
    p = run(write_config(tmp_path / "bad.cfg", **over), tmp_path, timeout=60)
    assert p.returncode != 0
    assert message in p.stderr, p.stderr


@needs_cli
@pytest.mark.gpu
def test_parameter_point_run_writes_reference_outputs(tmp_path):
    p = run(write_config(tmp_path / "point.cfg"), tmp_path)
    assert p.returncode == 0, p.stderr
    for label in ("Simulation data summary", "Simulated trajectories:", "Average # of scatterings:", "Capture rate raw error",
                  "Simulation time"):
        assert label in p.stdout, p.stdout
    # progress lines at the capture milestones (src/Data_Generation.cpp:661-694)
    progress = [l for l in p.stdout.splitlines() if "captured_particle_rate[1/s]=" in l]
    assert progress and "captured_particles=0/16" in progress[0] and "100 %" in progress[-1], progress
    dirs = [d for d in os.listdir(tmp_path) if d.startswith("results_")]
    assert len(dirs) == 1
    out = tmp_path / dirs[0]
    head, rows = {}, []
    for line in open(out / "bincount.txt"):
        if line.startswith("#"):
            if "=" in line:
                k, v = line[1:].split("=", 1)
                head[k.strip()] = v.strip()
        elif line.strip():
            rows.append(line.split())
    for key in ("captured_particles", "valid_trajectories", "capture_rate_valid", "capture_rate_valid_err",
                "capture_rate_valid_CI_95_lower", "capture_rate_valid_CI_95_upper", "numerical_failure_rate",
                "average_scatterings"):
        assert key in head, key
    assert int(head["captured_particles"]) >= 16
    assert len(rows) == 2000 and all(len(r) == 9 for r in rows)
    assert sum(float(r[1]) for r in rows) > 0.0
    ev = [l.split() for l in open(out / "evaporation_times.txt") if l.strip() and not l.startswith("#")]
    assert "# format_version = 3" in open(out / "evaporation_times.txt").read()
    assert all(len(r) == 3 and float(r[2]) > 0.0 for r in ev)


@needs_cli
@pytest.mark.gpu
def test_dark_photon_parameter_point_run(tmp_path):
    # the dark photon's proton cross section follows from the electron one, and names the output
    # folder (src/Dark_Photon.cpp:130-133, 157-161; src/main.cpp:89-92)
    p = run(write_config(tmp_path / "dp.cfg", DM_interaction='"Dark photon"', DM_form_factor='"General"',
                         DM_mediator_mass="0.2", DM_mass="1.0", DM_cross_section_electron="2.0e-39",
                         sample_size="16", max_trajectories="20000"), tmp_path)
    assert p.returncode == 0, p.stderr
    dirs = [d for d in os.listdir(tmp_path) if d.startswith("results_")]
    assert len(dirs) == 1
    mu_p = 1.0 * 0.93827208816 / (1.0 + 0.93827208816)
    mu_e = 1.0 * 0.51099895e-3 / (1.0 + 0.51099895e-3)
    assert dirs[0] == "results_%f_%f" % (0.0, math.log10(2.0e-39 * (mu_p / mu_e) ** 2))
    head, rows = read_header(tmp_path / dirs[0] / "bincount.txt")
    assert int(head["captured_particles"]) >= 16 and len(rows) == 2000


@needs_cli
@pytest.mark.gpu
def test_capture_run_prints_capture_summary(tmp_path):
    p = run(write_config(tmp_path / "capture.cfg", run_mode='"Capture"', sample_size="64", max_trajectories="8192",
                         DM_mass="1.0", DM_cross_section_nucleon="1.0e-35"), tmp_path)
    assert p.returncode == 0, p.stderr
    for label in ("CAPTURE MODE summary", "Simulated trajectories:", "Total # of scatterings:", "Captured particle rate [1/s]:"):
        assert label in p.stdout, p.stdout
    assert not [d for d in os.listdir(tmp_path) if d.startswith("results_")]


def read_header(path):
    head, rows = {}, []
    for line in open(path):
        if line.startswith("#"):
            if "=" in line:
                k, v = line[1:].split("=", 1)
                head[k.strip()] = v.strip()
        elif line.strip():
            rows.append(line.split())
    return head, rows


@needs_cli
@pytest.mark.gpu
def test_snapshot_reports_during_a_parameter_point_run(tmp_path):
    # a run of a few seconds (a million trajectories at the replay point) with a report a second
    p = run(write_config(tmp_path / "snap.cfg", sample_size="1000000000", max_trajectories="1000000",
                         maximum_number_of_scatterings="1000000", snapshot_enabled="true", snapshot_interval="1"), tmp_path)
    assert p.returncode == 0, p.stderr
    out = tmp_path / [d for d in os.listdir(tmp_path) if d.startswith("results_")][0]
    final, _ = read_header(out / "bincount.txt")
    seconds = float(final["simulation_time_seconds"])
    names = sorted(os.listdir(out / "snapshot"))
    reports = sorted((int(n[len("snapshot_"):-len("s.txt")]) for n in names if n.endswith("s.txt") and "_evap" not in n))
    assert reports == list(range(1, int(seconds) + 1)), (reports, seconds)
    assert len(reports) >= 2, seconds
    assert not [n for n in names if ".tmp." in n]
    final_events = {}
    for l in open(out / "evaporation_times.txt"):
        if l.strip() and not l.startswith("#"):
            r = l.split()
            final_events[int(r[1])] = r[2]
    totals, assigned = [], {}
    for t in reports:
        head, rows = read_header(out / "snapshot" / ("snapshot_%ds.txt" % t))
        if head["snapshot_status"] == "missed_writer_delay":
            continue
        assert head["snapshot_status"] == "merged" and head["snapshot_target_wall_time_s"] == str(t)
        assert head["snapshot_interval_s"] == "1.000"
        for key in ("capture_rate_raw", "capture_rate_valid_CI_95_upper", "valid_trajectories", "numerical_failures"):
            assert key in head
        assert len(rows) == 2000 and all(len(r) == 9 for r in rows)
        totals.append(int(head["total_trajectories"]))
        ev_head, ev_rows = read_header(out / "snapshot" / ("snapshot_%ds_evaporation_times.txt" % t))
        assert ev_head["format_version"] == "3" and ev_head["DIAGNOSTIC_ONLY"] == "1"
        lifetimes = [float(r[2]) for r in ev_rows]
        assert lifetimes == sorted(lifetimes)
        for r in ev_rows:
            assert int(r[1]) not in assigned     # each event in one report only
            assigned[int(r[1])] = r[2]
    assert totals == sorted(totals) and totals
    assert totals[-1] <= int(final["total_trajectories"])
    assert all(final_events.get(i) == v for i, v in assigned.items())


@needs_cli
@pytest.mark.gpu
def test_full_size_parameter_point_matches_one_launch(tmp_path):
    """The Parameter-point configuration at its full size (run until 8192 captures, 1000 x 1000
    grid, scatter cap 1e6, seed 7) through dms_sun, against the same trajectory ids in one
    launch through the C ABI: the driver's rounds must not change any count (results are keyed
    by trajectory id), and the file's invariants must hold."""
    import sys
    sys.path.insert(0, PACKAGE_DIR)
    import dms_b200
    p = run(write_config(tmp_path / "full.cfg", sample_size="8192", max_trajectories="0", interpolation_points="1000",
                         maximum_number_of_scatterings="1000000", fixed_seed="7"), tmp_path)
    assert p.returncode == 0, p.stderr
    out = tmp_path / [d for d in os.listdir(tmp_path) if d.startswith("results_")][0]
    head, rows = read_header(out / "bincount.txt")
    total, captured = int(head["total_trajectories"]), int(head["captured_particles"])
    valid, unresolved = int(head["valid_trajectories"]), int(head["unresolved_not_captured_trajectories"])
    assert captured >= 8192 and valid + unresolved == total and valid >= captured
    assert abs(float(head["capture_rate"]) - captured / total) < 1e-8
    assert all(float(x) >= 0.0 for r in rows for x in r[1:])
    ev = [l.split() for l in open(out / "evaporation_times.txt") if l.strip() and not l.startswith("#")]
    lifetimes = [float(r[2]) for r in ev]
    assert lifetimes == sorted(lifetimes) and 0 < len(ev) <= captured
    with dms_b200.Engine(0) as e:
        pid = e.add_point(dms_b200.point_params(0.3, 1e-36, interpolation_points=1000))
        e.run([(pid, 0, total)], dms_b200.run_opts(seed=7, max_scatterings=10 ** 6, time_limit_s=600.0))
        r = e.results(pid)
    c = r["counters"]
    assert c["trajectories"] == total and c["captured"] == captured
    assert c["total_scatterings"] == int(head["total_scatterings"])
    assert c["captured"] + c["completed_outward_escapes"] == valid
    assert c["numerical_failures"] == int(head["numerical_failures"])
    assert sorted(int(x[1]) for x in ev) == sorted(r["events"]["trajectory_id"].tolist())
    cap_dt = np.array([float(x[1]) for x in rows])
    assert np.allclose(cap_dt, r["histograms"][0], rtol=1e-9, atol=0)
