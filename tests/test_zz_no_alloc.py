"""dms_run_records_noalloc against dms_run_records, through the C ABI (B200 required).

The no-alloc entry point runs the same FP64 trajectory kernel as dms_run_records, only with
its scratch in a fixed device array, so the tolerance is exact: every record and every
histogram bin must be byte-identical.  The output buffers are pre-filled with garbage and
three calls run back to back, so the test also checks that each call clears what the previous
one left in the shared scratch.  The file name makes pytest collect it last."""
import ctypes

import numpy as np
import pytest

from engine_fixtures import REPLAY_POINT, dms_b200

pytestmark = pytest.mark.gpu

MAX_TRAJECTORIES = 128   # DMS_NOALLOC_MAX_TRAJECTORIES in include/dms.h


@pytest.fixture(scope="module")
def engine():
    e = dms_b200.Engine(0)
    c = ctypes
    e.lib.dms_run_records_noalloc.argtypes = [c.c_void_p, c.POINTER(dms_b200.RunOpts), c.c_int, c.c_uint64, c.c_uint64,
                                              c.c_void_p, c.c_void_p, c.c_void_p]
    p = REPLAY_POINT
    pid = e.add_point(dms_b200.point_params(p["mass_gev"], p["sigma_p_cm2"], interpolation_points=p["interpolation_points"]))
    yield e, pid
    e.close()


def run_noalloc(e, pid, first, count, opts, histograms):
    import torch

    rec_bytes = ctypes.sizeof(dms_b200.TrajRecord) * count
    d_rec = torch.full((rec_bytes,), 0xAB, dtype=torch.uint8, device="cuda:0")
    shape = (count, dms_b200.NUM_BINS)
    d_hd = torch.full(shape, float("nan"), dtype=torch.float64, device="cuda:0") if histograms else None
    d_hv = torch.full(shape, -7.0, dtype=torch.float64, device="cuda:0") if histograms else None
    torch.cuda.synchronize()
    e._check(e.lib.dms_run_records_noalloc(e.h, ctypes.byref(opts), pid, first, count, d_rec.data_ptr(),
                                           d_hd.data_ptr() if histograms else None,
                                           d_hv.data_ptr() if histograms else None))
    out = {"records": d_rec.cpu().numpy().tobytes()}
    if histograms:
        out["hist_dt"], out["hist_v2dt"] = d_hd.cpu().numpy(), d_hv.cpu().numpy()
    return out


def check_same(e, pid, first, count, opts, histograms):
    got = run_noalloc(e, pid, first, count, opts, histograms)
    want = e.run_records(pid, first, count, opts, histograms=histograms)
    assert got["records"] == bytes(want["records"])
    if histograms:
        assert np.array_equal(got["hist_dt"], want["hist_dt"])
        assert np.array_equal(got["hist_v2dt"], want["hist_v2dt"])
        assert np.any(got["hist_dt"] > 0.0)


def test_noalloc_matches_run_records_back_to_back(engine):
    e, pid = engine
    normal = dms_b200.run_opts(seed=7, capture_mode=False, max_scatterings=10 ** 6, time_limit_s=120.0)
    capture = dms_b200.run_opts(seed=7, capture_mode=True, max_scatterings=10 ** 6, time_limit_s=120.0)
    check_same(e, pid, 0, MAX_TRAJECTORIES, normal, histograms=True)
    check_same(e, pid, 500, 77, capture, histograms=False)
    check_same(e, pid, 1000, 40, normal, histograms=True)


def test_noalloc_rejects_oversize_and_accepts_empty(engine):
    e, pid = engine
    opts = dms_b200.run_opts(seed=7)
    rc = e.lib.dms_run_records_noalloc(e.h, ctypes.byref(opts), pid, 0, MAX_TRAJECTORIES + 1, None, None, None)
    assert rc == -1  # DMS_ERR_INVALID_ARGUMENT
    assert "at most %d" % MAX_TRAJECTORIES in e.lib.dms_last_error(e.h).decode()
    assert e.lib.dms_run_records_noalloc(e.h, ctypes.byref(opts), pid, 0, 0, None, None, None) == 0
    bad = dms_b200.run_opts(seed=7, max_trajectory_wall_time_s=-1.0)
    assert e.lib.dms_run_records_noalloc(e.h, ctypes.byref(bad), pid, 0, 4, None, None, None) == -1
    assert "max_trajectory_wall_time_sec" in e.lib.dms_last_error(e.h).decode()
