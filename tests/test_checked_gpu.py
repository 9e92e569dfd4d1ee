"""The bounds-checked build (libdms_cuda_checked.so, -DDMS_CHECKED): every solar-table knot,
rate-grid cell, histogram bin and row, work range and scattering target index is tested on
the device, and a launch that saw one out of bounds fails with DMS_ERR_STATE.  Both kernels run
the replay, direct-rate, dark-photon and ragged-launch workloads under it, and so does the
no-alloc entry point; the FP64 records must still equal the oracle's (B200 required).  The library is loaded in a child process, since one
process holds one engine library."""
import os
import subprocess
import sys

import pytest

from dms_ctypes import PACKAGE_DIR

pytestmark = pytest.mark.gpu

CHECKED = os.path.join(PACKAGE_DIR, "libdms_cuda_checked.so")
TESTS = os.path.dirname(os.path.abspath(__file__))

CHILD = r'''
import sys
sys.path.insert(0, %(tests)r)
sys.path.insert(0, %(pkg)r)
import dms_b200
dms_b200.LIBRARY = %(lib)r
from dms_ctypes import Oracle, point_params
from engine_fixtures import outcome
o = Oracle()
with dms_b200.Engine(0) as e:
    for kw, n_grid, capture in ((dict(), 200, False), (dict(), 200, True), (dict(), 0, True),
                                (dict(sigma_e_cm2=1e-40, interaction=2, mediator_mass_mev=1.0), 200, False)):
        params = dict(mass_gev=0.3, sigma_p_cm2=1e-36, interpolation_points=n_grid)
        params.update(kw)
        o.set_point(point_params(**params))
        pid = e.add_point(dms_b200.point_params(**params))
        if n_grid:
            e.set_rate_grid(pid, o.rate_grid())
        opts = dms_b200.run_opts(seed=7, capture_mode=capture, max_scatterings=10 ** 5, time_limit_s=120.0)
        a = e.run_records(pid, 0, 256, opts, histograms=not capture)["records"]
        if n_grid:
            b = o.run_records(7, pid, 0, 256, capture_mode=capture, max_scatterings=10 ** 5)["records"]
            bad = [i for i in range(256) if outcome(a[i]) != outcome(b[i])]
            assert not bad, bad[:5]
        for prec in (dms_b200.PRECISION_FP64, dms_b200.PRECISION_MIXED):
            e.reset_results(pid)
            e.run([(pid, 0, 1), (pid, 1, 0), (pid, 1, 700), (pid, 5000, 33)],
                  dms_b200.run_opts(seed=3, capture_mode=capture, max_scatterings=10 ** 5, time_limit_s=120.0,
                                    precision=prec))
            assert e.results(pid, events_capacity=1)["counters"]["trajectories"] == 734
        if n_grid and not capture:
            import ctypes, torch
            d_rec = torch.zeros(ctypes.sizeof(dms_b200.TrajRecord) * 96, dtype=torch.uint8, device="cuda:0")
            d_hd = torch.zeros((96, dms_b200.NUM_BINS), dtype=torch.float64, device="cuda:0")
            d_hv = torch.zeros_like(d_hd)
            e.run_records_noalloc(pid, 3000, 96, opts, d_rec.data_ptr(), d_hd.data_ptr(), d_hv.data_ptr())
            torch.cuda.synchronize()
            assert d_rec.cpu().numpy().tobytes() == bytes(e.run_records(pid, 3000, 96, opts)["records"])
print("checked build: no index out of bounds")
'''


@pytest.mark.skipif(not os.path.exists(CHECKED), reason="checked library not built (make checked)")
def test_checked_build_sees_no_index_out_of_bounds():
    code = CHILD % {"tests": TESTS, "pkg": PACKAGE_DIR, "lib": CHECKED}
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-4000:]
    assert "no index out of bounds" in p.stdout
