"""The FP64 operation counts per unit of work that bench.py's roofline uses (FLOP_PER_* in
bench.py) against the op-counting build of the oracle (oracle/liboracle_ops.so, the oracle
source compiled with a counting double), on a sample of the same workload (CPU)."""
import ctypes
import os
import re

import pytest

import dms_ctypes

OPS_LIB = os.path.join(dms_ctypes.REPO, "oracle", "liboracle_ops.so")
BENCH = os.path.join(dms_ctypes.REPO, "bench.py")


def bench_constants():
    text = open(BENCH).read()
    m = re.search(r"FLOP_PER_ATTEMPT, FLOP_PER_STEP, FLOP_PER_SCATTER, FLOP_PER_TRAJ = ([\d.]+), ([\d.]+), ([\d.]+), ([\d.]+)", text)
    return [float(x) for x in m.groups()]


@pytest.mark.skipif(not os.path.exists(OPS_LIB), reason="op-counting oracle not built (make -C oracle)")
def test_bench_flop_model_matches_the_counted_oracle(monkeypatch):
    monkeypatch.setattr(dms_ctypes, "ORACLE_LIB", OPS_LIB)
    o = dms_ctypes.Oracle()
    o.lib.dms_opcount_get.argtypes = [ctypes.c_void_p]
    o.set_point(dms_ctypes.point_params(0.3, 1e-36, interpolation_points=1000))
    o.lib.dms_opcount_reset()
    o.run_records(7, 0, 0, 600, capture_mode=False, max_scatterings=10 ** 6)
    out = (ctypes.c_uint64 * 24)()
    o.lib.dms_opcount_get(out)
    per_unit = [sum(out[5 * p + c] for c in range(5)) / out[20 + p] for p in range(4)]
    for counted, model in zip(per_unit, bench_constants()):
        assert counted == pytest.approx(model, rel=0.05), (per_unit, bench_constants())
