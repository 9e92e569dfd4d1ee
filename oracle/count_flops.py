"""Algorithmic FP64 operations per unit of work, from the op-counting build of the oracle
(oracle/liboracle_ops.so: the same C source with every double replaced by a counting type).

Measurement infrastructure: bench.py's roofline divides these per-unit counts, times the
engine's own work counters, by the kernel time.  Units: one RK45 attempt, one accepted free
step (its bookkeeping, optical depth and bincount beyond the attempt), one scattering (with
the segment start that follows it), one trajectory (initial conditions, Kepler shifts,
classification).  Every class of operation counts one (add, mul, div, sqrt, exp/erf/log1p).

Run:  make -C oracle && python oracle/count_flops.py [trajectories]
"""
import ctypes
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "tests"))
import dms_ctypes  # noqa: E402

UNITS = ["RK45 attempt", "accepted step", "scattering", "trajectory"]
CLASSES = ["add", "mul", "div", "sqrt", "transcendental"]


def main():
    n = int(sys.argv[1]) if len(sys.argv) > 1 else 2000
    dms_ctypes.ORACLE_LIB = os.path.join(HERE, "liboracle_ops.so")
    o = dms_ctypes.Oracle()
    o.lib.dms_opcount_get.argtypes = [ctypes.c_void_p]
    o.lib.dms_opcount_reset.argtypes = []
    # the bench workload: the Parameter-point point, seed 7, normal mode, scatter cap 1e6
    o.set_point(dms_ctypes.point_params(0.3, 1e-36, interpolation_points=1000))
    o.lib.dms_opcount_reset()
    o.run_records(7, 0, 0, n, capture_mode=False, max_scatterings=10 ** 6)
    out = (ctypes.c_uint64 * 24)()
    o.lib.dms_opcount_get(out)
    ops = [[out[5 * p + c] for c in range(5)] for p in range(4)]
    units = [out[20 + k] for k in range(4)]
    print("%d trajectories of m = 0.3 GeV, sigma = 1e-36 cm^2, seed 7" % n)
    for p in range(4):
        total = sum(ops[p])
        per = total / units[p] if units[p] else float("nan")
        detail = ", ".join("%s %.1f" % (CLASSES[c], ops[p][c] / units[p]) for c in range(5)) if units[p] else ""
        print("%-14s units %10d  FP64 ops per unit %8.1f  (%s)" % (UNITS[p], units[p], per, detail))


if __name__ == "__main__":
    main()
