"""The FP64 kernel's tail forms against its busy-warp forms (B200 required).

A trajectory's free steps take different code paths depending on its warp and block:
* while the work queue still has items: the RK45 stages as one loop and the optical-depth
  piece rates looked up one after another by the lane itself;
* once its block has seen the queue drained: the stages written out, and, in a warp with at most
  16 attempting lanes, the attempt computed by the lane and an idle lane of its warp (stages
  0/2/4 and 1/3/5), the piece rates of every finished step by the warp's lanes in rounds of
  32 lookups, and the next step's pre-step rate taken from that round instead of looked up at
  the step's head.
Every form forms each value with the same operations in the same order, so a trajectory's record
must not depend on which forms ran it.  The same 256 trajectory ids run alone (the queue drains at
once: tail forms throughout) and at the head of a 40 000-trajectory launch (busy forms until that
launch's own tail), with every record compared bit for bit.  Parameter-point configuration of the
bench (m = 0.3 GeV, sigma_n = 1e-36 cm^2, 1000 x 1000 grid, seed 7), max 1e5 scatterings."""
import json

import numpy as np
import pytest

from engine_fixtures import dms_b200, outcome, state

pytestmark = pytest.mark.gpu


def test_tail_and_busy_forms_give_the_same_records():
    with dms_b200.Engine(0) as e:
        pid = e.add_point(dms_b200.point_params(0.3, 1e-36, interpolation_points=1000))
        opts = dms_b200.run_opts(seed=7, max_scatterings=10 ** 5, time_limit_s=300.0)
        n = 256
        alone = e.run_records(pid, 0, n, opts)["records"]
        busy = e.run_records(pid, 0, 40000, opts)["records"]
        a = [outcome(alone[i]) for i in range(n)]
        b = [outcome(busy[i]) for i in range(n)]
        sa = np.array([state(alone[i]) for i in range(n)])
        sb = np.array([state(busy[i]) for i in range(n)])
        differ = [i for i in range(n) if a[i] != b[i] or not np.array_equal(sa[i].view(np.int64), sb[i].view(np.int64))]
        report = {"trajectories": n, "scatterings": int(sum(x[0] for x in a)), "differing": differ[:20]}
        print(json.dumps(report))
        assert sum(x[0] for x in a) > 0
        assert not differ, report
