"""Multi-rank path on the CPU: trajectory-id sharding and the end-of-run exchange, with two
`gloo` processes (no GPU).  The ranks run their shards through the C oracle, so the test also
shows that sharding by trajectory id reproduces the one-process run exactly."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as tmp

from engine_fixtures import dms_b200  # noqa: F401  (puts the package on sys.path)
import dms_parallel

POINT = dict(mass_gev=0.3, sigma_p_cm2=1e-36, interpolation_points=200)
TOTAL, SEED = 48, 7


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def oracle_results(first, count):
    """Accumulated results of trajectories [first, first + count) from oracle records."""
    import dms_ctypes
    o = dms_ctypes.Oracle()
    o.set_point(dms_ctypes.point_params(POINT["mass_gev"], POINT["sigma_p_cm2"],
                                        interpolation_points=POINT["interpolation_points"]))
    out = o.run_records(SEED, 0, first, count, histograms=True) if count else None
    counters = {k: 0 for k in dms_parallel.COUNTER_KEYS}
    counters["reasons"] = [0] * 11
    hist = np.zeros((8, 2000))
    events = []
    for i in range(count):
        r = out["records"][i]
        counters["trajectories"] += 1
        counters["total_scatterings"] += r.number_of_scatterings
        counters["reasons"][r.termination_reason] += 1
        if r.flags & 0x2:
            counters["captured"] += 1
            hist[0] += out["hist_dt"][i]
            hist[4] += out["hist_dt"][i] ** 2
            if r.lifetime_unbinding >= 0:
                events.append((r.trajectory_id, r.lifetime_unbinding))
    ev = np.array(events, dtype=dms_parallel.EVENT_DTYPE)
    return {"counters": counters, "histograms": hist, "events": ev}


def worker(rank, world, port, outdir):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        first, count = dms_parallel.shard(0, TOTAL, world, rank)
        combined = dms_parallel.reduce_results(oracle_results(first, count))
        np.save(os.path.join(outdir, "hist%d.npy" % rank), combined["histograms"])
        np.save(os.path.join(outdir, "events%d.npy" % rank), combined["events"])
        c = combined["counters"]
        np.save(os.path.join(outdir, "counters%d.npy" % rank),
                np.array([c[k] for k in dms_parallel.COUNTER_KEYS] + c["reasons"], dtype=np.int64))
    finally:
        dist.destroy_process_group()


def test_shard_partitions_ids():
    for total in (0, 1, 7, 1000, 1001):
        for world in (1, 2, 3, 8):
            spans = [dms_parallel.shard(5, total, world, r) for r in range(world)]
            ids = [i for f, n in spans for i in range(f, f + n)]
            assert ids == list(range(5, 5 + total))
            assert max(n for _, n in spans) - min(n for _, n in spans) <= 1
    with pytest.raises(ValueError):
        dms_parallel.shard(0, 10, 2, 2)


def test_two_rank_gloo_exchange_matches_single_process():
    world, port = 2, free_port()
    with tempfile.TemporaryDirectory() as d:
        tmp.start_processes(worker, args=(world, port, d), nprocs=world, start_method="spawn", join=True)
        single = oracle_results(0, TOTAL)
        want_counters = [single["counters"][k] for k in dms_parallel.COUNTER_KEYS] + single["counters"]["reasons"]
        for rank in range(world):
            assert np.load(os.path.join(d, "counters%d.npy" % rank)).tolist() == want_counters
            np.testing.assert_allclose(np.load(os.path.join(d, "hist%d.npy" % rank)), single["histograms"],
                                       rtol=1e-13, atol=0)
            ev = np.load(os.path.join(d, "events%d.npy" % rank))
            assert sorted(ev["trajectory_id"].tolist()) == sorted(single["events"]["trajectory_id"].tolist())
            assert sorted(ev["lifetime_unbinding"].tolist()) == sorted(single["events"]["lifetime_unbinding"].tolist())
        assert single["counters"]["captured"] > 0
