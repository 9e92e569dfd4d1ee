"""Runs a CPU implementation of the trajectory Monte Carlo over many trajectory ids in parallel,
one process per host core, and aggregates the outcomes the way the reference's ensemble driver
does (simulate_one_trajectory, src/Data_Generation.cpp:745-861):

* every id counts as a trajectory and adds its scatterings;
* a captured trajectory adds its 2000-bin dt and v^2 dt histograms (and their squares) to the
  captured sums, counts as a complete evaporation when its unbinding event was observed, and
  yields an evaporation event (trajectory id + 1, lifetime) when its lifetime is valid;
* an uncaptured trajectory that ended by outward escape adds its histograms to the
  not-captured sums.

The result has the layout of dms_b200.Engine.results(), so the ensemble comparisons of
dms_stats apply to it unchanged; it also carries the per-trajectory outcome of every id
(scatterings, termination reason, flags, draws, final time, lifetime, final state) for
trajectory-by-trajectory agreement counts.

Two implementations: "reference" (the reference's own sources compiled against the shims,
oracle/_ref/libdms_ref.so) and "oracle" (the C restatement, oracle/liboracle.so).  Workers are
started with the spawn method, so a parent that already initialised CUDA is safe.  Test
infrastructure only."""
import multiprocessing as mp
import os

import numpy as np

NUM_BINS = 2000
REASON_OUTWARD_ESCAPE = 1
FLAG_CAPTURED, FLAG_EVENT_OBSERVED = 0x2, 0x4
OUTCOME_DTYPE = np.dtype([("id", "<u8"), ("nscat", "<u8"), ("draws", "<u8"), ("reason", "<u4"), ("flags", "<u4"),
                          ("final_time", "<f8"), ("lifetime", "<f8"), ("final_state", "<f8", (7,))])
EVENT_DTYPE = np.dtype([("trajectory_id", "<u8"), ("lifetime_unbinding", "<f8")])

_IMPL = None


def _init(kind, params, grid):
    global _IMPL
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    if here not in sys.path:
        sys.path.insert(0, here)
    from dms_ctypes import Oracle, Reference, point_params
    impl = Reference() if kind == "reference" else Oracle()
    impl.set_point(point_params(**params))
    if grid is not None:
        impl.set_rate_grid(grid)
    _IMPL = impl


def _work(task):
    seed, point, first, count, capture_mode, max_scatterings = task
    res = _IMPL.run_records(seed, point, first, count, capture_mode=capture_mode, max_scatterings=max_scatterings,
                            histograms=not capture_mode)
    recs = res["records"]
    out = np.zeros(count, dtype=OUTCOME_DTYPE)
    for k in range(count):
        r = recs[k]
        out[k] = (r.trajectory_id, r.number_of_scatterings, r.number_of_draws, r.termination_reason, r.flags,
                  r.final_time, r.lifetime_unbinding,
                  (r.final_time,) + tuple(r.final_position) + tuple(r.final_velocity))
    hists = np.zeros((8, NUM_BINS))
    if not capture_mode:
        hd, hv = res["hist_dt"], res["hist_v2dt"]
        cap = (out["flags"] & FLAG_CAPTURED) != 0
        esc = ~cap & (out["reason"] == REASON_OUTWARD_ESCAPE)
        for sel, base in ((cap, 0), (esc, 2)):
            if np.any(sel):
                hists[base + 0] = hd[sel].sum(axis=0)
                hists[base + 1] = hv[sel].sum(axis=0)
                hists[base + 4] = (hd[sel] ** 2).sum(axis=0)
                hists[base + 5] = (hv[sel] ** 2).sum(axis=0)
    return first, out, hists


def run_ensemble(kind, params, seed, first, count, capture_mode=False, max_scatterings=10 ** 6, grid=None,
                 workers=None, chunk=128, point=0):
    """Runs ids [first, first + count) of one point through `kind` ("reference" or "oracle") on
    `workers` processes (default: every host core) and returns the aggregate (counters,
    histograms, events) with the per-trajectory `outcomes` sorted by id.  `grid` (oracle only)
    replaces the oracle's own rate grid.  `point` is the point index of the draw streams, which
    are keyed by (seed, point): it must be the engine's point id for a trajectory-by-trajectory
    comparison."""
    workers = workers or os.cpu_count() or 1
    tasks = [(seed, point, s, min(chunk, first + count - s), capture_mode, max_scatterings)
             for s in range(first, first + count, chunk)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers, initializer=_init, initargs=(kind, params, grid)) as pool:
        parts = pool.map(_work, tasks, chunksize=1)
    parts.sort(key=lambda p: p[0])
    outcomes = np.concatenate([p[1] for p in parts])
    hists = np.sum([p[2] for p in parts], axis=0)
    captured = (outcomes["flags"] & FLAG_CAPTURED) != 0
    observed = captured & ((outcomes["flags"] & FLAG_EVENT_OBSERVED) != 0)
    escaped = ~captured & (outcomes["reason"] == REASON_OUTWARD_ESCAPE)
    ev = captured & (outcomes["lifetime"] >= 0.0) if not capture_mode else np.zeros(len(outcomes), dtype=bool)
    events = np.zeros(int(ev.sum()), dtype=EVENT_DTYPE)
    events["trajectory_id"] = outcomes["id"][ev] + 1
    events["lifetime_unbinding"] = outcomes["lifetime"][ev]
    counters = {
        "trajectories": int(len(outcomes)),
        "total_scatterings": int(outcomes["nscat"].sum()),
        "captured": int(captured.sum()),
        "complete_evaporation": int(observed.sum()) if not capture_mode else 0,
        "completed_outward_escapes": int(escaped.sum()),
    }
    return {"counters": counters, "histograms": hists, "events": events, "outcomes": outcomes}
