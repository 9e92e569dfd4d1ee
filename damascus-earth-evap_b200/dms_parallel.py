"""Multi-GPU sharding of a job and its single end-of-run exchange (one process per GPU).

Trajectories are independent and every draw is keyed by (seed, point, trajectory id), so a job
shards by trajectory-id range with no collective on the data path: the union of the ranks'
ranges is the same set of trajectories, with the same draws, as a one-GPU run.  The only
exchange is at the end and replaces Perform_MPI_Reductions (src/Data_Generation.cpp:974-1210):
a sum of the per-point counters and histograms, and a gather of the evaporation events.

With the "nccl" backend the exchange runs over NVLink; with "gloo" it runs on the CPU (the
tests use gloo with two processes).  Result dictionaries are those of
dms_b200.Engine.results()."""
import numpy as np

COUNTER_KEYS = ("trajectories", "free", "reflected", "captured", "completed_outward_escapes", "complete_evaporation",
                "censored_captured", "invalid_survival", "initial_shift_failures", "final_reflection_shift_failures",
                "numerical_failures", "computational_truncations", "total_scatterings", "rk_steps", "events_dropped",
                "rk_attempts", "unfinished_trajectories", "unfinished_scatterings", "unfinished_rk_steps",
                "unfinished_rk_attempts")
EVENT_DTYPE = [("trajectory_id", np.uint64), ("lifetime_unbinding", np.float64)]


def shard(first, count, world, rank):
    """Contiguous share of trajectory ids [first, first + count) for `rank` of `world`: the
    remainder goes to the lowest ranks, so shares differ by at most one trajectory."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d outside a world of %d" % (rank, world))
    base, extra = divmod(count, world)
    start = first + rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def reduce_results(res, device="cpu", group=None):
    """Sums counters and histograms over all ranks and gathers the evaporation events (in
    rank order).  Every rank receives the combined result."""
    import torch
    import torch.distributed as dist

    c = res["counters"]
    counters = torch.tensor([int(c[k]) for k in COUNTER_KEYS] + [int(x) for x in c["reasons"]], dtype=torch.int64,
                            device=device)
    hist = torch.as_tensor(np.ascontiguousarray(res["histograms"], dtype=np.float64)).to(device)
    dist.all_reduce(counters, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(hist, op=dist.ReduceOp.SUM, group=group)

    ev = np.ascontiguousarray(res["events"]).astype(EVENT_DTYPE, copy=False)
    world = dist.get_world_size(group)
    n = torch.tensor([len(ev)], dtype=torch.int64, device=device)
    sizes = [torch.zeros(1, dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    sizes = [int(s.item()) for s in sizes]
    width = max(max(sizes), 1)
    # trajectory id and lifetime travel as two float64 columns; ids are exact below 2^53
    packed = np.zeros((width, 2), dtype=np.float64)
    packed[:len(ev), 0] = ev["trajectory_id"].astype(np.float64)
    packed[:len(ev), 1] = ev["lifetime_unbinding"]
    mine = torch.as_tensor(packed).to(device)
    parts = [torch.zeros_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    rows = np.concatenate([p.cpu().numpy()[:k] for p, k in zip(parts, sizes)]) if sum(sizes) else np.zeros((0, 2))
    events = np.zeros(len(rows), dtype=EVENT_DTYPE)
    events["trajectory_id"] = rows[:, 0].astype(np.uint64)
    events["lifetime_unbinding"] = rows[:, 1]

    vals = counters.cpu().tolist()
    out_counters = {k: vals[i] for i, k in enumerate(COUNTER_KEYS)}
    out_counters["reasons"] = vals[len(COUNTER_KEYS):]
    return {"counters": out_counters, "histograms": hist.cpu().numpy(), "events": events}
