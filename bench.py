#!/usr/bin/env python
"""Benchmark of the trajectory engine: scatterings/s (and trajectories/s) on B200.

Workload (one "step"): the Parameter-point evaporation configuration -- SI contact,
m_DM = 0.3 GeV, sigma_n = 1e-36 cm^2, AGSS09, Standard Halo Model (v0 = 220, v_esc = 544,
v_sun = (11.1, 232.2, 7.3) km/s), 1000 x 1000 rate grid, max 1e6 scatterings, seed 7 -- run
over one batch of TRAJECTORIES trajectory ids per GPU (enough for the 8192 captured particles
of the configuration's sample_size; the captured count of every step is checked).  Each step
uses fresh trajectory ids.  Inputs are generated on the device from the Philox draw stream, so
"inputs resident" means the solar tables and rate grid; the per-step host input is the work
range.  The per-lane histogram scratch (2.4 GB) exceeds L2, and L2 is additionally flushed
between steps.

Arms:
  default            the CUDA engine through its C ABI (libdms_cuda.so)
  --impl reference   the reference's own CPU implementation of the path (oracle/_ref: the
                     reference sources compiled against restated third-party shims), all host
                     cores, bounded per-step samples of the same workload
"""
import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PACKAGE_DIR = os.path.join(REPO, "damascus-earth-evap_b200")
sys.path.insert(0, PACKAGE_DIR)
sys.path.insert(0, os.path.join(REPO, "tests"))

MASS_GEV, SIGMA_CM2, GRID_N, SEED, MAX_SCAT = 0.3, 1e-36, 1000, 7, 10 ** 6
TRAJECTORIES = 65536
SAMPLE_SIZE = 8192
METRIC = "scatterings/s & trajectories/s on 1 B200, batched-FP32 vs plain-FP64 form"
WORKLOAD = ("Parameter-point evaporation (config 1): SI contact m=0.3 GeV sigma_n=1e-36 cm2, AGSS09, SHM, "
            "1000x1000 rate grid, max 1e6 scatterings, seed 7; %d trajectories per GPU per step (>= 8192 captures)" % TRAJECTORIES)
# Algorithmic FP64 operations per unit of work (add, sub, mul, div, sqrt and each elementary
# function count one), counted by the instrumented oracle build (oracle/liboracle_ops.so) on
# this parameter point in Parameter-point (normal) mode: per RK45 attempt, per accepted free
# step (event reconstruction, 4-piece optical depth, bincount, energy), per scattering
# (64-channel rate sum, free-gas target velocity, kinematics) and per trajectory (initial
# conditions, Kepler shift, classification).
FLOP_PER_ATTEMPT, FLOP_PER_STEP, FLOP_PER_SCATTER, FLOP_PER_TRAJ = 214.8, 622.3, 2455.0, 3374.0
# DRAM bytes (read + write) of the FP64 trajectory kernel per trajectory of this point, from one
# ncu capture of one 65 536-trajectory batch (ids 0-65 535: 2.671 GB read + 6.777 GB written, 635
# bytes per accepted step): the lane state's local-memory traffic and the termination flush of
# the per-lane histogram rows.
TRAFFIC_PER_TRAJECTORY = (2.671374e9 + 6.777167e9) / 65536


def hbm_peak_gbs():
    """The measured HBM copy bandwidth of this pool's B200s (MEASURED_PEAKS.json, written next to
    this file by the machine's set-up), else the earlier measurement 6650 GB/s."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            peaks = json.load(f)
        for key in ("hbm_gbs", "hbm_GBs", "hbm"):
            if key in peaks and isinstance(peaks[key], (int, float)):
                return float(peaks[key]), "measured (MEASURED_PEAKS.json %s)" % key
    except (OSError, ValueError):
        pass
    return 6650.0, "fallback 6.65 TB/s (no measured peak file)"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ------------------------------------------------------------------------------------------
# clocks during the timed region
class ClockSampler:
    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None
        self.thread = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ------------------------------------------------------------------------------------------
# CPU arm: the reference build (or the C oracle port) in worker processes.  A step is the same
# set of (point slot, trajectory ids) that the GPU arm times: the draw streams are keyed by
# (seed, point, id), so both arms simulate the same trajectories.
_cpu = {}


def _cpu_init(kind):
    import dms_ctypes
    if kind == "reference":
        impl = dms_ctypes.Reference()
    else:
        impl = dms_ctypes.Oracle()
    impl.set_point(dms_ctypes.point_params(MASS_GEV, SIGMA_CM2, interpolation_points=GRID_N))
    _cpu["impl"] = impl


def _cpu_work(task):
    point, first, count = task
    res = _cpu["impl"].run_records(SEED, point, first, count, capture_mode=False, max_scatterings=MAX_SCAT)["records"]
    return count, sum(r.number_of_scatterings for r in res), sum(1 for r in res if r.flags & 0x2)


def cpu_kind():
    import dms_ctypes
    return "reference" if os.path.exists(dms_ctypes.REF_LIB) else "port"


def cpu_pool(cores):
    kind = cpu_kind()
    ctx = mp.get_context("spawn")
    pool = ctx.Pool(cores, initializer=_cpu_init, initargs=(kind,))
    return pool, kind


def step_ids(step, world=1, rank=0):
    """First trajectory id of a step's batch (the GPU arm's ids(step))."""
    return (step * world + rank) * TRAJECTORIES


def cpu_step(pool, point, first, count=TRAJECTORIES, chunk=64):
    """Runs one step's trajectory ids on every worker; returns (trajectories, scatterings,
    captured, wall seconds)."""
    tasks = [(point, f, min(chunk, first + count - f)) for f in range(first, first + count, chunk)]
    t0 = time.perf_counter()
    out = pool.map(_cpu_work, tasks, chunksize=1)
    wall = time.perf_counter() - t0
    return sum(o[0] for o in out), sum(o[1] for o in out), sum(o[2] for o in out), wall


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    t_setup = time.perf_counter()
    pool, kind = cpu_pool(cores)
    pool.map(_cpu_work, [(0, 0, 1)] * cores)  # forces initialisation of every worker
    log("reference arm: %d workers ready (%s) in %.1fs" % (cores, kind, time.perf_counter() - t_setup))
    K, W = args.steps, args.warmup
    # warm-up: the GPU arm's warm-up batches (point slot K, ids of steps 0..W-1)
    for w in range(W):
        cpu_step(pool, K, step_ids(w))
    tot_traj = tot_scat = tot_cap = 0
    tot_time = 0.0
    per_step = []
    for s in range(K):
        # timed step s: point slot s, the ids of step W + s, as the GPU arm's timed launch
        ntraj, nscat, ncap, wall = cpu_step(pool, s, step_ids(W + s))
        tot_traj += ntraj
        tot_scat += nscat
        tot_cap += ncap
        tot_time += wall
        per_step.append(wall)
    pool.close()
    pool.join()
    value = tot_scat / tot_time
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "scatterings/s", "n_gpus": args.gpus,
        "steps": K, "warmup": W, "ms_per_step": 1e3 * tot_time / max(K, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "trajectories_per_s": tot_traj / tot_time, "captured_per_s": tot_cap / tot_time,
        "same_config": True,
        "config": {"workload": WORKLOAD, "mass_gev": MASS_GEV, "sigma_cm2": SIGMA_CM2, "seed": SEED,
                   "trajectory_ids": "the GPU arm's timed steps: point slot s, ids [(W + s) %d, (W + s + 1) %d)" % (
                       TRAJECTORIES, TRAJECTORIES),
                   "l2": "n/a (CPU)"},
        "step_seconds": {"median": statistics.median(per_step), "min": min(per_step), "max": max(per_step)},
        "cpu_baseline": {"value": value, "unit": "scatterings/s", "cores": cores, "kind": kind,
                         "sample": "the %d timed steps' %d trajectory ids each, %d trajectories in total, chunks of 64 "
                                   "on %d processes" % (K, TRAJECTORIES, tot_traj, cores)},
        "e2e": {"value": value, "unit": "scatterings/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------
# engine arm
def add_results(acc, res):
    """Running sum of Engine.results() dictionaries (counters, histograms, events)."""
    import numpy as np
    if acc is None:
        return {"counters": dict(res["counters"]), "histograms": res["histograms"].copy(), "events": res["events"].copy()}
    for k, v in res["counters"].items():
        acc["counters"][k] = [a + b for a, b in zip(acc["counters"][k], v)] if k == "reasons" else acc["counters"][k] + v
    acc["histograms"] += res["histograms"]
    acc["events"] = np.concatenate([acc["events"], res["events"]])
    return acc


def run_engine_arm(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    import numpy as np
    import torch
    import torch.distributed as dist

    pool = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # spawn the CPU workers before the first GPU call
        pool, kind = cpu_pool(os.cpu_count() or 1)
    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local_rank),
                                timeout=__import__("datetime").timedelta(seconds=600))
    import dms_b200
    import dms_parallel
    import dms_stats
    engine = dms_b200.Engine(local_rank)
    params = dms_b200.point_params(MASS_GEV, SIGMA_CM2, interpolation_points=GRID_N)
    K, R = args.steps, args.repeats
    # one accumulator slot (a copy of the point) per timed step, so that the K steps of one
    # launch keep separate results; slot `solo` serves the warm-up, isolated and steady runs.
    # Slot s is point s: the draw streams are keyed by (seed, point, id).
    pids = [engine.add_point(params) for _ in range(K)]
    solo = engine.add_point(params)
    fp64, mixed = dms_b200.PRECISION_FP64, dms_b200.PRECISION_MIXED
    opts = {prec: dms_b200.run_opts(seed=SEED, capture_mode=False, max_scatterings=MAX_SCAT, time_limit_s=600.0,
                                    precision=prec) for prec in (fp64, mixed)}
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2
    peak = engine.fp64_peak_tflops()
    # the autotuner picks block size, blocks per SM, queue chunk and the warp batching of each
    # form on this point (short trial launches over fresh ids; results never depend on them)
    tuning = {}
    if args.autotune_seconds > 0:
        for prec in (fp64, mixed):
            tuned, trials = engine.autotune([(pids[0], 0, TRAJECTORIES)], opts[prec], trial_seconds=args.autotune_seconds)
            opts[prec] = tuned
            tuning["fp64" if prec == fp64 else "mixed"] = dict(dms_b200.lane_options(tuned), trials=trials)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    def ids(step):
        return step_ids(step, world, rank)

    def batch(first_step):
        return [(pids[s], ids(first_step + s), TRAJECTORIES) for s in range(K)]

    # warm-up: W isolated steps per form; the last one of each gives the isolated step time
    isolated = {}
    for prec in (fp64, mixed):
        for w in range(args.warmup):
            engine.reset_results(solo)
            engine.run([(solo, ids(w), TRAJECTORIES)], opts[prec])
            isolated[prec] = engine.last_kernel_ms()
            flush.zero_()

    def timed(prec, first_step):
        """K steps of one form in one launch: device time and per-step results."""
        for p in pids:
            engine.reset_results(p)
        clocks = ClockSampler(local_rank)
        clocks.start()
        barrier()
        engine.run(batch(first_step), opts[prec])
        barrier()
        ms = engine.last_kernel_ms()
        info = clocks.stop()
        per_step = [engine.results(p, events_capacity=1 << 16) for p in pids]
        acc = None
        for r in per_step:
            acc = add_results(acc, r)
        flush.zero_()
        return ms, acc, min(r["counters"]["captured"] for r in per_step), info

    def repeated(prec):
        """The timed launch R times on the same ids; the median launch is the reported one."""
        runs = [timed(prec, args.warmup) for _ in range(R)]
        order = sorted(range(R), key=lambda i: runs[i][0])
        med = runs[order[R // 2]]
        return med, [r[0] for r in runs]

    (dev_ms, tot, min_captured, clock_info), fp64_ms = repeated(fp64)
    if not args.no_mixed:
        (mix_ms, mix_tot, _, mix_clocks), mixed_ms = repeated(mixed)
    # e2e: the same K steps through the C ABI from the host: work ranges in, the whole launch
    # recomputed, then every step's counters, histograms and evaporation events out.  The same
    # trajectory ids as the timed launch, so that the difference to `value` is the host
    # round trip and not a different tail (a batch lasts as long as its longest trajectory)
    e2e_runs = []
    for _ in range(R):
        for p in pids:
            engine.reset_results(p)
        barrier()
        t0 = time.perf_counter()
        engine.run(batch(args.warmup), opts[fp64])
        e2e_scat = 0
        d2h_bytes = 0
        for p in pids:
            res = engine.results(p, events_capacity=1 << 16)
            e2e_scat += res["counters"]["total_scatterings"]
            d2h_bytes += 8 * 32 + res["histograms"].nbytes + 16 * len(res["events"])
        barrier()
        e2e_runs.append((time.perf_counter() - t0, e2e_scat, d2h_bytes))
        flush.zero_()
    e2e_s, e2e_scat, d2h_bytes = sorted(e2e_runs)[R // 2]
    # steady state: a queue far longer than the run, stopped by the wall-clock limit; every
    # scattering done counts, in finished and in unfinished trajectories.  Two windows of
    # different length are run and the rate is the difference quotient, which removes the
    # initial-state pre-pass and the ramp-up and ramp-down of the lanes.
    steady = {}
    if args.steady_seconds > 0:
        def window(prec, seconds):
            engine.reset_results(solo)
            o = dms_b200.run_opts(seed=SEED, capture_mode=False, max_scatterings=MAX_SCAT, time_limit_s=seconds,
                                  precision=prec)
            try:
                engine.run([(solo, 1 << 40, 1 << 23)], o)
            except dms_b200.EngineError as e:
                if "cancelled" not in str(e):
                    raise
            c = engine.results(solo, events_capacity=1)["counters"]
            # counted algorithmic FP64 operations of the work done (the FLOP model below)
            ops = (FLOP_PER_ATTEMPT * (c["rk_attempts"] + c["unfinished_rk_attempts"]) +
                   FLOP_PER_STEP * (c["rk_steps"] + c["unfinished_rk_steps"]) +
                   FLOP_PER_SCATTER * (c["total_scatterings"] + c["unfinished_scatterings"]) +
                   FLOP_PER_TRAJ * c["trajectories"])
            return (engine.last_kernel_ms(), c["total_scatterings"] + c["unfinished_scatterings"],
                    c["rk_steps"] + c["unfinished_rk_steps"], ops)
        for name, prec in (("fp64", fp64), ("mixed", mixed)):
            t1, s1, n1, f1 = window(prec, 0.5 * args.steady_seconds)
            t2, s2, n2, f2 = window(prec, 1.5 * args.steady_seconds)
            dt = (t2 - t1) * 1e-3
            steady[name] = {"scatterings_per_s": (s2 - s1) / dt, "steps_per_s": (n2 - n1) / dt,
                            "counted_tflops": (f2 - f1) / dt / 1e12, "windows_ms": [t1, t2]}
        steady["fp64"]["fp64_pipe_frac"] = steady["fp64"]["counted_tflops"] / peak if peak > 0 else None
        steady["fp64"]["fp64_pipe_frac_of"] = "measured DFMA peak of this run"
        steady["mixed_over_fp64"] = steady["mixed"]["scatterings_per_s"] / steady["fp64"]["scatterings_per_s"]

    # the multi-GPU exchange (the end-of-run merge of the shards); on one GPU it is the identity
    if world > 1:
        tot = dms_parallel.reduce_results(tot, device="cuda")
    c = tot["counters"]
    e2e_total = torch.tensor([float(e2e_scat)], dtype=torch.float64, device="cuda")
    times = torch.tensor([dev_ms, e2e_s], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(e2e_total, op=dist.ReduceOp.SUM)
        dist.all_reduce(times, op=dist.ReduceOp.MAX)
    dev_s = float(times[0]) * 1e-3
    value = float(c["total_scatterings"]) / dev_s
    traj_rate = float(c["trajectories"]) / dev_s
    e2e_value = float(e2e_total[0]) / float(times[1])
    flops = (FLOP_PER_ATTEMPT * c["rk_attempts"] + FLOP_PER_STEP * c["rk_steps"] +
             FLOP_PER_SCATTER * c["total_scatterings"] + FLOP_PER_TRAJ * c["trajectories"])
    achieved = flops / dev_s / 1e12 / max(world, 1)  # per GPU, against one GPU's peak
    grid = run_grid_measurement(engine, args.grid_seconds) if args.grid_seconds > 0 and world == 1 else None
    stress = run_stress_measurement(engine, args.stress_seconds) if args.stress_seconds > 0 and world == 1 else None
    line = None
    if rank == 0:
        def spread(xs):
            return {"median": statistics.median(xs), "min": min(xs), "max": max(xs), "runs": len(xs)}
        line = {
            "metric": METRIC, "value": value, "unit": "scatterings/s", "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": dev_ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "trajectories_per_s": traj_rate,
            "captured_per_step_min": min_captured,
            "launch_ms": spread(fp64_ms),
            "isolated_step_ms": {"fp64": isolated[fp64], "mixed": isolated[mixed]},
            "config": {"workload": WORKLOAD, "mass_gev": MASS_GEV, "sigma_cm2": SIGMA_CM2, "grid": GRID_N,
                       "trajectories_per_gpu_step": TRAJECTORIES, "seed": SEED, "precision": "fp64 (no FMA contraction)",
                       "steps_submission": "the K timed steps are K batches (one accumulator slot each, slot s = point s) "
                                           "of one persistent launch, so they share one tail; isolated_step_ms is one "
                                           "batch launched alone; the timed launch runs %d times and the median is "
                                           "reported" % R,
                       "parallelism": "trajectory ids sharded over %d GPU(s), no data-path collective; one end-of-run "
                                      "exchange of counters, histograms and events" % world,
                       "l2": "per-lane histogram scratch (2.4 GB) exceeds L2; 256 MB flush between launches"},
            "e2e": {"value": e2e_value, "unit": "scatterings/s", "h2d_bytes_per_step": 24,
                    "d2h_bytes_per_step": int(d2h_bytes / max(K, 1)),
                    "seconds": spread([r[0] for r in e2e_runs]),
                    "work": "the timed launch's trajectory ids, recomputed, host wall clock"},
            "gpu_launches": 2,
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak if peak > 0 else None,
                         "frac_of": "measured DFMA peak of this run (MEASURED_PEAKS.json holds no FP64 figure)",
                         "traffic": TRAFFIC_PER_TRAJECTORY * c["trajectories"] / max(world, 1),
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one 65536-trajectory "
                                           "batch of this point, per trajectory x trajectories of this launch",
                         "peak_source": "measured in this run: DFMA-chain kernel on all SMs (2 FLOP per FMA)",
                         "flop_model": "%.1f/attempt + %.1f/step + %.0f/scattering + %.0f/trajectory (counted)" % (
                             FLOP_PER_ATTEMPT, FLOP_PER_STEP, FLOP_PER_SCATTER, FLOP_PER_TRAJ)},
            "clocks": clock_info,
        }
        # the memory view of the same launch: its DRAM bytes over its time against the HBM copy
        # bandwidth, which shows that the kernel is not memory-bound
        hbm_peak, hbm_source = hbm_peak_gbs()
        hbm_achieved = line["roofline"]["traffic"] / dev_s / 1e9
        line["roofline"]["hbm"] = {"achieved": hbm_achieved, "peak": hbm_peak, "unit": "GB/s",
                                   "frac": hbm_achieved / hbm_peak, "peak_source": hbm_source}
        if steady:
            line["steady_state"] = steady
        if not args.no_mixed:
            mix_s = mix_ms * 1e-3
            mc = mix_tot["counters"]
            err = dms_stats.compare_runs(tot, mix_tot)
            gates = dms_stats.reference_gates(tot, mix_tot)
            line["mixed"] = {
                "value": mc["total_scatterings"] / mix_s, "unit": "scatterings/s",
                "trajectories_per_s": mc["trajectories"] / mix_s, "ms_per_step": mix_ms / K,
                "launch_ms": spread(mixed_ms),
                "speedup_vs_fp64": (mc["total_scatterings"] / mix_s) / (c["total_scatterings"] / dev_s),
                "dtype": MIXED_DTYPE,
                "error_vs_fp64": {k: err[k] for k in ("capture_fraction_rel_error", "capture_fraction_sigmas",
                                                      "radial_chi2", "radial_dof", "radial_p_value",
                                                      "radial_max_bin_deviation", "evaporation_rate_rel_error",
                                                      "mean_scatterings_rel_error")},
                "reference_gates": {k: {"pass": bool(ok), "value": v} for k, (ok, v) in gates.items()},
                "clocks": mix_clocks,
                "gpu_launches": 2,
            }
        if tuning:
            line["autotune"] = dict(tuning, note="0 = the library default; trials of %.2f s over fresh ids, scored by "
                                                 "accepted steps per second" % args.autotune_seconds)
        if grid is not None:
            line["grid_20_points"] = grid
        if stress is not None:
            line["heavy_scattering"] = stress
    engine.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        if pool is not None:
            # the reference's CPU path on the first timed steps' own trajectory ids
            n_steps = min(K, 3)
            ntraj = nscat = 0
            wall = 0.0
            for s in range(n_steps):
                t, sc, _, w = cpu_step(pool, s, step_ids(args.warmup + s))
                ntraj += t
                nscat += sc
                wall += w
            pool.close()
            pool.join()
            line["cpu_baseline"] = {"value": nscat / wall, "unit": "scatterings/s", "cores": os.cpu_count() or 1,
                                    "kind": cpu_kind(),
                                    "sample": "the trajectory ids of the first %d timed steps (%d trajectories, the same "
                                              "(point, id) draw streams as the GPU launch), %.1f s on every core" % (
                                                  n_steps, ntraj, wall)}
        print(json.dumps(line, default=float), flush=True)


MIXED_DTYPE = "f32 stages/geometry/rates + f64 state, energy at scatterings, error norm, optical depth, accumulators"


GRID_MASSES = (0.1, 0.3, 1.0, 3.0)
GRID_SIGMAS = (1e-39, 1e-38, 1e-37, 1e-36, 1e-35)
GRID_PER_POINT = 1 << 17
GRID_MAX_SCAT = 10 ** 5


def _bounded_run(engine, ranges, opts):
    """One launch stopped by its wall-clock limit; returns (kernel ms, finished)."""
    import dms_b200
    try:
        engine.run(ranges, opts)
        return engine.last_kernel_ms(), True
    except dms_b200.EngineError as e:
        if "cancelled" not in str(e):
            raise
        return engine.last_kernel_ms(), False


def run_grid_measurement(engine, seconds):
    """The 20-point mass x cross-section grid in one persistent launch per form (2^17
    trajectories per point, 2^21 in all, max 1e5 scatterings).  Its heavy points (m >= 1 GeV at
    sigma >= 1e-37 cm^2) capture particles that scatter up to the cap, so the full launch is
    hours of work; it runs for a bounded wall time and the rate counts every scattering done,
    in finished trajectories and in those the time limit left unfinished.  Per point, the mixed
    form's errors against the FP64 form are computed over the trajectories each form finished."""
    import dms_b200
    import dms_stats
    pids = [engine.add_point(dms_b200.point_params(m, s, interpolation_points=GRID_N))
            for m in GRID_MASSES for s in GRID_SIGMAS]
    out = {"workload": "20-point grid m in %s GeV x sigma_n in %s cm2, %d trajectories per point, max %d scatterings, "
                       "seed %d, one launch per form bounded to %.0f s" % (list(GRID_MASSES), list(GRID_SIGMAS),
                                                                          GRID_PER_POINT, GRID_MAX_SCAT, SEED, seconds)}
    per_form = {}
    for name, prec in (("fp64", dms_b200.PRECISION_FP64), ("mixed", dms_b200.PRECISION_MIXED)):
        for pid in pids:
            engine.reset_results(pid)
        opts = dms_b200.run_opts(seed=SEED, max_scatterings=GRID_MAX_SCAT, time_limit_s=seconds, precision=prec)
        ms, finished = _bounded_run(engine, [(pid, 0, GRID_PER_POINT) for pid in pids], opts)
        res = [engine.results(pid, events_capacity=1 << 18) for pid in pids]
        per_form[name] = res
        tot = {k: 0 for k in ("trajectories", "total_scatterings", "rk_steps", "unfinished_trajectories",
                              "unfinished_scatterings", "unfinished_rk_steps", "captured")}
        for r in res:
            for k in tot:
                tot[k] += r["counters"][k]
        scat = tot["total_scatterings"] + tot["unfinished_scatterings"]
        steps = tot["rk_steps"] + tot["unfinished_rk_steps"]
        out[name] = {"kernel_ms": ms, "finished": finished, "scatterings_per_s": scat / ms * 1e3,
                     "steps_per_s": steps / ms * 1e3, "finished_trajectories_per_s": tot["trajectories"] / ms * 1e3,
                     "counters": tot}
    out["mixed_over_fp64_scatterings_per_s"] = out["mixed"]["scatterings_per_s"] / out["fp64"]["scatterings_per_s"]
    points = []
    for k, pid in enumerate(pids):
        a, b = per_form["fp64"][k], per_form["mixed"][k]
        entry = {"mass_gev": GRID_MASSES[k // len(GRID_SIGMAS)], "sigma_cm2": GRID_SIGMAS[k % len(GRID_SIGMAS)],
                 "finished": [a["counters"]["trajectories"], b["counters"]["trajectories"]]}
        if a["counters"]["trajectories"] and b["counters"]["trajectories"]:
            e = dms_stats.compare_runs(a, b)
            entry.update({k2: e[k2] for k2 in ("capture_fraction_rel_error", "capture_fraction_sigmas", "radial_chi2",
                                               "radial_dof", "radial_p_value", "radial_max_bin_deviation",
                                               "evaporation_rate_rel_error")})
        points.append(entry)
    out["points"] = points
    out["errors_over"] = "the trajectories each form finished within its time limit (long ones are under-represented)"
    return out


def run_stress_measurement(engine, seconds):
    """The heavy-scattering point (m = 0.1 GeV, sigma_n = 1e-33 cm^2, max 1e7 scatterings, seed
    11): mean free paths far below R_sun and up to millions of scatterings per captured
    particle.  Its full run (262144 captures) is far beyond a bench; each form runs a
    2^20-trajectory launch for a bounded wall time and reports its scattering rate (finished
    and unfinished trajectories) and, among finished trajectories, the fraction cut off by the
    scattering limit."""
    import dms_b200
    pid = engine.add_point(dms_b200.point_params(0.1, 1e-33, interpolation_points=GRID_N))
    out = {"workload": "m=0.1 GeV sigma_n=1e-33 cm2, max 1e7 scatterings, seed 11, 2^20 trajectories, "
                       "one launch per form bounded to %.0f s" % seconds}
    for name, prec in (("fp64", dms_b200.PRECISION_FP64), ("mixed", dms_b200.PRECISION_MIXED)):
        engine.reset_results(pid)
        opts = dms_b200.run_opts(seed=11, max_scatterings=10 ** 7, time_limit_s=seconds, precision=prec)
        ms, _ = _bounded_run(engine, [(pid, 0, 1 << 20)], opts)
        c = engine.results(pid, events_capacity=1)["counters"]
        finished = c["trajectories"]
        out[name] = {"kernel_ms": ms,
                     "scatterings_per_s": (c["total_scatterings"] + c["unfinished_scatterings"]) / ms * 1e3,
                     "steps_per_s": (c["rk_steps"] + c["unfinished_rk_steps"]) / ms * 1e3,
                     "finished_trajectories": finished, "unfinished_trajectories": c["unfinished_trajectories"],
                     "captured": c["captured"],
                     "cutoff_fraction_of_finished": c["reasons"][5] / finished if finished else None}
    out["mixed_over_fp64_scatterings_per_s"] = out["mixed"]["scatterings_per_s"] / out["fp64"]["scatterings_per_s"]
    return out


def run_grid(args):
    import dms_b200
    with dms_b200.Engine(0) as engine:
        print(json.dumps(run_grid_measurement(engine, args.grid_only_seconds), default=float), flush=True)


def run_stress(args):
    import dms_b200
    with dms_b200.Engine(0) as engine:
        print(json.dumps(run_stress_measurement(engine, args.stress_only_seconds), default=float), flush=True)


def run_profile_case(args):
    """One trajectory launch for a profiler (no timing): `single` runs trajectory id 1612 alone
    (the longest of ids 0..16383 of this point, 38944 accepted steps in the FP64 form: the
    per-lane latency of the tail), `saturated` runs 2^19 trajectories (about seven per resident
    lane, with the batch's tail), `steady` runs a queue of 2^21 trajectories that every lane
    leaves after 1024 loop iterations (the steady state without a tail; the stop is the same in
    every profiler pass), `step` runs one bench step (65536 trajectories)."""
    import dms_b200
    prec = dms_b200.PRECISION_MIXED if args.precision == "mixed" else dms_b200.PRECISION_FP64
    engine = dms_b200.Engine(0)
    pid = engine.add_point(dms_b200.point_params(MASS_GEV, SIGMA_CM2, interpolation_points=GRID_N))
    budget = 1024 if args.profile_case == "steady" else 0
    opts = dms_b200.run_opts(seed=SEED, capture_mode=False, max_scatterings=MAX_SCAT, time_limit_s=300.0, precision=prec,
                             iteration_budget=budget)
    first, count = {"single": (1612, 1), "saturated": (0, 1 << 19), "steady": (0, 1 << 21),
                    "step": (0, TRAJECTORIES)}[args.profile_case]
    try:
        engine.run([(pid, first, count)], opts)
    except dms_b200.EngineError as e:
        if not budget or "budget" not in str(e):
            raise
    c = engine.results(pid, events_capacity=1)["counters"]
    print(json.dumps({"profile_case": args.profile_case, "precision": args.precision, "kernel_ms": engine.last_kernel_ms(),
                      "trajectories": c["trajectories"], "rk_steps": c["rk_steps"] + c["unfinished_rk_steps"],
                      "rk_attempts": c["rk_attempts"] + c["unfinished_rk_attempts"],
                      "scatterings": c["total_scatterings"] + c["unfinished_scatterings"]}), flush=True)
    engine.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision measurement")
    ap.add_argument("--steady-seconds", type=float, default=2.0,
                    help="length of the steady-state measurement per form (0 skips it)")
    ap.add_argument("--repeats", type=int, default=3, help="runs of the timed launch and of the e2e leg (median reported)")
    ap.add_argument("--autotune-seconds", type=float, default=0.2,
                    help="trial length of the launch autotuner run before the timed launches (0 skips it)")
    ap.add_argument("--grid-seconds", type=float, default=20.0,
                    help="bounded 20-point grid launch per form inside the bench line (0 skips it)")
    ap.add_argument("--stress-seconds", type=float, default=10.0,
                    help="bounded heavy-scattering launch per form inside the bench line (0 skips it)")
    ap.add_argument("--profile-case", choices=["single", "saturated", "steady", "step"],
                    help="run one trajectory launch for a profiler and exit")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64", help="form used by --profile-case")
    ap.add_argument("--grid-only-seconds", type=float, default=0.0,
                    help="run only the 20-point grid launch, this many seconds per form")
    ap.add_argument("--stress-only-seconds", type=float, default=0.0,
                    help="run only the heavy-scattering point, this many seconds per form")
    args = ap.parse_args()
    args.repeats = max(1, args.repeats)
    if args.grid_only_seconds > 0:
        run_grid(args)
    elif args.stress_only_seconds > 0:
        run_stress(args)
    elif args.profile_case:
        run_profile_case(args)
    elif args.impl == "reference":
        run_reference_arm(args)
    else:
        run_engine_arm(args)


if __name__ == "__main__":
    main()
