"""Python binding of the engine's C ABI (include/dms.h) through ctypes.

The engine is libdms_cuda.so in this directory (built by `make -C damascus-earth-evap_b200`).
There is no CPU fallback: loading fails loudly when the library or a CUDA device is missing.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the in-tree engine library; DMS_LIBRARY names another build of it
LIBRARY = os.environ.get("DMS_LIBRARY", os.path.join(HERE, "libdms_cuda.so"))
SOLAR_MODEL = os.path.join(HERE, "data", "model_agss09.dat")

NUM_BINS = 2000
NUM_COUNTERS = 32
NUM_HISTS = 8
COUNTER_NAMES = {0: "trajectories", 1: "free", 2: "reflected", 3: "captured", 4: "completed_outward_escapes",
                 5: "complete_evaporation", 6: "censored_captured", 7: "invalid_survival", 8: "initial_shift_failures",
                 9: "final_reflection_shift_failures", 10: "numerical_failures", 11: "computational_truncations",
                 12: "total_scatterings", 13: "rk_steps", 14: "events_dropped", 15: "rk_attempts",
                 27: "unfinished_trajectories", 28: "unfinished_scatterings", 29: "unfinished_rk_steps",
                 30: "unfinished_rk_attempts", 31: "reflections_dropped"}
REASON_BASE = 16
HIST_NAMES = ["captured_dt", "captured_v2dt", "not_captured_dt", "not_captured_v2dt", "captured_dt_sq",
              "captured_v2dt_sq", "not_captured_dt_sq", "not_captured_v2dt_sq"]
ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "I/O error", -4: "no solar model", -5: "no such point",
          -6: "capacity", -7: "iteration budget exhausted", -8: "cancelled", -9: "bad state"}


class TrajRecord(ctypes.Structure):
    _fields_ = [("trajectory_id", ctypes.c_uint64), ("number_of_scatterings", ctypes.c_uint64),
                ("number_of_draws", ctypes.c_uint64), ("point", ctypes.c_uint32),
                ("termination_reason", ctypes.c_uint32), ("flags", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("initial_time", ctypes.c_double), ("initial_position", ctypes.c_double * 3),
                ("initial_velocity", ctypes.c_double * 3), ("final_time", ctypes.c_double),
                ("final_position", ctypes.c_double * 3), ("final_velocity", ctypes.c_double * 3),
                ("t_capture", ctypes.c_double), ("t_last_bound", ctypes.c_double),
                ("t_final_unbinding_scatter", ctypes.c_double), ("t_boundary_escape", ctypes.c_double),
                ("t_termination", ctypes.c_double), ("max_free_energy_drift_eV", ctypes.c_double),
                ("max_free_energy_drift_rel", ctypes.c_double), ("lifetime_unbinding", ctypes.c_double)]


class PointParams(ctypes.Structure):
    _fields_ = [("mass_gev", ctypes.c_double), ("sigma_p_cm2", ctypes.c_double), ("sigma_e_cm2", ctypes.c_double),
                ("fn_over_fp", ctypes.c_double), ("halo_v0_kms", ctypes.c_double), ("halo_vesc_kms", ctypes.c_double),
                ("halo_vobs_kms", ctypes.c_double * 3), ("interpolation_points", ctypes.c_uint32),
                ("interaction", ctypes.c_uint32), ("mediator_mass_mev", ctypes.c_double)]


INTERACTION_SI = 0
INTERACTION_DARK_PHOTON_CONTACT = 1
INTERACTION_DARK_PHOTON_GENERAL = 2


class RunOpts(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint32), ("capture_mode", ctypes.c_int32), ("max_scatterings", ctypes.c_uint64),
                ("max_free_steps", ctypes.c_uint64), ("boundary_radius_rsun", ctypes.c_double),
                ("precision", ctypes.c_int32), ("threads_per_block", ctypes.c_uint32),
                ("blocks_per_sm", ctypes.c_uint32), ("queue_chunk", ctypes.c_uint32),
                ("iteration_budget", ctypes.c_uint64), ("time_limit_s", ctypes.c_double),
                ("max_trajectory_wall_time_s", ctypes.c_double), ("scatter_batch", ctypes.c_uint32),
                ("scatter_wait", ctypes.c_uint32), ("final_batch", ctypes.c_uint32), ("final_wait", ctypes.c_uint32)]

LANE_OPTION_NAMES = ("threads_per_block", "blocks_per_sm", "queue_chunk", "scatter_batch", "scatter_wait", "final_batch",
                     "final_wait")


class WorkRange(ctypes.Structure):
    _fields_ = [("point_id", ctypes.c_int32), ("reserved", ctypes.c_uint32), ("first_trajectory", ctypes.c_uint64),
                ("count", ctypes.c_uint64)]


class EvaporationEvent(ctypes.Structure):
    _fields_ = [("trajectory_id", ctypes.c_uint64), ("lifetime_unbinding", ctypes.c_double)]


# numpy view of dms_evaporation_event
EVENT_DTYPE = np.dtype([("trajectory_id", np.uint64), ("lifetime_unbinding", np.float64)])


class Reflection(ctypes.Structure):
    _fields_ = [("trajectory_id", ctypes.c_uint64), ("speed_kms", ctypes.c_double), ("cos_sun_velocity", ctypes.c_double)]


class PointResults(ctypes.Structure):
    _fields_ = [("counters", ctypes.c_uint64 * NUM_COUNTERS), ("histograms", ctypes.POINTER(ctypes.c_double)),
                ("events", ctypes.POINTER(EvaporationEvent)), ("events_capacity", ctypes.c_uint64),
                ("events_count", ctypes.c_uint64), ("reflections", ctypes.POINTER(Reflection)),
                ("reflections_capacity", ctypes.c_uint64), ("reflections_count", ctypes.c_uint64)]


class Progress(ctypes.Structure):
    _fields_ = [("running", ctypes.c_int32), ("reserved", ctypes.c_int32), ("total", ctypes.c_uint64),
                ("dispatched", ctypes.c_uint64), ("elapsed_s", ctypes.c_double)]


# int (*dms_progress_fn)(dms_ctx*, void*)
PROGRESS_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p)


class GenerateOpts(ctypes.Structure):
    _fields_ = [("sample_size", ctypes.c_uint32), ("max_trajectories", ctypes.c_uint32), ("seed", ctypes.c_uint32),
                ("capture_mode", ctypes.c_int32), ("max_scatterings", ctypes.c_uint64),
                ("boundary_radius_rsun", ctypes.c_double), ("sigma_p_cm2", ctypes.c_double),
                ("round_capacity", ctypes.c_uint64), ("time_limit_s", ctypes.c_double),
                ("max_trajectory_wall_time_s", ctypes.c_double), ("threads_per_block", ctypes.c_uint32),
                ("blocks_per_sm", ctypes.c_uint32), ("snapshot_dir", ctypes.c_char_p),
                ("snapshot_interval_s", ctypes.c_double), ("snapshot_mass_gev", ctypes.c_double),
                ("snapshot_sigma_cm2", ctypes.c_double), ("max_free_steps", ctypes.c_uint64),
                ("print_progress", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class GenerateSummary(ctypes.Structure):
    _fields_ = [("counters", ctypes.c_uint64 * NUM_COUNTERS), ("rounds", ctypes.c_uint64),
                ("final_round_trajectories", ctypes.c_uint64), ("capture_target_overshoot", ctypes.c_uint64),
                ("sync_interval", ctypes.c_uint64), ("next_trajectory", ctypes.c_uint64),
                ("early_stop_reason", ctypes.c_int32), ("reserved", ctypes.c_int32), ("computing_time_s", ctypes.c_double)]


STOP_NAMES = {0: "none", 1: "max_trajectories_reached", 2: "capture_target_not_reached",
              3: "initial_shift_failure_fraction_exceeded", 4: "invalid_trajectory_fraction_exceeded"}


class ReflectionSpectrum(ctypes.Structure):
    _fields_ = [("trajectories", ctypes.c_uint64), ("reflections", ctypes.c_uint64), ("reflection_ratio", ctypes.c_double),
                ("entering_rate_per_s", ctypes.c_double), ("reflection_rate_per_s", ctypes.c_double),
                ("distance_au", ctypes.c_double), ("flux_per_s_cm2", ctypes.c_double), ("speed_min_kms", ctypes.c_double),
                ("speed_max_kms", ctypes.c_double), ("mean_speed_kms", ctypes.c_double)]


def point_params(mass_gev, sigma_p_cm2, sigma_e_cm2=1e-80, interpolation_points=1000, v0=220.0, vesc=544.0,
                 vobs=(11.1, 232.2, 7.3), fn_over_fp=1.0, interaction=INTERACTION_SI, mediator_mass_mev=0.0):
    """A point in low-mass mode with the Standard Halo Model of the reference configs: SI contact by
    default, or a dark photon (contact or General with mediator_mass_mev) driven by sigma_e_cm2."""
    return PointParams(mass_gev, sigma_p_cm2, sigma_e_cm2, fn_over_fp, v0, vesc, (ctypes.c_double * 3)(*vobs),
                       interpolation_points, interaction, mediator_mass_mev)


_lib = None


def library():
    """Loads libdms_cuda.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBRARY):
        raise RuntimeError("libdms_cuda.so not built: run `make -C %s`" % HERE)
    lib = ctypes.CDLL(LIBRARY)
    c = ctypes
    vp = c.c_void_p
    lib.dms_create.argtypes = [c.POINTER(vp), c.c_int]
    lib.dms_destroy.argtypes = [vp]
    lib.dms_last_error.argtypes = [vp]
    lib.dms_last_error.restype = c.c_char_p
    lib.dms_cancel.argtypes = [vp]
    lib.dms_load_solar_model.argtypes = [vp, c.c_char_p]
    lib.dms_solar_table.argtypes = [vp, c.c_int, vp, c.c_size_t]
    lib.dms_add_point.argtypes = [vp, c.POINTER(PointParams), c.POINTER(c.c_int)]
    lib.dms_num_points.argtypes = [vp]
    lib.dms_set_rate_grid.argtypes = [vp, c.c_int, vp, c.c_uint32]
    lib.dms_get_rate_grid.argtypes = [vp, c.c_int, vp, c.c_uint32]
    lib.dms_rate.argtypes = [vp, c.c_int, c.c_int, vp, vp, vp, c.c_size_t]
    lib.dms_default_run_opts.argtypes = [c.POINTER(RunOpts)]
    lib.dms_default_run_opts.restype = None
    lib.dms_run.argtypes = [vp, c.POINTER(RunOpts), c.POINTER(WorkRange), c.c_int]
    lib.dms_autotune.argtypes = [vp, c.POINTER(RunOpts), c.POINTER(WorkRange), c.c_int, c.c_double, c.POINTER(RunOpts),
                                 c.POINTER(c.c_int)]
    lib.dms_run_records.argtypes = [vp, c.POINTER(RunOpts), c.c_int, c.c_uint64, c.c_uint64, c.POINTER(TrajRecord), vp, vp]
    lib.dms_run_records_noalloc.argtypes = [vp, c.POINTER(RunOpts), c.c_int, c.c_uint64, c.c_uint64, vp, vp, vp]
    lib.dms_get_results.argtypes = [vp, c.c_int, c.POINTER(PointResults)]
    lib.dms_reset_results.argtypes = [vp, c.c_int]
    lib.dms_num_bins.restype = c.c_int
    lib.dms_last_kernel_ms.argtypes = [vp, c.POINTER(c.c_double)]
    lib.dms_measure_fp64_peak.argtypes = [vp, c.POINTER(c.c_double)]
    lib.dms_check_certified_math.argtypes = [vp, c.c_uint64, c.c_uint64, c.POINTER(c.c_uint64)]
    lib.dms_get_reflection_spectrum.argtypes = [vp, c.c_int, c.c_uint32, c.c_uint32, c.c_double, c.POINTER(ReflectionSpectrum)]
    lib.dms_reflection_spectrum_pdf.argtypes = [vp, c.c_int, c.c_uint32, c.c_uint32, vp, c.c_size_t, vp]
    lib.dms_set_progress_callback.argtypes = [vp, PROGRESS_FN, vp, c.c_double]
    lib.dms_default_generate_opts.argtypes = [c.POINTER(GenerateOpts)]
    lib.dms_default_generate_opts.restype = None
    lib.dms_generate_data.argtypes = [vp, c.c_int, c.POINTER(GenerateOpts), c.POINTER(GenerateSummary)]
    lib.dms_write_outputs.argtypes = [vp, c.c_int, c.POINTER(GenerateSummary), c.c_double, c.c_double, c.c_char_p]
    lib.dms_peek_progress.argtypes = [vp, c.POINTER(Progress)]
    lib.dms_peek_results.argtypes = [vp, c.c_int, c.POINTER(PointResults)]
    _lib = lib
    return lib


PRECISION_FP64 = 0
PRECISION_MIXED = 1


def run_opts(seed=1, capture_mode=False, max_scatterings=10 ** 14, max_free_steps=10 ** 12, boundary_rsun=2.0,
             threads_per_block=0, blocks_per_sm=0, time_limit_s=0.0, iteration_budget=0, precision=PRECISION_FP64,
             max_trajectory_wall_time_s=0.0, queue_chunk=0, scatter_batch=0, scatter_wait=0, final_batch=0, final_wait=0):
    o = RunOpts()
    library().dms_default_run_opts(ctypes.byref(o))
    o.seed = seed
    o.capture_mode = int(bool(capture_mode))
    o.max_scatterings = max_scatterings
    o.max_free_steps = max_free_steps
    o.boundary_radius_rsun = boundary_rsun
    o.threads_per_block = threads_per_block
    o.blocks_per_sm = blocks_per_sm
    o.time_limit_s = time_limit_s
    o.iteration_budget = iteration_budget
    o.precision = precision
    o.max_trajectory_wall_time_s = max_trajectory_wall_time_s
    o.queue_chunk = queue_chunk
    o.scatter_batch, o.scatter_wait, o.final_batch, o.final_wait = scatter_batch, scatter_wait, final_batch, final_wait
    return o


def lane_options(opts):
    """The lane-scheduling fields of a RunOpts (the autotuner's knobs) as a dict."""
    return {k: int(getattr(opts, k)) for k in LANE_OPTION_NAMES}


class EngineError(RuntimeError):
    pass


class Engine:
    """One engine context on one CUDA device."""

    def __init__(self, device=0, solar_model=SOLAR_MODEL):
        self.lib = library()
        self.h = ctypes.c_void_p()
        rc = self.lib.dms_create(ctypes.byref(self.h), device)
        if rc != 0:
            raise EngineError("dms_create failed (%s): no usable CUDA device %d" % (ERRORS.get(rc, rc), device))
        if solar_model is not None:
            self._check(self.lib.dms_load_solar_model(self.h, solar_model.encode()))

    def _check(self, rc):
        if rc < 0:
            raise EngineError("%s: %s" % (ERRORS.get(rc, rc), self.lib.dms_last_error(self.h).decode()))
        return rc

    def close(self):
        if self.h:
            self.lib.dms_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solar_table(self, which):
        n = self._check(self.lib.dms_solar_table(self.h, which, None, 0))
        out = np.zeros(n)
        self._check(self.lib.dms_solar_table(self.h, which, out.ctypes.data, n))
        return out

    def add_point(self, params):
        pid = ctypes.c_int(-1)
        self._check(self.lib.dms_add_point(self.h, ctypes.byref(params), ctypes.byref(pid)))
        return pid.value

    def set_rate_grid(self, point, grid):
        g = np.ascontiguousarray(grid, dtype=np.float64)
        self._check(self.lib.dms_set_rate_grid(self.h, point, g.ctypes.data, g.shape[0]))

    def rate_grid(self, point, n):
        g = np.zeros((n, n))
        self._check(self.lib.dms_get_rate_grid(self.h, point, g.ctypes.data, n))
        return g

    def rate(self, point, r_km, v_kms, interpolated=True):
        r = np.ascontiguousarray(r_km, dtype=np.float64)
        v = np.ascontiguousarray(v_kms, dtype=np.float64)
        out = np.zeros_like(r)
        self._check(self.lib.dms_rate(self.h, point, int(interpolated), r.ctypes.data, v.ctypes.data, out.ctypes.data, r.size))
        return out

    def run(self, ranges, opts):
        """ranges: iterable of (point_id, first_trajectory, count)."""
        ranges = list(ranges)
        arr = (WorkRange * len(ranges))(*[WorkRange(p, 0, f, c) for p, f, c in ranges])
        self._check(self.lib.dms_run(self.h, ctypes.byref(opts), arr, len(ranges)))

    def autotune(self, ranges, opts, trial_seconds=0.25):
        """dms_autotune: returns (tuned RunOpts, number of trial launches)."""
        ranges = list(ranges)
        arr = (WorkRange * len(ranges))(*[WorkRange(p, 0, f, c) for p, f, c in ranges])
        tuned = RunOpts()
        n = ctypes.c_int(0)
        self._check(self.lib.dms_autotune(self.h, ctypes.byref(opts), arr, len(ranges), trial_seconds, ctypes.byref(tuned),
                                          ctypes.byref(n)))
        return tuned, n.value

    def run_records(self, point, first, count, opts, histograms=False):
        recs = (TrajRecord * count)()
        hd = np.zeros((count, NUM_BINS)) if histograms else None
        hv = np.zeros((count, NUM_BINS)) if histograms else None
        self._check(self.lib.dms_run_records(self.h, ctypes.byref(opts), point, first, count, recs,
                                             hd.ctypes.data if hd is not None else None,
                                             hv.ctypes.data if hv is not None else None))
        out = {"records": recs}
        if histograms:
            out["hist_dt"], out["hist_v2dt"] = hd, hv
        return out

    def run_records_noalloc(self, point, first, count, opts, d_records, d_hist_dt=None, d_hist_v2dt=None):
        """dms_run_records_noalloc: the same records written into caller-owned DEVICE buffers
        (integer device addresses, e.g. a torch tensor's data_ptr()); the library allocates
        nothing for the call."""
        self._check(self.lib.dms_run_records_noalloc(self.h, ctypes.byref(opts), point, first, count, d_records,
                                                     d_hist_dt, d_hist_v2dt))

    def results(self, point, events_capacity=1 << 20, reflections_capacity=0):
        """Accumulated results of a point (dms_get_results)."""
        return self._results(self.lib.dms_get_results, point, events_capacity, reflections_capacity)

    def peek_results(self, point, events_capacity=1 << 20):
        """Results of the trajectories finished so far while a launch is in flight, from inside a
        progress callback (dms_peek_results): `events` holds the published prefix."""
        return self._results(self.lib.dms_peek_results, point, events_capacity, 0)

    def peek_progress(self):
        p = Progress()
        self._check(self.lib.dms_peek_progress(self.h, ctypes.byref(p)))
        return {"running": bool(p.running), "total": int(p.total), "dispatched": int(p.dispatched),
                "elapsed_s": p.elapsed_s}

    def set_progress_callback(self, fn, interval_s=1.0):
        """Calls fn(engine) about every interval_s seconds while `run` / `run_records` wait for a
        launch, on the calling thread; a true return (or an exception) cancels the run.  None
        removes the hook."""
        if fn is None:
            self._check(self.lib.dms_set_progress_callback(self.h, PROGRESS_FN(), None, 0.0))
            self._progress = None
            return

        def hook(ctx, user):
            try:
                return 1 if fn(self) else 0
            except Exception as e:  # an exception cannot cross the C frames: cancel instead
                self.progress_error = e
                return 1
        self.progress_error = None
        self._progress = PROGRESS_FN(hook)  # kept alive while the library holds the pointer
        self._check(self.lib.dms_set_progress_callback(self.h, self._progress, None, interval_s))

    def _results(self, getter, point, events_capacity, reflections_capacity):
        res = PointResults()
        hist = np.zeros(NUM_HISTS * NUM_BINS)
        events = np.empty(events_capacity, dtype=EVENT_DTYPE)
        refl = np.zeros(reflections_capacity, dtype=[("trajectory_id", np.uint64), ("speed_kms", np.float64),
                                                      ("cos_sun_velocity", np.float64)])
        res.histograms = hist.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        res.events = events.ctypes.data_as(ctypes.POINTER(EvaporationEvent))
        res.events_capacity = events_capacity
        res.reflections = refl.ctypes.data_as(ctypes.POINTER(Reflection))
        res.reflections_capacity = reflections_capacity
        self._check(getter(self.h, point, ctypes.byref(res)))
        counters = {name: int(res.counters[k]) for k, name in COUNTER_NAMES.items()}
        counters["reasons"] = [int(res.counters[REASON_BASE + k]) for k in range(11)]
        ev = events[:min(res.events_count, events_capacity)].copy()
        out = {"counters": counters, "histograms": hist.reshape(NUM_HISTS, NUM_BINS), "events": ev,
               "reflections_count": int(res.reflections_count)}
        if reflections_capacity:
            out["reflections"] = refl[:min(res.reflections_count, reflections_capacity)]
        return out

    def generate(self, point, sample_size, max_trajectories=0, seed=0, capture_mode=False, max_scatterings=None,
                 boundary_rsun=2.0, sigma_p_cm2=1e-36, max_free_steps=0, time_limit_s=0.0):
        """Simulation_Data::Generate_Data through dms_generate_data: rounds until sample_size
        captures, the trajectory budget or a run-level fuse; returns the summary."""
        g = GenerateOpts()
        self.lib.dms_default_generate_opts(ctypes.byref(g))
        g.sample_size, g.max_trajectories, g.seed = sample_size, max_trajectories, seed
        g.capture_mode = int(bool(capture_mode))
        if max_scatterings is not None:
            g.max_scatterings = max_scatterings
        g.boundary_radius_rsun, g.sigma_p_cm2 = boundary_rsun, sigma_p_cm2
        g.max_free_steps, g.time_limit_s = max_free_steps, time_limit_s
        summary = GenerateSummary()
        self._check(self.lib.dms_generate_data(self.h, point, ctypes.byref(g), ctypes.byref(summary)))
        counters = {name: int(summary.counters[k]) for k, name in COUNTER_NAMES.items()}
        counters["reasons"] = [int(summary.counters[REASON_BASE + k]) for k in range(11)]
        return {"summary": summary, "counters": counters, "early_stop": STOP_NAMES[summary.early_stop_reason],
                "rounds": int(summary.rounds), "computing_time_s": summary.computing_time_s}

    def write_outputs(self, point, generated, mass_gev, sigma_cm2, directory):
        """Write_Output_Files: bincount.txt and evaporation_times.txt into directory."""
        self._check(self.lib.dms_write_outputs(self.h, point, ctypes.byref(generated["summary"]), mass_gev, sigma_cm2,
                                               directory.encode()))

    def reflection_spectrum(self, point, rings=1, ring=0, dm_density_gev_cm3=0.4):
        s = ReflectionSpectrum()
        self._check(self.lib.dms_get_reflection_spectrum(self.h, point, rings, ring, dm_density_gev_cm3, ctypes.byref(s)))
        return {name: getattr(s, name) for name, _ in ReflectionSpectrum._fields_}

    def reflection_pdf(self, point, u_kms, rings=1, ring=0):
        u = np.ascontiguousarray(u_kms, dtype=np.float64)
        out = np.zeros_like(u)
        self._check(self.lib.dms_reflection_spectrum_pdf(self.h, point, rings, ring, u.ctypes.data, u.size, out.ctypes.data))
        return out

    def last_kernel_ms(self):
        ms = ctypes.c_double(0.0)
        self._check(self.lib.dms_last_kernel_ms(self.h, ctypes.byref(ms)))
        return ms.value

    def fp64_peak_tflops(self):
        t = ctypes.c_double(0.0)
        self._check(self.lib.dms_measure_fp64_peak(self.h, ctypes.byref(t)))
        return t.value

    def check_certified_math(self, n, seed=1):
        """dms_check_certified_math: (div mismatches, div fallbacks, sqrt mismatches, sqrt fallbacks)."""
        counts = (ctypes.c_uint64 * 4)()
        self._check(self.lib.dms_check_certified_math(self.h, n, seed, counts))
        return tuple(int(x) for x in counts)

    def reset_results(self, point):
        self._check(self.lib.dms_reset_results(self.h, point))
