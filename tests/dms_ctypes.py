"""ctypes layouts of the engine's C ABI (include/dms.h) and loaders for the three
implementations the tests compare: the CUDA engine, the C oracle and the reference build
of the oracle (the reference's own sources compiled against the shims in oracle/shim)."""
import ctypes
import os

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PACKAGE_DIR = os.path.join(REPO, "damascus-earth-evap_b200")
SOLAR_MODEL = os.path.join(PACKAGE_DIR, "data", "model_agss09.dat")
ORACLE_LIB = os.path.join(REPO, "oracle", "liboracle.so")
REF_LIB = os.path.join(REPO, "oracle", "_ref", "libdms_ref.so")
ENGINE_LIB = os.path.join(PACKAGE_DIR, "libdms_cuda.so")

NUM_BINS = 2000
NUM_TARGETS = 63
RSUN_KM = 6.957e5
C_KMS = 299792.458

REASON_NAMES = ["Unknown", "OutwardEscape", "Scatter", "WallTimeLimit", "MaxFreeSteps", "MaxScatterings",
                "NonFiniteState", "SpeedLimit", "NumericalFailure", "CaptureMode", "EnergyDriftEscape"]
REC_SHIFT_OK, REC_CAPTURED, REC_EVENT_OBSERVED, REC_SURVIVAL_VALID = 0x1, 0x2, 0x4, 0x8
REC_BOUNDARY_ESCAPE, REC_FREE, REC_REFLECTED, REC_REFLECT_SHIFT_OK, REC_INVALID_ESCAPE = 0x10, 0x20, 0x40, 0x80, 0x100


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


def point_params(mass_gev, sigma_p_cm2, sigma_e_cm2=1e-80, interpolation_points=1000,
                 v0=220.0, vesc=544.0, vobs=(11.1, 232.2, 7.3), fn_over_fp=1.0, interaction=INTERACTION_SI,
                 mediator_mass_mev=0.0):
    """A point with the Standard Halo Model of tests/config_unittest.cfg:78-80: SI contact by
    default, or a dark photon (contact / General) driven by sigma_e_cm2."""
    return PointParams(mass_gev, sigma_p_cm2, sigma_e_cm2, fn_over_fp, v0, vesc, (ctypes.c_double * 3)(*vobs),
                       interpolation_points, interaction, mediator_mass_mev)


def records_to_dicts(records):
    out = []
    for r in records:
        out.append({
            "id": r.trajectory_id, "nscat": r.number_of_scatterings, "draws": r.number_of_draws,
            "reason": r.termination_reason, "flags": r.flags,
            "initial": (r.initial_time, tuple(r.initial_position), tuple(r.initial_velocity)),
            "final": (r.final_time, tuple(r.final_position), tuple(r.final_velocity)),
            "t_capture": r.t_capture, "t_last_bound": r.t_last_bound,
            "t_final_unbinding": r.t_final_unbinding_scatter, "t_boundary_escape": r.t_boundary_escape,
            "t_termination": r.t_termination, "lifetime": r.lifetime_unbinding,
        })
    return out


class Oracle:
    """The C oracle (oracle/liboracle.so)."""

    def __init__(self, path=SOLAR_MODEL):
        lib = ctypes.CDLL(ORACLE_LIB)
        lib.dms_oracle_create.restype = ctypes.c_void_p
        lib.dms_oracle_create.argtypes = [ctypes.c_char_p]
        lib.dms_oracle_destroy.argtypes = [ctypes.c_void_p]
        lib.dms_oracle_set_point.argtypes = [ctypes.c_void_p, ctypes.POINTER(PointParams)]
        lib.dms_oracle_query.restype = ctypes.c_double
        lib.dms_oracle_query.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        lib.dms_oracle_num_nodes.argtypes = [ctypes.c_void_p]
        lib.dms_oracle_tables.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 6
        lib.dms_oracle_rate_grid.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.dms_oracle_set_rate_grid.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32]
        lib.dms_oracle_run_from_starts.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int,
                                                   ctypes.c_uint64, ctypes.c_double, ctypes.c_uint64, ctypes.c_uint64,
                                                   ctypes.c_void_p, ctypes.POINTER(TrajRecord), ctypes.c_void_p,
                                                   ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
        lib.dms_oracle_run_reflections.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64,
                                                   ctypes.c_double, ctypes.c_uint64, ctypes.c_uint64,
                                                   ctypes.POINTER(TrajRecord), ctypes.c_void_p]
        lib.dms_oracle_run_records.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int,
                                               ctypes.c_uint64, ctypes.c_double, ctypes.c_uint64, ctypes.c_uint64,
                                               ctypes.POINTER(TrajRecord), ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
        self.lib = lib
        self.h = lib.dms_oracle_create(path.encode())
        if not self.h:
            raise RuntimeError("oracle: cannot load solar model " + path)
        self.point_n = None

    def close(self):
        if self.h:
            self.lib.dms_oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_point(self, params):
        rc = self.lib.dms_oracle_set_point(self.h, ctypes.byref(params))
        if rc != 0:
            raise RuntimeError("oracle set_point failed %d" % rc)
        self.point_n = params.interpolation_points

    def query(self, what, a=0.0, b=0.0, c=0.0):
        return self.lib.dms_oracle_query(self.h, what, a, b, c)

    def tables(self):
        import numpy as np
        n = self.lib.dms_oracle_num_nodes(self.h)
        arrs = [np.zeros(n) for _ in range(5)] + [np.zeros(n * NUM_TARGETS)]
        self.lib.dms_oracle_tables(self.h, *[a.ctypes.data for a in arrs])
        r, gm, t, vesc2, ne, nt = arrs
        return dict(r=r, gm=gm, temperature_gev=t, vesc2=vesc2, n_e=ne, n_targets=nt.reshape(n, NUM_TARGETS))

    def rate_grid(self):
        import numpy as np
        g = np.zeros(self.point_n * self.point_n)
        self.lib.dms_oracle_rate_grid(self.h, g.ctypes.data)
        return g.reshape(self.point_n, self.point_n)

    def run_reflections(self, seed, point, first, count, max_scatterings=10**6, boundary_rsun=2.0):
        """Records and the per-trajectory reflection-spectrum sample (speed at 1 AU, cosine to the
        Sun's velocity; NaN unless a recorded reflection), Parameter-point mode."""
        import numpy as np
        recs = (TrajRecord * count)()
        out = np.zeros((count, 2))
        rc = self.lib.dms_oracle_run_reflections(self.h, seed, point, max_scatterings, boundary_rsun, first, count, recs,
                                                 out.ctypes.data)
        if rc != 0:
            raise RuntimeError("oracle run_reflections failed %d" % rc)
        return recs, out

    def run_from_starts(self, seed, point, first, starts, capture_mode=False, max_scatterings=10**6, boundary_rsun=2.0,
                        trace_capacity=0):
        """Records of ids [first, first + len(starts)) started from the given events after the
        initial Kepler shift (rows t, x, v; e.g. the reference's own), with the usual draws."""
        import numpy as np
        st = np.ascontiguousarray(starts, dtype=np.float64).reshape(-1, 7)
        count = len(st)
        recs = (TrajRecord * count)()
        tr = np.zeros((max(trace_capacity, 1), 3)) if trace_capacity else None
        tl = ctypes.c_size_t(0)
        rc = self.lib.dms_oracle_run_from_starts(self.h, seed, point, int(capture_mode), max_scatterings, boundary_rsun, first,
                                                 count, st.ctypes.data, recs, tr.ctypes.data if tr is not None else None,
                                                 trace_capacity, ctypes.byref(tl))
        if rc != 0:
            raise RuntimeError("oracle run_from_starts failed %d" % rc)
        out = {"records": recs}
        if trace_capacity:
            out["trace"] = tr[: min(tl.value, trace_capacity)]
        return out

    def set_rate_grid(self, grid):
        """Replays on a grid built elsewhere (e.g. the engine's device-built grid)."""
        import numpy as np
        g = np.ascontiguousarray(grid, dtype=np.float64).reshape(-1)
        rc = self.lib.dms_oracle_set_rate_grid(self.h, g.ctypes.data, self.point_n)
        if rc != 0:
            raise RuntimeError("oracle set_rate_grid failed %d" % rc)

    def run_records(self, seed, point, first, count, capture_mode=False, max_scatterings=10**6, boundary_rsun=2.0,
                    histograms=False, trace_capacity=0):
        import numpy as np
        recs = (TrajRecord * count)()
        hd = np.zeros((count, NUM_BINS)) if histograms else None
        hv = np.zeros((count, NUM_BINS)) if histograms else None
        tr = np.zeros((max(trace_capacity, 1), 3)) if trace_capacity else None
        tl = ctypes.c_size_t(0)
        rc = self.lib.dms_oracle_run_records(self.h, seed, point, int(capture_mode), max_scatterings, boundary_rsun,
                                             first, count, recs, hd.ctypes.data if hd is not None else None,
                                             hv.ctypes.data if hv is not None else None,
                                             tr.ctypes.data if tr is not None else None, trace_capacity,
                                             ctypes.byref(tl))
        if rc != 0:
            raise RuntimeError("oracle run_records failed %d" % rc)
        out = {"records": recs}
        if histograms:
            out["hist_dt"], out["hist_v2dt"] = hd, hv
        if trace_capacity:
            out["trace"] = tr[: min(tl.value, trace_capacity)]
        return out


class Reference:
    """The reference's own hot-path sources, built with the shims (oracle/_ref/libdms_ref.so).
    Not thread-safe: one draw stream per process."""

    def __init__(self):
        os.environ.setdefault("DMS_SOLAR_MODEL_PATH", SOLAR_MODEL)
        lib = ctypes.CDLL(REF_LIB)
        lib.dms_ref_query.restype = ctypes.c_double
        lib.dms_ref_query.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        lib.dms_ref_set_point.argtypes = [ctypes.POINTER(PointParams)]
        lib.dms_ref_run_records.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, ctypes.c_uint64,
                                            ctypes.c_double, ctypes.c_uint64, ctypes.c_uint64,
                                            ctypes.POINTER(TrajRecord), ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
        lib.dms_ref_run_reflections.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_double,
                                                ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(TrajRecord), ctypes.c_void_p]
        lib.dms_ref_generate_data.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, ctypes.c_uint32,
                                              ctypes.c_uint32, ctypes.c_uint64, ctypes.c_char_p]
        lib.dms_ref_last_error.restype = ctypes.c_char_p
        self.lib = lib
        if lib.dms_ref_init() != 0:
            raise RuntimeError("reference init failed: %s" % lib.dms_ref_last_error())

    def set_point(self, params):
        if self.lib.dms_ref_set_point(ctypes.byref(params)) != 0:
            raise RuntimeError("reference set_point failed: %s" % self.lib.dms_ref_last_error())

    def query(self, what, a=0.0, b=0.0, c=0.0):
        return self.lib.dms_ref_query(what, a, b, c)

    def run_records(self, seed, point, first, count, capture_mode=False, max_scatterings=10**6, boundary_rsun=2.0,
                    histograms=False, trace_capacity=0):
        import numpy as np
        recs = (TrajRecord * count)()
        hd = np.zeros((count, NUM_BINS)) if histograms else None
        hv = np.zeros((count, NUM_BINS)) if histograms else None
        tr = np.zeros((max(trace_capacity, 1), 3)) if trace_capacity else None
        tl = ctypes.c_size_t(0)
        rc = self.lib.dms_ref_run_records(seed, point, int(capture_mode), max_scatterings, boundary_rsun, first, count,
                                          recs, hd.ctypes.data if hd is not None else None,
                                          hv.ctypes.data if hv is not None else None,
                                          tr.ctypes.data if tr is not None else None, trace_capacity,
                                          ctypes.byref(tl))
        if rc != 0:
            raise RuntimeError("reference run_records failed: %s" % self.lib.dms_ref_last_error())
        out = {"records": recs}
        if histograms:
            out["hist_dt"], out["hist_v2dt"] = hd, hv
        if trace_capacity:
            out["trace"] = tr[: min(tl.value, trace_capacity)]
        return out

    def run_reflections(self, seed, point, first, count, max_scatterings=10**6, boundary_rsun=2.0):
        """Records of ids [first, first + count) in Parameter-point mode and, per trajectory, the
        reflection-spectrum sample (speed at 1 AU [km/s], cosine to the Sun's velocity; NaN when the
        trajectory is not a recorded reflection)."""
        import numpy as np
        recs = (TrajRecord * count)()
        out = np.zeros((count, 2))
        rc = self.lib.dms_ref_run_reflections(seed, point, max_scatterings, boundary_rsun, first, count, recs,
                                              out.ctypes.data)
        if rc != 0:
            raise RuntimeError("reference run_reflections failed: %s" % self.lib.dms_ref_last_error())
        return recs, out
