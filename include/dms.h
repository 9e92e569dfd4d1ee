/*
 * dms.h — C ABI of the B200 trajectory engine (libdms_cuda.so).
 *
 * The engine replaces the per-trajectory Monte Carlo of DaMaSCUS-SUN-EVAP and the MPI batching
 * that drives it.  Reference interfaces replaced, by entry point:
 *   dms_load_solar_model   Solar_Model::Solar_Model()                include/Solar_Model.hpp:320,
 *                                                                    src/Solar_Model.cpp:128-166
 *   dms_add_point          DM particle construction + Solar_Model::Interpolate_Total_DM_Scattering_Rate
 *                                                                    src/Parameter_Scan.cpp:386-471,
 *                                                                    include/Solar_Model.hpp:338
 *   dms_run                Simulation_Data::Generate_Data trajectory loop (simulate_one_trajectory
 *                          + MPI rounds/tail work)                  include/Data_Generation.hpp:134,
 *                                                                    src/Data_Generation.cpp:488-972
 *   dms_run_records        Initial_Conditions + Hyperbolic_Kepler_Shift + Trajectory_Simulator::Simulate
 *                          for listed trajectories                   include/Simulation_Trajectory.hpp:174
 *   dms_get_results        Simulation_Data accumulators after Perform_MPI_Reductions
 *                                                                    src/Data_Generation.cpp:974-1210
 *   dms_rate               Solar_Model::Total_DM_Scattering_Rate     include/Solar_Model.hpp:334
 *   dms_set_progress_callback, dms_peek_progress, dms_peek_results
 *                          SnapshotRecorder + SnapshotHeartbeat (live progress of a run)
 *                                                                    src/Snapshot_Shared_State.cpp:65-164,
 *                                                                    src/Snapshot_Heartbeat.cpp:236-270
 *
 * Conventions: every call returns DMS_OK (0) or a negative DMS_ERR_* code, and the message of
 * the last failure is available from dms_last_error().  No C++ exception crosses the ABI.
 * Pointers passed in are caller-owned and only read during the call (copied where kept).
 * One host thread per context; contexts on different devices may coexist.
 * Units: km, s, km/s, eV, K; cross sections in cm^2 and masses in GeV at the boundary.
 */
#ifndef DMS_H
#define DMS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------------ */
#define DMS_OK                    0
#define DMS_ERR_INVALID_ARGUMENT (-1)
#define DMS_ERR_CUDA             (-2)
#define DMS_ERR_IO               (-3)
#define DMS_ERR_NO_SOLAR_MODEL   (-4)
#define DMS_ERR_NO_POINT         (-5)
#define DMS_ERR_CAPACITY         (-6)
#define DMS_ERR_BUDGET           (-7)
#define DMS_ERR_CANCELLED        (-8)
#define DMS_ERR_STATE            (-9)

/* ---- termination reasons: TrajectoryTerminationReason, include/Simulation_Trajectory.hpp:35-48 */
#define DMS_REASON_UNKNOWN              0
#define DMS_REASON_OUTWARD_ESCAPE       1
#define DMS_REASON_SCATTER              2
#define DMS_REASON_WALL_TIME_LIMIT      3
#define DMS_REASON_MAX_FREE_STEPS       4
#define DMS_REASON_MAX_SCATTERINGS      5
#define DMS_REASON_NON_FINITE_STATE     6
#define DMS_REASON_SPEED_LIMIT          7
#define DMS_REASON_NUMERICAL_FAILURE    8
#define DMS_REASON_CAPTURE_MODE         9
#define DMS_REASON_ENERGY_DRIFT_ESCAPE 10
#define DMS_REASON_COUNT               11

/* record flags */
#define DMS_REC_SHIFT_OK          0x01u   /* initial Hyperbolic_Kepler_Shift succeeded */
#define DMS_REC_CAPTURED          0x02u   /* TrajectoryBincount::is_captured */
#define DMS_REC_EVENT_OBSERVED    0x04u
#define DMS_REC_SURVIVAL_VALID    0x08u
#define DMS_REC_BOUNDARY_ESCAPE   0x10u
#define DMS_REC_FREE              0x20u   /* Trajectory_Result::Particle_Free */
#define DMS_REC_REFLECTED         0x40u   /* Trajectory_Result::Particle_Reflected */
#define DMS_REC_REFLECT_SHIFT_OK  0x80u   /* final Kepler shift to 1 AU succeeded (reflected only) */
#define DMS_REC_INVALID_ESCAPE    0x100u  /* numerically_invalid_escape */

/* Per-trajectory outcome (Trajectory_Result + TrajectoryBincount scalars,
 * include/Simulation_Trajectory.hpp:53-85, 101-114).  Times in s, positions in km,
 * velocities in km/s.  The same layout is produced by the engine, the CPU oracle and the
 * reference build of the oracle. */
typedef struct
{
	uint64_t trajectory_id;
	uint64_t number_of_scatterings;
	uint64_t number_of_draws;          /* uniform draws consumed (replay check) */
	uint32_t point;
	uint32_t termination_reason;       /* DMS_REASON_* */
	uint32_t flags;                    /* DMS_REC_* */
	uint32_t reserved;
	double initial_time;               /* event after the initial Kepler shift */
	double initial_position[3];
	double initial_velocity[3];
	double final_time;
	double final_position[3];
	double final_velocity[3];
	double t_capture;                  /* -1 if never captured */
	double t_last_bound;
	double t_final_unbinding_scatter;  /* NaN if none */
	double t_boundary_escape;          /* NaN if none */
	double t_termination;
	double max_free_energy_drift_eV;
	double max_free_energy_drift_rel;
	double lifetime_unbinding;         /* t_final_unbinding - t_capture for completed events, else -1 */
} dms_traj_record;

/* ---- context ----------------------------------------------------------------------------- */
typedef struct dms_ctx dms_ctx;

int dms_create(dms_ctx** ctx, int device);
void dms_destroy(dms_ctx* ctx);
const char* dms_last_error(const dms_ctx* ctx);
/* Request cancellation of a running dms_run from another host thread (mapped flag). */
int dms_cancel(dms_ctx* ctx);

/* ---- solar model ------------------------------------------------------------------------- */
/* Loads the AGSS09 table (35 columns, 20 header lines) and builds the radial tables on the
 * device: G*M(r), T(r), v_esc^2(r), n_e(r) and n_i(r) for the 63 isotope targets. */
int dms_load_solar_model(dms_ctx* ctx, const char* path);

/* Copies one radial table back from the device (Solar_Model's interpolation tables,
 * include/Solar_Model.hpp:294-305): which = 0 knots r [km], 1 G*M [km^3/s^2], 2 T [GeV],
 * 3 v_esc^2 [km^2/s^2], 4 n_e [1/km^3], 5 n_i [1/km^3] node-major (knots x 63).
 * Returns the number of values (also when out is NULL) or a negative DMS_ERR_*. */
int dms_solar_table(dms_ctx* ctx, int which, double* out, size_t capacity);

/* ---- parameter points -------------------------------------------------------------------- */

/* DM interaction models (low-mass mode, DM_light = true):
 *   SI                    DM_Particle_Standard "SI" with a contact interaction:
 *                         sigma_N = sigma_p (mu_N/mu_p)^2 [Z + (f_n/f_p)(A - Z)]^2, isotropic angle
 *   DARK_PHOTON_CONTACT   DM_Particle_Dark_Photon, DM_form_factor "Contact"
 *                         (src/Dark_Photon.cpp:157-184, 190-210): the cross sections follow from the
 *                         electron one, sigma_p = sigma_e (mu_p/mu_e)^2 and
 *                         sigma_N = sigma_p (mu_N/mu_p)^2 Z^2; isotropic angle
 *   DARK_PHOTON_GENERAL   "General", a dark photon of mass DM_mediator_mass: the contact cross
 *                         sections times (q_ref^2 + m^2)^2 / (m^2 (m^2 + q_max^2)) with
 *                         q_ref = alpha m_e and q_max = 2 mu v (v the DM speed), and the scattering
 *                         angle cos = (m^2 (2 xi - 1) + q_max^2 xi) / (m^2 + q_max^2 xi)
 *                         (src/Dark_Photon.cpp:192-229, 302-325)
 * For the dark photon, sigma_p_cm2 and fn_over_fp are not used (the reference reads only
 * DM_cross_section_electron, src/Parameter_Scan.cpp:508-519). */
#define DMS_INTERACTION_SI                   0
#define DMS_INTERACTION_DARK_PHOTON_CONTACT  1
#define DMS_INTERACTION_DARK_PHOTON_GENERAL  2

typedef struct
{
	double mass_gev;                   /* DM_mass */
	double sigma_p_cm2;                /* DM_cross_section_nucleon (SI) */
	double sigma_e_cm2;                /* DM_cross_section_electron */
	double fn_over_fp;                 /* 1.0 when DM_isospin_conserved */
	double halo_v0_kms;                /* SHM_v0 */
	double halo_vesc_kms;              /* SHM_vEscape */
	double halo_vobs_kms[3];           /* SHM_vObserver */
	uint32_t interpolation_points;     /* N of the N x N total-rate grid; N < 2: no grid, every
	                                      lookup sums the 64 channels (Total_DM_Scattering_Rate_Computed) */
	uint32_t interaction;              /* DMS_INTERACTION_* */
	double mediator_mass_mev;          /* DM_mediator_mass of DARK_PHOTON_GENERAL [MeV], > 0 */
} dms_point_params;

/* Adds a parameter point and builds its N x N total-rate grid on the device (one kernel,
 * Total_DM_Scattering_Rate_Computed at every node, src/Solar_Model.cpp:395-465). */
int dms_add_point(dms_ctx* ctx, const dms_point_params* params, int* point_id);
int dms_num_points(const dms_ctx* ctx);

/* Replaces / reads the N x N total-rate grid of a point (N*N doubles, radius-major, 1/s):
 * the rate_grid member of Solar_Model after Interpolate_Total_DM_Scattering_Rate
 * (include/Solar_Model.hpp:309), for callers that build or cache the grid elsewhere. */
int dms_set_rate_grid(dms_ctx* ctx, int point_id, const double* grid, uint32_t n);
int dms_get_rate_grid(dms_ctx* ctx, int point_id, double* grid, uint32_t n);

/* Scattering rate [1/s] of point `point_id` at radius r_km and speed v_kms, through the
 * interpolated grid (interpolated = 1) or the direct sum over targets (interpolated = 0).
 * Evaluated on the device for n query pairs. */
int dms_rate(dms_ctx* ctx, int point_id, int interpolated, const double* r_km, const double* v_kms, double* rate_out, size_t n);

/* ---- runs -------------------------------------------------------------------------------- */
/* FP64: every operation in the reference's FP64 order (bit-identical with the CPU oracle).
 * MIXED: the batched FP32 form (no reference counterpart; the reference is FP64 only): RK45
 * stages, the 3-D event, chord geometry and rate interpolation in FP32; propagator state,
 * time, optical depth, orbital energy, the RK45 error norm, scattering kinematics and the
 * accumulators in FP64.  Agrees with FP64 statistically, not trajectory by trajectory. */
#define DMS_PRECISION_FP64  0
#define DMS_PRECISION_MIXED 1

typedef struct
{
	uint32_t seed;                     /* fixed_seed; draw-stream key */
	int32_t capture_mode;              /* 1: stop each trajectory at the first post-scatter E < 0 */
	uint64_t max_scatterings;          /* maximum_number_of_scatterings */
	uint64_t max_free_steps;           /* maximum_free_time_steps */
	double boundary_radius_rsun;       /* initial_and_final_radius / R_sun (2.0) */
	int32_t precision;                 /* DMS_PRECISION_* */
	uint32_t threads_per_block;        /* 32, 64, 96 or 128; 0 = 128 */
	uint32_t blocks_per_sm;            /* resident blocks per SM; 0 = as many as fit */
	uint32_t queue_chunk;              /* trajectory ids a lane claims from the work queue at a time
	                                      (1..1024); 0 = 1 */
	uint64_t iteration_budget;         /* per-lane loop-iteration bound; 0 = default */
	double time_limit_s;               /* wall-clock bound of one launch, enforced through the
	                                      cancel flag; 0 = none */
	double max_trajectory_wall_time_s; /* max_trajectory_wall_time_sec: a trajectory whose wall time
	                                      on its lane exceeds it ends with
	                                      DMS_REASON_WALL_TIME_LIMIT (checked before and after each
	                                      RK45 step, src/Simulation_Trajectory.cpp:824-840); 0 = none */
	/* Warp batching of the rare phases (no reference counterpart; results do not depend on it):
	 * a lane that reaches a scattering point (a termination) waits until scatter_batch
	 * (final_batch) lanes of its warp are there, or it has waited scatter_wait (final_wait)
	 * loop iterations, or no lane of the warp is stepping; then the warp runs the scattering
	 * (termination) code once for all of them.  0 = defaults 16 / 32 / 8 / 32; batches up to
	 * 32, waits up to 1024. */
	uint32_t scatter_batch;
	uint32_t scatter_wait;
	uint32_t final_batch;
	uint32_t final_wait;
} dms_run_opts;

typedef struct
{
	int32_t point_id;
	uint32_t reserved;
	uint64_t first_trajectory;         /* trajectory ids [first, first + count) */
	uint64_t count;
} dms_work_range;

void dms_default_run_opts(dms_run_opts* opts);

/* Autotuner of the launch (no reference counterpart): picks threads_per_block, blocks_per_sm,
 * queue_chunk and the warp-batching thresholds (the lane-compaction interval of the persistent
 * kernel) for the points of `ranges` and the precision of `base`.  Each trial is a launch of
 * trial_seconds wall time over fresh trajectory ids of those points (ids from 2^40 on, results
 * kept in a scratch accumulator, so the points' own results are untouched), scored by accepted
 * free steps per second; the parameters are searched one at a time from the defaults
 * (coordinate descent, two passes).  *tuned receives `base` with the best setting; the chosen
 * setting changes throughput only, never results (every draw is keyed by trajectory id).
 * trials (may be NULL) receives the number of trial launches. */
int dms_autotune(dms_ctx* ctx, const dms_run_opts* base, const dms_work_range* ranges, int n_ranges, double trial_seconds,
                 dms_run_opts* tuned, int* trials);

/* Simulates every trajectory of the given ranges in one persistent launch and adds the
 * outcomes to the per-point accumulators (counters, the four 2000-bin histograms with their
 * per-trajectory sums of squares, completed evaporation events). */
int dms_run(dms_ctx* ctx, const dms_run_opts* opts, const dms_work_range* ranges, int n_ranges);

/* Simulates trajectories [first, first + count) of one point and returns one record per
 * trajectory (host buffer of `count` records).  Does not touch the accumulators.  When
 * hist_dt / hist_v2dt are non-null they receive each trajectory's own 2000-bin
 * histograms (count * 2000 doubles each). */
int dms_run_records(dms_ctx* ctx, const dms_run_opts* opts, int point_id, uint64_t first, uint64_t count,
                    dms_traj_record* records, double* hist_dt, double* hist_v2dt);

/* No counterpart in the reference.  dms_run_records for a caller that cannot allocate device
 * memory when it runs: it allocates nothing.  d_records (count records) and, when non-null,
 * d_hist_dt / d_hist_v2dt (count * 2000 doubles each) are DEVICE buffers owned by the caller,
 * filled with the same values dms_run_records returns.  The run's scratch (work queue, status
 * word, initial states, one 2000-bin histogram row per lane) is a fixed array of
 * DMS_NOALLOC_SCRATCH_BYTES in the library's device image, so at most
 * DMS_NOALLOC_MAX_TRAJECTORIES trajectories fit one
 * call; larger counts return DMS_ERR_INVALID_ARGUMENT.  It always runs the FP64 kernel:
 * opts->precision is ignored (MIXED runs FP64 too), and so are threads_per_block and
 * blocks_per_sm (one lane per trajectory); the other options, the per-trajectory wall-time
 * limit included, apply as in dms_run_records.  Like the other launching calls it is refused
 * (DMS_ERR_STATE) from a progress callback.  The first call on a device looks the array up
 * and keeps its address for the life of the process; make that call before any stream capture
 * on that device starts, and do not reset the device (cudaDeviceReset) between calls.  Every
 * call on a device shares the array: calls that overlap on the GPU (two contexts or two host
 * threads on one device) race.  DMS_NOALLOC_SCRATCH_BYTES is 4 104 448 bytes (about 3.9 MiB). */
#define DMS_NOALLOC_MAX_TRAJECTORIES 128
#define DMS_NOALLOC_SCRATCH_BYTES    (256 + DMS_NOALLOC_MAX_TRAJECTORIES * (64 + 2000 * 16))
int dms_run_records_noalloc(dms_ctx* ctx, const dms_run_opts* opts, int point_id, uint64_t first, uint64_t count,
                            dms_traj_record* d_records, double* d_hist_dt, double* d_hist_v2dt);

/* ---- results ----------------------------------------------------------------------------- */
/* Counter slots of dms_point_results.counters (Simulation_Data members,
 * include/Data_Generation.hpp:78-95). */
#define DMS_CNT_TRAJECTORIES              0
#define DMS_CNT_FREE                      1
#define DMS_CNT_REFLECTED                 2
#define DMS_CNT_CAPTURED                  3
#define DMS_CNT_COMPLETED_OUTWARD         4
#define DMS_CNT_COMPLETE_EVAPORATION      5
#define DMS_CNT_CENSORED_CAPTURED         6
#define DMS_CNT_INVALID_SURVIVAL          7
#define DMS_CNT_INITIAL_SHIFT_FAILURES    8
#define DMS_CNT_FINAL_REFLECTION_SHIFT_FAILURES 9
#define DMS_CNT_NUMERICAL_FAILURES        10
#define DMS_CNT_COMPUTATIONAL_TRUNCATIONS 11
#define DMS_CNT_TOTAL_SCATTERINGS         12
#define DMS_CNT_RK_STEPS                  13   /* accepted free-propagation steps (work counter) */
#define DMS_CNT_EVENTS_DROPPED            14   /* evaporation events beyond the buffer capacity */
#define DMS_CNT_RK_ATTEMPTS               15   /* RK45 stage evaluations incl. rejected tries (work counter) */
#define DMS_CNT_REASON_BASE               16   /* + DMS_REASON_*: trajectories per termination reason */
/* work of the trajectories that a cancelled (time limit) or budget-stopped launch left
 * unfinished; they are not in any counter above */
#define DMS_CNT_UNFINISHED_TRAJECTORIES   27
#define DMS_CNT_UNFINISHED_SCATTERINGS    28
#define DMS_CNT_UNFINISHED_RK_STEPS       29
#define DMS_CNT_UNFINISHED_RK_ATTEMPTS    30
#define DMS_CNT_REFLECTIONS_DROPPED       31   /* reflected-particle records beyond the buffer capacity */
#define DMS_NUM_COUNTERS                  32

/* Histogram slots (each DMS_NUM_BINS doubles), src/Data_Generation.cpp:101-110 */
#define DMS_HIST_CAPTURED_DT         0
#define DMS_HIST_CAPTURED_V2DT       1
#define DMS_HIST_NOT_CAPTURED_DT     2
#define DMS_HIST_NOT_CAPTURED_V2DT   3
#define DMS_HIST_CAPTURED_DT_SQ      4
#define DMS_HIST_CAPTURED_V2DT_SQ    5
#define DMS_HIST_NOT_CAPTURED_DT_SQ  6
#define DMS_HIST_NOT_CAPTURED_V2DT_SQ 7
#define DMS_NUM_HISTS                8

/* CompactEvaporationEvent, include/Data_Generation.hpp:48-54 */
typedef struct
{
	uint64_t trajectory_id;
	double lifetime_unbinding;
} dms_evaporation_event;

/* A reflected particle (not captured, escaped outward after at least one scattering) whose
 * orbit was carried to 1 AU (Hyperbolic_Kepler_Shift): the data behind the reflection
 * spectrum, src/Data_Generation.cpp:824-846.  cos_sun_velocity is the cosine of the angle
 * between its position at 1 AU and the Sun's velocity (Isoreflection_Angle,
 * src/Simulation_Utilities.cpp:82-92), from which the isoreflection ring follows. */
typedef struct
{
	uint64_t trajectory_id;            /* trajectory index + 1 */
	double speed_kms;                  /* speed at 1 AU */
	double cos_sun_velocity;
} dms_reflection;

typedef struct
{
	uint64_t counters[DMS_NUM_COUNTERS];
	double* histograms;                /* caller buffer: DMS_NUM_HISTS * DMS_NUM_BINS doubles, or NULL */
	dms_evaporation_event* events;     /* caller buffer of events_capacity entries, or NULL */
	uint64_t events_capacity;
	uint64_t events_count;             /* events stored on the device (copied: min(count, capacity)) */
	dms_reflection* reflections;       /* caller buffer of reflections_capacity entries, or NULL */
	uint64_t reflections_capacity;
	uint64_t reflections_count;        /* reflections stored on the device */
} dms_point_results;

int dms_get_results(dms_ctx* ctx, int point_id, dms_point_results* results);
int dms_reset_results(dms_ctx* ctx, int point_id);

/* ---- Progress while a run is in flight ------------------------------------------------------
 * Replaces the per-step SnapshotRecorder hooks and the heartbeat thread
 * (src/Snapshot_Shared_State.cpp:65-78, src/Snapshot_Heartbeat.cpp:236-270): the kernel takes no
 * per-step hook; instead the thread that called dms_run (or dms_run_records) polls the launch
 * and calls fn about every interval_s seconds of wall time until the kernel ends.  fn may call
 * dms_peek_progress and dms_peek_results; the calls that launch work or change what the kernel
 * reads (dms_run*, dms_add_point, dms_set_rate_grid, dms_reset_results, dms_rate,
 * dms_load_solar_model, dms_measure_fp64_peak) return DMS_ERR_STATE there.  A non-zero return
 * cancels the run (dms_run then returns DMS_ERR_CANCELLED) and ends the calls for that run.
 * fn = NULL removes the hook. */
typedef int (*dms_progress_fn)(dms_ctx* ctx, void* user);
int dms_set_progress_callback(dms_ctx* ctx, dms_progress_fn fn, void* user, double interval_s);

typedef struct
{
	int32_t running;        /* 1 while a launch is in flight */
	int32_t reserved;
	uint64_t total;         /* work items of the launch in flight (or of the last one) */
	uint64_t dispatched;    /* work items taken by lanes so far, at most total */
	double elapsed_s;       /* wall time since the launch began */
} dms_progress;
int dms_peek_progress(dms_ctx* ctx, dms_progress* progress);

/* dms_get_results for a run in flight: counters and histograms of the trajectories finished so
 * far, read on a second stream beside the running kernel, and the evaporation events published
 * so far.  events_count is the number of leading published events copied (an event that another
 * lane is still writing ends the prefix; it is published by a later call).  The view is for
 * progress reports only: a trajectory finishing during the copy may be counted without its
 * histogram rows, or the reverse.  Reflections are not part of it (reflections_count = 0). */
int dms_peek_results(dms_ctx* ctx, int point_id, dms_point_results* results);

/* Sizes a caller needs to know. */
int dms_num_bins(void);

/* Device time [ms] of the last trajectory launch of dms_run / dms_run_records, measured with
 * CUDA events on the context's stream around the kernel (no reference counterpart: the
 * reference reports wall-clock computing_time only, src/Data_Generation.cpp:953-954). */
int dms_last_kernel_ms(const dms_ctx* ctx, double* ms);

/* Measures the device's FP64 FMA throughput [TFLOP/s, 2 FLOP per FMA] with a kernel of
 * independent DFMA chains over every SM: the roofline denominator of the FP64 trajectory
 * kernel (a diagnostic with no reference counterpart). */
int dms_measure_fp64_peak(dms_ctx* ctx, double* tflops);

/* Self-test of the certified straight-line FP64 division and square root that the FP64 RK45
 * attempts use (a diagnostic with no reference counterpart): n random operand pairs, each
 * divided and square-rooted both ways.  counts[0] = quotients whose certificate held but whose
 * bits differ from IEEE a / b (must be 0), counts[1] = quotients whose certificate failed (the
 * kernel then falls back to IEEE), counts[2], counts[3] the same for sqrt. */
int dms_check_certified_math(dms_ctx* ctx, uint64_t n, uint64_t seed, uint64_t* counts);

#ifdef __cplusplus
}
#endif

#endif /* DMS_H */
