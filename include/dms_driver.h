/*
 * dms_driver.h — run driver of the engine (part of libdms_cuda.so): the Generate_Data loop,
 * the output files and the summaries of the reference's "Capture" and "Parameter point" run
 * modes, on top of the trajectory entry points of dms.h.
 *
 *   dms_generate_data   Simulation_Data::Generate_Data           include/Data_Generation.hpp:134,
 *                                                                src/Data_Generation.cpp:488-972
 *   dms_write_outputs   Simulation_Data::Write_Output_Files      include/Data_Generation.hpp:137,
 *                       (bincount.txt, evaporation_times.txt)    src/Data_Generation.cpp:1212-1300
 *   dms_print_summary   Print_Summary / Print_Capture_Mode_Summary
 *                                                                src/Data_Generation.cpp:1366-1499
 *   snapshot_* options  SnapshotHeartbeat + Snapshot_IO reports  src/Snapshot_Heartbeat.cpp:236-354,
 *                       (snapshot/snapshot_{t}s.txt and          src/Snapshot_IO.cpp:508-650, 925-947
 *                       snapshot_{t}s_evaporation_times.txt)
 */
#ifndef DMS_DRIVER_H
#define DMS_DRIVER_H

#include <stdint.h>

#include "dms.h"

#ifdef __cplusplus
extern "C" {
#endif

/* SimulationStopReason, include/Data_Generation.hpp:56-63 */
#define DMS_STOP_NONE                        0
#define DMS_STOP_MAX_TRAJECTORIES            1
#define DMS_STOP_CAPTURE_TARGET_NOT_REACHED  2
#define DMS_STOP_INITIAL_SHIFT_FAILURES      3
#define DMS_STOP_INVALID_TRAJECTORIES        4

typedef struct
{
	uint32_t sample_size;        /* captured particles to collect */
	uint32_t max_trajectories;   /* 0 = unlimited */
	uint32_t seed;               /* fixed_seed */
	int32_t capture_mode;
	uint64_t max_scatterings;    /* maximum_number_of_scatterings */
	double boundary_radius_rsun; /* initial_and_final_radius / R_sun of Configure (2.0); below 1 every
	                                initial Kepler shift fails, as in the reference */
	double sigma_p_cm2;          /* selects the round granularity (the reference's sync interval) */
	uint64_t round_capacity;     /* most trajectories per launch; 0 = 2^20 */
	double time_limit_s;         /* per launch, 0 = none */
	double max_trajectory_wall_time_s;  /* per trajectory (max_trajectory_wall_time_sec), 0 = none */
	uint32_t threads_per_block;  /* 0 = default */
	uint32_t blocks_per_sm;      /* 0 = default */
	/* Wall-clock progress reports (snapshot_enabled / snapshot_interval of the configuration):
	 * with snapshot_dir set and snapshot_interval_s a positive whole number of seconds, the
	 * k-th report is written to snapshot_dir/snapshot_{k*interval}s.txt, with the evaporation
	 * events first seen by it in snapshot_{k*interval}s_evaporation_times.txt.  Ignored in
	 * capture mode (src/Data_Generation.cpp:490-491).  mass and sigma go into the headers. */
	const char* snapshot_dir;    /* NULL = no snapshots */
	double snapshot_interval_s;
	double snapshot_mass_gev;
	double snapshot_sigma_cm2;
	uint64_t max_free_steps;     /* maximum_free_time_steps of Configure; 0 = the default (1e12) */
	int32_t print_progress;      /* 1: progress lines on stdout at 0, 1, 5, 10, 20, 40, 60, 80 and 100 % of
	                                the captures, checked while launches run and after each
	                                (src/Data_Generation.cpp:661-694).  With snapshots or progress
	                                lines on, dms_generate_data uses the context's progress hook
	                                (dms_set_progress_callback) and removes it when it returns. */
	int32_t reserved;
} dms_generate_opts;

typedef struct
{
	uint64_t counters[DMS_NUM_COUNTERS];
	uint64_t rounds;                   /* launches (mpi_sync_rounds) */
	uint64_t final_round_trajectories;
	uint64_t capture_target_overshoot;
	uint64_t sync_interval;            /* normal_mode_mpi_sync_interval (0 in capture mode) */
	uint64_t next_trajectory;          /* first unused trajectory id */
	int32_t early_stop_reason;         /* DMS_STOP_* */
	int32_t reserved;
	double computing_time_s;
} dms_generate_summary;

void dms_default_generate_opts(dms_generate_opts* opts);
int dms_generate_data(dms_ctx* ctx, int point_id, const dms_generate_opts* opts, dms_generate_summary* summary);
int dms_write_outputs(dms_ctx* ctx, int point_id, const dms_generate_summary* summary, double mass_gev, double sigma_cm2,
                      const char* output_dir);
int dms_print_summary(dms_ctx* ctx, int point_id, const dms_generate_summary* summary, int capture_mode);

/* ---- reflection spectrum (Reflection_Spectrum, src/Reflection_Spectrum.cpp:12-73) -------------
 * From the reflected particles recorded by dms_run (dms_reflection): the particles of one
 * isoreflection ring (equal-area rings around the Sun's velocity, Isoreflection_Ring_Angles,
 * src/Simulation_Utilities.cpp:323-336), the DM entering rate pi R_sun^2 n (<u> + v_esc^2 <1/u>)
 * (DM_Entering_Rate, :63-71), the reflection rate (entering rate x reflected fraction) and the
 * flux at 1 AU. */
typedef struct
{
	uint64_t trajectories;             /* trajectories behind the sample */
	uint64_t reflections;              /* recorded reflected particles in the ring */
	double reflection_ratio;           /* reflections / trajectories (Reflection_Ratio) */
	double entering_rate_per_s;
	double reflection_rate_per_s;
	double distance_au;                /* 1 */
	double flux_per_s_cm2;             /* reflection rate / (4 pi d^2) x rings */
	double speed_min_kms, speed_max_kms;  /* spectrum domain: [0, 1.05 x highest speed] */
	double mean_speed_kms;
} dms_reflection_spectrum;

int dms_get_reflection_spectrum(dms_ctx* ctx, int point_id, uint32_t rings, uint32_t ring, double dm_density_gev_cm3,
                                dms_reflection_spectrum* out);
/* Speed distribution of the ring's reflected particles at the n speeds u_kms [1/(km/s)]: a
 * Gaussian kernel density estimate (Silverman bandwidth, mirrored at the lower domain edge),
 * zero outside the domain.  Multiply by reflection_rate_per_s for the differential spectrum. */
int dms_reflection_spectrum_pdf(dms_ctx* ctx, int point_id, uint32_t rings, uint32_t ring, const double* u_kms, size_t n,
                                double* pdf);
int dms_print_reflection_summary(const dms_reflection_spectrum* spectrum);

#ifdef __cplusplus
}
#endif
#endif /* DMS_DRIVER_H */
