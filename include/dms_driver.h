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
	double boundary_radius_rsun; /* 2.0 */
	double sigma_p_cm2;          /* selects the round granularity (the reference's sync interval) */
	uint64_t round_capacity;     /* most trajectories per launch; 0 = 2^20 */
	double time_limit_s;         /* per launch, 0 = none */
	uint32_t threads_per_block;  /* 0 = default */
	uint32_t blocks_per_sm;      /* 0 = default */
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

#ifdef __cplusplus
}
#endif
#endif /* DMS_DRIVER_H */
