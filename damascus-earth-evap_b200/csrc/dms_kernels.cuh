// Kernel interfaces of the trajectory engine (launched from dms_capi.cu).
#pragma once

#include <cstdint>

#include "dms_device.cuh"

// Minimum resident 128-thread blocks per SM the trajectory kernels are compiled for (caps
// their registers at 65536 / (128 * n)).
#ifndef DMS_TRAJ_MIN_BLOCKS
#define DMS_TRAJ_MIN_BLOCKS 4
#endif
// RK45 form of the kernels: 0 = one loop over the six stages (a short hot loop: fewer
// instruction-cache misses with every lane busy), 1 = the stages written out (a shorter
// dependent chain for a lane that runs alone), 2 = the loop while the work queue still has
// items and the written-out stages once the block has seen it drained (a lane's fetch, or the
// queue head read every 64 iterations).  With the FP64 tail attempts paired across two lanes
// (DMS_PAIRED_ATTEMPTS), form 2 is the default: measured 13 % more accepted steps per second
// with every lane busy than form 1, the same time per step for a lane that runs alone.
#ifndef DMS_RK_UNROLLED
#define DMS_RK_UNROLLED 2
#endif
// FP64 RK45 attempts with the certified straight-line division and square root of
// dms_fastmath.cuh (1) or with IEEE `/` and sqrt (0); the results are the same bits.
#ifndef DMS_CERTIFIED_MATH
#define DMS_CERTIFIED_MATH 1
#endif
// FP64 attempts of lanes that run with idle lanes beside them are computed by two lanes
// (rk45_attempt_pair) when 1; always by the lane alone when 0.  The same bits either way.
#ifndef DMS_PAIRED_ATTEMPTS
#define DMS_PAIRED_ATTEMPTS 1
#endif
// Pairing applies to warps with at most DMS_PAIR_MAX_LANES attempting lanes (up to 16, every
// one paired with an idle lane) and, when DMS_PAIR_ONLY_DRAINED, only once the block has seen
// the work queue drained (the tail of a launch).
#ifndef DMS_PAIR_MAX_LANES
#define DMS_PAIR_MAX_LANES 16
#endif
#ifndef DMS_PAIR_ONLY_DRAINED
#define DMS_PAIR_ONLY_DRAINED 1
#endif
#ifndef DMS_RK_UNROLLED_MIXED
#define DMS_RK_UNROLLED_MIXED 1
#endif
// The FP64 tail pipeline (a second warp of a drained block makes a lone lane's step head and
// attempts while the lane finishes its previous step) when 1.
#ifndef DMS_TAIL_PIPELINE
#define DMS_TAIL_PIPELINE 1
#endif
#ifndef DMS_TRAJ_MIN_BLOCKS_MIXED
#define DMS_TRAJ_MIN_BLOCKS_MIXED 4
#endif

namespace dms
{

// Status bits written by the kernels (device status word).
enum : unsigned int
{
	STATUS_CANCELLED = 1u,
	STATUS_BUDGET = 2u,
	STATUS_IC_REJECTION = 4u,
	STATUS_BAD_RANGE = 8u,
};

// Initial state of one work item, computed for the whole launch before the persistent kernel
// starts: the event after Initial_Conditions and the Kepler shift to the boundary (the raw
// initial event when the shift fails), and the uniform draws consumed.
enum : uint32_t
{
	INIT_IC_OK = 1u,     // initial conditions found within the attempt bound
	INIT_SHIFT_OK = 2u,  // Hyperbolic_Kepler_Shift succeeded
};
struct InitState
{
	Event ic;
	uint32_t draws;
	uint32_t flags;
};
static_assert(sizeof(InitState) == 64, "one initial state per 64 bytes");

struct RunParams
{
	DevSolar S;
	// FP32 images of the knot, G*M and G*M-slope tables (mixed-precision kernel only)
	const float* sf_r;
	const float* sf_gm;
	const float* sf_gm_s;
	const float* sf_vesc2;
	const float* sf_vesc2_s;
	const DevPoint* points;
	int n_points;
	// work: ranges and their prefix offsets (n_ranges + 1)
	const int32_t* range_point;
	const uint64_t* range_first;
	const uint64_t* range_offset;
	int n_ranges;
	uint64_t total;
	unsigned long long* queue_head;
	// options
	uint32_t seed;
	int capture_mode;
	uint64_t max_scatterings;
	uint64_t max_free_steps;
	double boundary;          // km
	uint64_t iteration_budget;
	uint64_t wall_limit_ns;  // per-trajectory wall-clock limit (max_trajectory_wall_time_sec); 0 = none
	// lane scheduling (dms_run_opts; never changes results): ids claimed per queue fetch and
	// the warp batching of scatterings and terminations
	uint32_t queue_chunk;
	int scatter_batch, scatter_wait, final_batch, final_wait;
	int ic_max_attempts;
	// accumulators (accumulate mode)
	unsigned long long* counters;   // n_points x DMS_NUM_COUNTERS
	double* hists;                  // n_points x DMS_NUM_HISTS x DMS_NUM_BINS
	dms_evaporation_event* events;  // n_points x event_capacity
	unsigned long long* event_count;// n_points
	uint64_t event_capacity;
	dms_reflection* reflections;    // n_points x event_capacity
	unsigned long long* reflection_count; // n_points
	// records mode (records != nullptr): one record per work index
	dms_traj_record* records;
	double* rec_hist_dt;
	double* rec_hist_v2dt;
	// per-lane histogram scratch: lanes x DMS_NUM_BINS of (dt, v2dt)
	double2* lane_hist;
	// initial state of every work index (written by initial_state_kernel)
	InitState* init;
	const volatile int* cancel;
	unsigned int* status;
};

// Range of work index w: the largest k with range_offset[k] <= w (binary search).
__device__ __forceinline__ int find_range(const RunParams& R, uint64_t w)
{
	int lo = 0, hi = R.n_ranges - 1;
	while(lo < hi)
	{
		const int mid = (lo + hi + 1) >> 1;
		if(R.range_offset[mid] <= w)
			lo = mid;
		else
			hi = mid - 1;
	}
	return lo;
}

// Checked build: reads and clears the bounds-status bits of the FP64 and the mixed kernels'
// translation units (always 0 without DMS_CHECKED).
unsigned int Take_Bounds_Status();
unsigned int Take_Bounds_Status_Mixed();

// Initial states of all p.total work indices into p.init (one thread per work index); the
// trajectory kernels read them.  Launched on the same stream before every trajectory launch.
void Launch_Initial_States(const RunParams& p, cudaStream_t stream);
void Launch_Trajectories(const RunParams& p, int blocks, int threads, cudaStream_t stream);
void Launch_Rate_Grid(const DevSolar& S, const DevPoint* point, double* grid, int n, cudaStream_t stream);
void Launch_Rate_Query(const DevSolar& S, const DevPoint* point, int interpolated, const double* r, const double* v, double* out,
                       size_t n, cudaStream_t stream);
// mixed-precision (batched FP32) trajectory kernel and the FP32 image of a rate grid
void Launch_Trajectories_Mixed(const RunParams& p, int blocks, int threads, cudaStream_t stream);
void Launch_To_Float(const double* in, float* out, size_t n, cudaStream_t stream);
int Trajectory_Mixed_Max_Blocks_Per_SM(int threads);
int Trajectory_Kernel_Registers();
int Trajectory_Max_Blocks_Per_SM(int threads);
double Measure_FP64_Peak(int sm_count, cudaStream_t stream);
// Self-test of the certified division and square root (dms_fastmath.cuh) against IEEE on n
// random operand pairs; out (4 device counters, zeroed by the caller) as in dms_check_certified_math.
void Check_Certified_Math(uint64_t n, uint64_t seed, unsigned long long* out, int sm_count, cudaStream_t stream);

}	// namespace dms
