// Kernel interfaces of the trajectory engine (launched from dms_capi.cu).
#pragma once

#include <cstdint>

#include "dms_device.cuh"

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

struct RunParams
{
	DevSolar S;
	// FP32 images of the knot, G*M and G*M-slope tables (mixed-precision kernel only)
	const float* sf_r;
	const float* sf_gm;
	const float* sf_gm_s;
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
	int ic_max_attempts;
	// accumulators (accumulate mode)
	unsigned long long* counters;   // n_points x DMS_NUM_COUNTERS
	double* hists;                  // n_points x DMS_NUM_HISTS x DMS_NUM_BINS
	dms_evaporation_event* events;  // n_points x event_capacity
	unsigned long long* event_count;// n_points
	uint64_t event_capacity;
	// records mode (records != nullptr): one record per work index
	dms_traj_record* records;
	double* rec_hist_dt;
	double* rec_hist_v2dt;
	// per-lane histogram scratch: lanes x DMS_NUM_BINS of (dt, v2dt)
	double2* lane_hist;
	const volatile int* cancel;
	unsigned int* status;
};

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

}	// namespace dms
