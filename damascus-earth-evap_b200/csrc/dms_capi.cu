// C ABI of the trajectory engine (include/dms.h): context, device memory, launches.
//
// Device memory layout of a context (all FP64 unless noted):
//   radial tables   one allocation: r, G*M, T, v_esc^2, n_e (+ slopes) and the 63 isotope densities
//                   node-major (+ slopes), and the uint16 bucket index of the knot search
//   points          DevPoint[capacity] (constants of every parameter point) and one N x N rate
//                   grid per point (radius-major, as the reference's rate_grid)
//   accumulators    counters [points x 32] u64, histograms [points x 8 x 2000], evaporation
//                   events [points x event capacity]
//   lane scratch    one 2000-bin (dt, v2dt) row per resident lane; zero between trajectories
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <iostream>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/dms.h"
#include "../../include/dms_driver.h"
#include "dms_host_model.h"
#include "dms_kernels.cuh"

using namespace dms;

struct dms_ctx
{
	int device = 0;
	int sm_count = 0;
	std::string error;
	cudaStream_t stream = nullptr;
	// solar model
	bool has_solar = false;
	SolarTables tables;
	void* d_tables = nullptr;
	DevSolar dsolar{};
	float* d_tables_f = nullptr;    // FP32 r, G*M, G*M slope for the mixed-precision kernel
	// points
	std::vector<PointConstants> points;
	std::vector<double*> d_grids;
	std::vector<float*> d_grids_f;  // FP32 image of each rate grid, rebuilt when stale
	std::vector<char> grid_f_valid;
	DevPoint* d_points = nullptr;
	int point_capacity = 0;
	// accumulators
	unsigned long long* d_counters = nullptr;
	double* d_hists = nullptr;
	dms_evaporation_event* d_events = nullptr;
	unsigned long long* d_event_count = nullptr;
	dms_reflection* d_refl = nullptr;              // [points x event capacity]
	unsigned long long* d_refl_count = nullptr;
	uint64_t event_capacity = 1ULL << 20;
	// run scratch
	double2* d_lane_hist = nullptr;
	size_t lane_capacity = 0;
	InitState* d_init = nullptr;    // initial state of every work index of a launch
	uint64_t init_capacity = 0;
	unsigned long long* d_queue = nullptr;
	unsigned int* d_status = nullptr;
	int* h_cancel = nullptr;       // mapped host memory
	int* d_cancel = nullptr;
	cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
	double last_kernel_ms = 0.0;
	// progress of the launch in flight (dms_set_progress_callback, dms_peek_*)
	dms_progress_fn progress_fn = nullptr;
	void* progress_user = nullptr;
	double progress_interval_s = 1.0;
	cudaStream_t peek_stream = nullptr;  // non-blocking: its copies run beside the kernel
	bool running = false;
	uint64_t launch_total = 0;
	std::chrono::steady_clock::time_point launch_start{};
};

namespace
{
int Fail(dms_ctx* ctx, int code, const std::string& msg)
{
	if(ctx)
		ctx->error = msg;
	return code;
}

// A progress callback runs while its launch is in flight; it may only peek.  Calls that would
// reallocate or overwrite what the kernel uses are refused there.
#define DMS_NOT_IN_FLIGHT(ctx)                                                                         \
	do                                                                                                 \
	{                                                                                                  \
		if((ctx)->running)                                                                             \
			return Fail((ctx), DMS_ERR_STATE, "not allowed while a launch is in flight (progress callback)"); \
	} while(0)

#define DMS_CUDA(ctx, call)                                                                                   \
	do                                                                                                        \
	{                                                                                                         \
		const cudaError_t e_ = (call);                                                                        \
		if(e_ != cudaSuccess)                                                                                 \
			return Fail(ctx, DMS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));             \
	} while(0)

constexpr int MAX_POINTS = 4096;

int Grow_Points(dms_ctx* ctx, int needed)
{
	if(needed <= ctx->point_capacity)
		return DMS_OK;
	int cap = std::max(8, ctx->point_capacity);
	while(cap < needed) cap *= 2;
	DevPoint* np = nullptr;
	unsigned long long* nc = nullptr;
	double* nh = nullptr;
	dms_evaporation_event* ne = nullptr;
	unsigned long long* nn = nullptr;
	dms_reflection* nr = nullptr;
	unsigned long long* nrc = nullptr;
	DMS_CUDA(ctx, cudaMalloc(&np, sizeof(DevPoint) * cap));
	DMS_CUDA(ctx, cudaMalloc(&nc, sizeof(unsigned long long) * DMS_NUM_COUNTERS * cap));
	DMS_CUDA(ctx, cudaMalloc(&nh, sizeof(double) * DMS_NUM_HISTS * DMS_NUM_BINS * cap));
	DMS_CUDA(ctx, cudaMalloc(&ne, sizeof(dms_evaporation_event) * ctx->event_capacity * cap));
	DMS_CUDA(ctx, cudaMalloc(&nn, sizeof(unsigned long long) * cap));
	DMS_CUDA(ctx, cudaMalloc(&nr, sizeof(dms_reflection) * ctx->event_capacity * cap));
	DMS_CUDA(ctx, cudaMalloc(&nrc, sizeof(unsigned long long) * cap));
	DMS_CUDA(ctx, cudaMemset(nrc, 0, sizeof(unsigned long long) * cap));
	DMS_CUDA(ctx, cudaMemset(nc, 0, sizeof(unsigned long long) * DMS_NUM_COUNTERS * cap));
	DMS_CUDA(ctx, cudaMemset(nh, 0, sizeof(double) * DMS_NUM_HISTS * DMS_NUM_BINS * cap));
	DMS_CUDA(ctx, cudaMemset(nn, 0, sizeof(unsigned long long) * cap));
	// an evaporation slot with trajectory id 0 is unpublished (dms_peek_results)
	DMS_CUDA(ctx, cudaMemset(ne, 0, sizeof(dms_evaporation_event) * ctx->event_capacity * cap));
	const int old = static_cast<int>(ctx->points.size());
	if(old > 0)
	{
		DMS_CUDA(ctx, cudaMemcpy(np, ctx->d_points, sizeof(DevPoint) * old, cudaMemcpyDeviceToDevice));
		DMS_CUDA(ctx, cudaMemcpy(nc, ctx->d_counters, sizeof(unsigned long long) * DMS_NUM_COUNTERS * old, cudaMemcpyDeviceToDevice));
		DMS_CUDA(ctx, cudaMemcpy(nh, ctx->d_hists, sizeof(double) * DMS_NUM_HISTS * DMS_NUM_BINS * old, cudaMemcpyDeviceToDevice));
		for(int p = 0; p < old; p++)
			DMS_CUDA(ctx, cudaMemcpy(ne + p * ctx->event_capacity, ctx->d_events + p * ctx->event_capacity,
			                         sizeof(dms_evaporation_event) * ctx->event_capacity, cudaMemcpyDeviceToDevice));
		DMS_CUDA(ctx, cudaMemcpy(nn, ctx->d_event_count, sizeof(unsigned long long) * old, cudaMemcpyDeviceToDevice));
		for(int p = 0; p < old; p++)
			DMS_CUDA(ctx, cudaMemcpy(nr + p * ctx->event_capacity, ctx->d_refl + p * ctx->event_capacity,
			                         sizeof(dms_reflection) * ctx->event_capacity, cudaMemcpyDeviceToDevice));
		DMS_CUDA(ctx, cudaMemcpy(nrc, ctx->d_refl_count, sizeof(unsigned long long) * old, cudaMemcpyDeviceToDevice));
	}
	cudaFree(ctx->d_points);
	cudaFree(ctx->d_counters);
	cudaFree(ctx->d_hists);
	cudaFree(ctx->d_events);
	cudaFree(ctx->d_event_count);
	cudaFree(ctx->d_refl);
	cudaFree(ctx->d_refl_count);
	ctx->d_refl = nr;
	ctx->d_refl_count = nrc;
	ctx->d_points = np;
	ctx->d_counters = nc;
	ctx->d_hists = nh;
	ctx->d_events = ne;
	ctx->d_event_count = nn;
	ctx->point_capacity = cap;
	return DMS_OK;
}

int Ensure_Lanes(dms_ctx* ctx, size_t lanes)
{
	if(lanes <= ctx->lane_capacity)
		return DMS_OK;
	cudaFree(ctx->d_lane_hist);
	ctx->d_lane_hist = nullptr;
	ctx->lane_capacity = 0;
	DMS_CUDA(ctx, cudaMalloc(&ctx->d_lane_hist, sizeof(double2) * DMS_NUM_BINS * lanes));
	DMS_CUDA(ctx, cudaMemset(ctx->d_lane_hist, 0, sizeof(double2) * DMS_NUM_BINS * lanes));
	ctx->lane_capacity = lanes;
	return DMS_OK;
}

int Ensure_Init(dms_ctx* ctx, uint64_t total)
{
	if(total <= ctx->init_capacity)
		return DMS_OK;
	cudaFree(ctx->d_init);
	ctx->d_init = nullptr;
	ctx->init_capacity = 0;
	const uint64_t cap = std::max<uint64_t>(total, 1 << 16);
	DMS_CUDA(ctx, cudaMalloc(&ctx->d_init, sizeof(InitState) * cap));
	ctx->init_capacity = cap;
	return DMS_OK;
}

int Check_Run_Opts(dms_ctx* ctx, const dms_run_opts* o)
{
	if(!o)
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "null run options");
	if(!(o->boundary_radius_rsun > 0.0) || !std::isfinite(o->boundary_radius_rsun))
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "boundary radius must be finite and positive");
	if(o->precision != DMS_PRECISION_FP64 && o->precision != DMS_PRECISION_MIXED)
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "unsupported precision");
	if(o->threads_per_block != 0 && (o->threads_per_block % 32 != 0 || o->threads_per_block > 128))
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "threads_per_block must be a multiple of 32 up to 128");
	if(o->queue_chunk > 1024)
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "queue_chunk must be at most 1024");
	if(o->scatter_batch > 32 || o->final_batch > 32 || o->scatter_wait > 1024 || o->final_wait > 1024)
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "warp batching: batches up to 32 lanes, waits up to 1024 iterations");
	return DMS_OK;
}

// The lane-scheduling options of a launch (dms_run_opts, 0 = default).
void Apply_Lane_Options(RunParams& p, const dms_run_opts* o)
{
	p.queue_chunk = o->queue_chunk ? o->queue_chunk : 1u;
	p.scatter_batch = o->scatter_batch ? static_cast<int>(o->scatter_batch) : 16;
	p.scatter_wait = o->scatter_wait ? static_cast<int>(o->scatter_wait) : 32;
	p.final_batch = o->final_batch ? static_cast<int>(o->final_batch) : 8;
	p.final_wait = o->final_wait ? static_cast<int>(o->final_wait) : 32;
}

// One persistent launch over the given work; polls for completion, enforcing the wall-clock
// limit through the mapped cancel flag.
int Launch_And_Wait(dms_ctx* ctx, const dms_run_opts* o, RunParams& p)
{
	if(!(o->max_trajectory_wall_time_s >= 0.0) || !std::isfinite(o->max_trajectory_wall_time_s))
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "'max_trajectory_wall_time_sec' must be finite and non-negative");
	p.wall_limit_ns = static_cast<uint64_t>(o->max_trajectory_wall_time_s * 1.0e9);
	if(o->max_trajectory_wall_time_s > 0.0 && p.wall_limit_ns == 0)
		p.wall_limit_ns = 1;
	Apply_Lane_Options(p, o);
	const int threads = o->threads_per_block ? static_cast<int>(o->threads_per_block) : 128;
	const bool mixed = o->precision == DMS_PRECISION_MIXED;
	const int max_per_sm = mixed ? Trajectory_Mixed_Max_Blocks_Per_SM(threads) : Trajectory_Max_Blocks_Per_SM(threads);
	if(max_per_sm <= 0)
		return Fail(ctx, DMS_ERR_CUDA, "trajectory kernel cannot be resident with this block size");
	int per_sm = o->blocks_per_sm ? static_cast<int>(o->blocks_per_sm) : max_per_sm;
	per_sm = per_sm > max_per_sm ? max_per_sm : per_sm;
	int blocks = ctx->sm_count * per_sm;
	const uint64_t needed_blocks = (p.total + threads - 1) / threads;
	if(static_cast<uint64_t>(blocks) > needed_blocks)
		blocks = static_cast<int>(std::max<uint64_t>(1, needed_blocks));
	const size_t lanes = static_cast<size_t>(blocks) * threads;
	int rc = Ensure_Lanes(ctx, lanes);
	if(rc != DMS_OK)
		return rc;
	rc = Ensure_Init(ctx, p.total);
	if(rc != DMS_OK)
		return rc;
	p.lane_hist = ctx->d_lane_hist;
	p.init = ctx->d_init;
	p.queue_head = ctx->d_queue;
	p.status = ctx->d_status;
	p.cancel = ctx->d_cancel;
	p.seed = o->seed;
	p.capture_mode = o->capture_mode ? 1 : 0;
	p.max_scatterings = o->max_scatterings;
	p.max_free_steps = o->max_free_steps;
	p.boundary = o->boundary_radius_rsun * DMS_RSUN_KM;
	p.iteration_budget = o->iteration_budget ? o->iteration_budget : ~0ULL;
	p.ic_max_attempts = 1 << 20;
	p.S = ctx->dsolar;
	p.points = ctx->d_points;
	p.n_points = static_cast<int>(ctx->points.size());
	if(mixed)
	{
		for(size_t i = 0; i < ctx->points.size(); i++)
			if(!ctx->grid_f_valid[i])
			{
				const size_t n = static_cast<size_t>(ctx->points[i].grid_n);
				Launch_To_Float(ctx->d_grids[i], ctx->d_grids_f[i], n * n, ctx->stream);
				DMS_CUDA(ctx, cudaGetLastError());
				ctx->grid_f_valid[i] = 1;
			}
		p.sf_r = ctx->d_tables_f;
		p.sf_gm = ctx->d_tables_f + ctx->dsolar.n;
		p.sf_gm_s = ctx->d_tables_f + 2 * static_cast<size_t>(ctx->dsolar.n);
		p.sf_vesc2 = ctx->d_tables_f + 3 * static_cast<size_t>(ctx->dsolar.n);
		p.sf_vesc2_s = ctx->d_tables_f + 4 * static_cast<size_t>(ctx->dsolar.n);
	}
#ifdef DMS_CHECKED
	// bits left by a launch that does not report them (dms_run_records_noalloc) are dropped
	(void)(mixed ? Take_Bounds_Status_Mixed() : Take_Bounds_Status());
#endif
	*ctx->h_cancel = 0;
	DMS_CUDA(ctx, cudaMemsetAsync(ctx->d_queue, 0, sizeof(unsigned long long), ctx->stream));
	DMS_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(unsigned int), ctx->stream));
	// one NVTX range per launch, so that a profiler timeline shows each trajectory launch
	const std::string range = std::string(mixed ? "dms mixed launch: " : "dms fp64 launch: ") + std::to_string(p.total) + " trajectories";
	nvtxRangePushA(range.c_str());
	struct Pop
	{
		~Pop() { nvtxRangePop(); }
	} pop;
	DMS_CUDA(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
	Launch_Initial_States(p, ctx->stream);
	DMS_CUDA(ctx, cudaGetLastError());
	if(mixed)
		Launch_Trajectories_Mixed(p, blocks, threads, ctx->stream);
	else
		Launch_Trajectories(p, blocks, threads, ctx->stream);
	DMS_CUDA(ctx, cudaGetLastError());
	DMS_CUDA(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
	const auto start = std::chrono::steady_clock::now();
	ctx->running = true;
	ctx->launch_total = p.total;
	ctx->launch_start = start;
	auto last_progress = start;
	bool cancelled_by_limit = false, cancelled_by_hook = false;
	for(;;)
	{
		const cudaError_t q = cudaStreamQuery(ctx->stream);
		if(q == cudaSuccess)
			break;
		if(q != cudaErrorNotReady)
		{
			ctx->running = false;
			return Fail(ctx, DMS_ERR_CUDA, std::string("trajectory kernel: ") + cudaGetErrorString(q));
		}
		const auto now = std::chrono::steady_clock::now();
		if(o->time_limit_s > 0.0 && !cancelled_by_limit)
		{
			const double el = std::chrono::duration<double>(now - start).count();
			if(el > o->time_limit_s)
			{
				*reinterpret_cast<volatile int*>(ctx->h_cancel) = 1;
				cancelled_by_limit = true;
			}
		}
		if(ctx->progress_fn && !cancelled_by_hook && std::chrono::duration<double>(now - last_progress).count() >= ctx->progress_interval_s)
		{
			last_progress = now;
			if(ctx->progress_fn(ctx, ctx->progress_user) != 0)
			{
				*reinterpret_cast<volatile int*>(ctx->h_cancel) = 1;
				cancelled_by_hook = true;
			}
		}
		std::this_thread::sleep_for(std::chrono::microseconds(200));
	}
	ctx->running = false;
	float kernel_ms = 0.0f;
	DMS_CUDA(ctx, cudaEventElapsedTime(&kernel_ms, ctx->ev_start, ctx->ev_stop));
	ctx->last_kernel_ms = kernel_ms;
	unsigned int status = 0;
	DMS_CUDA(ctx, cudaMemcpy(&status, ctx->d_status, sizeof status, cudaMemcpyDeviceToHost));
	if(status & STATUS_CANCELLED)
		return Fail(ctx, DMS_ERR_CANCELLED, cancelled_by_limit ? "run cancelled: wall-clock limit reached"
		                                    : cancelled_by_hook ? "run cancelled by the progress callback" : "run cancelled");
	if(status & STATUS_BUDGET)
		return Fail(ctx, DMS_ERR_BUDGET, "run stopped: per-lane iteration budget exhausted");
	if(status & STATUS_IC_REJECTION)
		ctx->error = "warning: an initial-condition rejection loop hit its attempt bound";
#ifdef DMS_CHECKED
	const unsigned int bounds = mixed ? Take_Bounds_Status_Mixed() : Take_Bounds_Status();
	if(bounds != 0)
		return Fail(ctx, DMS_ERR_STATE, "checked build: an index left its bounds (bits " + std::to_string(bounds) + ")");
#endif
	return DMS_OK;
}

void Fill_Dev_Point(const PointConstants& c, double* grid, DevPoint& d)
{
	std::memset(&d, 0, sizeof d);
	d.m_dm = c.m_dm;
	d.sigma_e = c.sigma_e;
	d.v0 = c.v0;
	d.vesc_halo = c.vesc_halo;
	d.vobs = c.vobs;
	for(int i = 0; i < 3; i++) d.vel_obs[i] = c.vel_obs[i];
	d.n_esc = c.n_esc;
	d.avg_speed = c.avg_speed;
	d.eta0 = c.eta0;
	d.grid_inv_r = c.grid_inv_r;
	d.grid_inv_v = c.grid_inv_v;
	d.grid_vmax = c.grid_vmax;
	d.grid = grid;
	d.grid_n = c.grid_n;
	for(int k = 0; k < DMS_NUM_TARGETS; k++) d.sigma_t[k] = c.sigma_target[k];
	d.interaction = static_cast<int>(c.interaction);
	d.ff_num = c.ff_num;
	d.ff_m2 = c.ff_m2;
	for(int k = 0; k <= DMS_NUM_TARGETS; k++) d.q2c[k] = c.q2c[k];
}
}	// namespace

extern "C" {

int dms_create(dms_ctx** out, int device)
{
	if(!out)
		return DMS_ERR_INVALID_ARGUMENT;
	*out = nullptr;
	dms_ctx* ctx = new(std::nothrow) dms_ctx();
	if(!ctx)
		return DMS_ERR_CAPACITY;
	int count = 0;
	cudaError_t e = cudaGetDeviceCount(&count);
	if(e != cudaSuccess || device < 0 || device >= count)
	{
		delete ctx;
		return DMS_ERR_CUDA;
	}
	ctx->device = device;
	if(cudaSetDevice(device) != cudaSuccess || cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
	   cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
	   cudaStreamCreateWithFlags(&ctx->peek_stream, cudaStreamNonBlocking) != cudaSuccess ||
	   cudaMalloc(&ctx->d_queue, sizeof(unsigned long long)) != cudaSuccess || cudaMalloc(&ctx->d_status, sizeof(unsigned int)) != cudaSuccess ||
	   cudaHostAlloc(&ctx->h_cancel, sizeof(int), cudaHostAllocMapped) != cudaSuccess ||
	   cudaHostGetDevicePointer(reinterpret_cast<void**>(&ctx->d_cancel), ctx->h_cancel, 0) != cudaSuccess ||
	   cudaEventCreate(&ctx->ev_start) != cudaSuccess || cudaEventCreate(&ctx->ev_stop) != cudaSuccess)
	{
		dms_destroy(ctx);
		return DMS_ERR_CUDA;
	}
	*ctx->h_cancel = 0;
	*out = ctx;
	return DMS_OK;
}

void dms_destroy(dms_ctx* ctx)
{
	if(!ctx)
		return;
	cudaSetDevice(ctx->device);
	if(ctx->stream)
		cudaStreamSynchronize(ctx->stream);
	for(double* g : ctx->d_grids) cudaFree(g);
	for(float* g : ctx->d_grids_f) cudaFree(g);
	cudaFree(ctx->d_init);
	cudaFree(ctx->d_tables_f);
	cudaFree(ctx->d_tables);
	cudaFree(ctx->d_points);
	cudaFree(ctx->d_counters);
	cudaFree(ctx->d_hists);
	cudaFree(ctx->d_events);
	cudaFree(ctx->d_event_count);
	cudaFree(ctx->d_refl);
	cudaFree(ctx->d_refl_count);
	cudaFree(ctx->d_lane_hist);
	cudaFree(ctx->d_queue);
	cudaFree(ctx->d_status);
	if(ctx->h_cancel)
		cudaFreeHost(ctx->h_cancel);
	if(ctx->ev_start)
		cudaEventDestroy(ctx->ev_start);
	if(ctx->ev_stop)
		cudaEventDestroy(ctx->ev_stop);
	if(ctx->stream)
		cudaStreamDestroy(ctx->stream);
	if(ctx->peek_stream)
		cudaStreamDestroy(ctx->peek_stream);
	delete ctx;
}

const char* dms_last_error(const dms_ctx* ctx) { return ctx ? ctx->error.c_str() : "null context"; }

int dms_cancel(dms_ctx* ctx)
{
	if(!ctx || !ctx->h_cancel)
		return DMS_ERR_INVALID_ARGUMENT;
	*reinterpret_cast<volatile int*>(ctx->h_cancel) = 1;
	return DMS_OK;
}

int dms_num_bins(void) { return DMS_NUM_BINS; }

int dms_measure_fp64_peak(dms_ctx* ctx, double* tflops)
{
	if(!ctx || !tflops)
		return DMS_ERR_INVALID_ARGUMENT;
	DMS_NOT_IN_FLIGHT(ctx);
	DMS_CUDA(ctx, cudaSetDevice(ctx->device));
	const double t = Measure_FP64_Peak(ctx->sm_count, ctx->stream);
	if(!(t > 0.0))
		return Fail(ctx, DMS_ERR_CUDA, "FP64 peak probe failed");
	*tflops = t;
	return DMS_OK;
}

int dms_check_certified_math(dms_ctx* ctx, uint64_t n, uint64_t seed, uint64_t* counts)
{
	if(!ctx || !counts)
		return DMS_ERR_INVALID_ARGUMENT;
	DMS_NOT_IN_FLIGHT(ctx);
	DMS_CUDA(ctx, cudaSetDevice(ctx->device));
	unsigned long long* d = nullptr;
	DMS_CUDA(ctx, cudaMalloc(&d, 4 * sizeof(unsigned long long)));
	struct Free
	{
		void* p;
		~Free() { cudaFree(p); }
	} f{d};
	DMS_CUDA(ctx, cudaMemsetAsync(d, 0, 4 * sizeof(unsigned long long), ctx->stream));
	Check_Certified_Math(n, seed, d, ctx->sm_count, ctx->stream);
	DMS_CUDA(ctx, cudaGetLastError());
	unsigned long long h[4];
	DMS_CUDA(ctx, cudaMemcpyAsync(h, d, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
	DMS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
	for(int i = 0; i < 4; i++) counts[i] = h[i];
	return DMS_OK;
}

int dms_last_kernel_ms(const dms_ctx* ctx, double* ms)
{
	if(!ctx || !ms)
		return DMS_ERR_INVALID_ARGUMENT;
	*ms = ctx->last_kernel_ms;
	return DMS_OK;
}

int dms_load_solar_model(dms_ctx* ctx, const char* path)
{
	if(!ctx || !path)
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "null argument");
	DMS_NOT_IN_FLIGHT(ctx);
	DMS_CUDA(ctx, cudaSetDevice(ctx->device));
	SolarTables t;
	const std::string err = Load_Solar_Tables(path, t);
	if(!err.empty())
		return Fail(ctx, DMS_ERR_IO, err);
	const size_t n = t.n, nt = static_cast<size_t>(t.n) * DMS_NUM_TARGETS;
	const size_t doubles = 9 * n + 2 * nt + DMS_NUM_TARGETS;
	const size_t bytes = doubles * sizeof(double) + sizeof(uint16_t) * t.bucket_index.size();
	std::vector<char> host(bytes);
	double* h = reinterpret_cast<double*>(host.data());
	const std::vector<double>* parts[11] = {&t.r, &t.gm, &t.gm_s, &t.temp, &t.temp_s, &t.vesc2, &t.vesc2_s, &t.ne, &t.ne_s, &t.nt, &t.nt_s};
	size_t offsets[11];
	size_t off = 0;
	for(int k = 0; k < 11; k++)
	{
		offsets[k] = off;
		std::memcpy(h + off, parts[k]->data(), parts[k]->size() * sizeof(double));
		off += parts[k]->size();
	}
	const size_t off_mass = off;
	std::memcpy(h + off, t.target_mass_gev, sizeof(double) * DMS_NUM_TARGETS);
	off += DMS_NUM_TARGETS;
	std::memcpy(h + off, t.bucket_index.data(), sizeof(uint16_t) * t.bucket_index.size());
	void* d = nullptr;
	DMS_CUDA(ctx, cudaMalloc(&d, bytes));
	const cudaError_t ce = cudaMemcpy(d, host.data(), bytes, cudaMemcpyHostToDevice);
	if(ce != cudaSuccess)
	{
		cudaFree(d);
		return Fail(ctx, DMS_ERR_CUDA, std::string("table upload: ") + cudaGetErrorString(ce));
	}
	cudaFree(ctx->d_tables);
	ctx->d_tables = d;
	const double* dd = reinterpret_cast<const double*>(d);
	DevSolar& S = ctx->dsolar;
	S.n = t.n;
	S.nbuckets = t.nbuckets;
	S.bucket_single_step = t.bucket_single_step;
	S.bucket_scale = static_cast<double>(t.nbuckets) / DMS_RSUN_KM;
	S.r = dd + offsets[0];
	S.gm = dd + offsets[1];
	S.gm_s = dd + offsets[2];
	S.temp = dd + offsets[3];
	S.temp_s = dd + offsets[4];
	S.vesc2 = dd + offsets[5];
	S.vesc2_s = dd + offsets[6];
	S.ne = dd + offsets[7];
	S.ne_s = dd + offsets[8];
	S.nt = dd + offsets[9];
	S.nt_s = dd + offsets[10];
	S.target_mass = dd + off_mass;
	S.bucket = reinterpret_cast<const uint16_t*>(dd + off);
	// FP32 images of the tables the mixed-precision kernel reads every step: knots, G*M and
	// v_esc^2 with their slopes
	std::vector<float> hf(5 * n);
	for(size_t i = 0; i < n; i++)
	{
		hf[i] = static_cast<float>(t.r[i]);
		hf[n + i] = static_cast<float>(t.gm[i]);
		hf[2 * n + i] = static_cast<float>(t.gm_s[i]);
		hf[3 * n + i] = static_cast<float>(t.vesc2[i]);
		hf[4 * n + i] = static_cast<float>(t.vesc2_s[i]);
	}
	float* df = nullptr;
	DMS_CUDA(ctx, cudaMalloc(&df, sizeof(float) * hf.size()));
	const cudaError_t cf = cudaMemcpy(df, hf.data(), sizeof(float) * hf.size(), cudaMemcpyHostToDevice);
	if(cf != cudaSuccess)
	{
		cudaFree(df);
		return Fail(ctx, DMS_ERR_CUDA, std::string("table upload: ") + cudaGetErrorString(cf));
	}
	cudaFree(ctx->d_tables_f);
	ctx->d_tables_f = df;
	ctx->tables = std::move(t);
	ctx->has_solar = true;
	return DMS_OK;
}

int dms_solar_table(dms_ctx* ctx, int which, double* out, size_t capacity)
{
	if(!ctx)
		return DMS_ERR_INVALID_ARGUMENT;
	if(!ctx->has_solar)
		return Fail(ctx, DMS_ERR_NO_SOLAR_MODEL, "no solar model loaded");
	const DevSolar& S = ctx->dsolar;
	const double* src = nullptr;
	size_t n = S.n;
	switch(which)
	{
		case 0: src = S.r; break;
		case 1: src = S.gm; break;
		case 2: src = S.temp; break;
		case 3: src = S.vesc2; break;
		case 4: src = S.ne; break;
		case 5:
			src = S.nt;
			n = static_cast<size_t>(S.n) * DMS_NUM_TARGETS;
			break;
		default: return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "unknown table");
	}
	if(out)
	{
		if(capacity < n)
			return Fail(ctx, DMS_ERR_CAPACITY, "output buffer too small");
		DMS_CUDA(ctx, cudaMemcpy(out, src, n * sizeof(double), cudaMemcpyDeviceToHost));
	}
	return static_cast<int>(n);
}

int dms_add_point(dms_ctx* ctx, const dms_point_params* params, int* point_id)
{
	if(!ctx || !params)
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "null argument");
	DMS_NOT_IN_FLIGHT(ctx);
	if(!ctx->has_solar)
		return Fail(ctx, DMS_ERR_NO_SOLAR_MODEL, "load a solar model before adding points");
	if(static_cast<int>(ctx->points.size()) >= MAX_POINTS)
		return Fail(ctx, DMS_ERR_CAPACITY, "too many parameter points");
	DMS_CUDA(ctx, cudaSetDevice(ctx->device));
	PointConstants c;
	const std::string err = Make_Point_Constants(ctx->tables, *params, c);
	if(!err.empty())
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, err);
	const int id = static_cast<int>(ctx->points.size());
	int rc = Grow_Points(ctx, id + 1);
	if(rc != DMS_OK)
		return rc;
	double* grid = nullptr;
	float* grid_f = nullptr;
	if(c.grid_n > 0)  // interpolation_points < 2: no grid, rates are computed per lookup
	{
		DMS_CUDA(ctx, cudaMalloc(&grid, sizeof(double) * c.grid_n * c.grid_n));
		const cudaError_t e0 = cudaMalloc(&grid_f, sizeof(float) * c.grid_n * c.grid_n);
		if(e0 != cudaSuccess)
		{
			cudaFree(grid);
			return Fail(ctx, DMS_ERR_CUDA, cudaGetErrorString(e0));
		}
	}
	DevPoint d;
	Fill_Dev_Point(c, grid, d);
	d.grid_f = grid_f;
	const cudaError_t e1 = cudaMemcpy(ctx->d_points + id, &d, sizeof d, cudaMemcpyHostToDevice);
	if(e1 != cudaSuccess)
	{
		cudaFree(grid);
		cudaFree(grid_f);
		return Fail(ctx, DMS_ERR_CUDA, cudaGetErrorString(e1));
	}
	if(c.grid_n > 0)
		Launch_Rate_Grid(ctx->dsolar, ctx->d_points + id, grid, c.grid_n, ctx->stream);
	const cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
	if(e2 != cudaSuccess || cudaGetLastError() != cudaSuccess)
	{
		cudaFree(grid);
		cudaFree(grid_f);
		return Fail(ctx, DMS_ERR_CUDA, std::string("rate grid kernel: ") + cudaGetErrorString(e2));
	}
	ctx->points.push_back(c);
	ctx->d_grids.push_back(grid);
	ctx->d_grids_f.push_back(grid_f);
	ctx->grid_f_valid.push_back(c.grid_n > 0 ? 0 : 1);
	DMS_CUDA(ctx, cudaMemset(ctx->d_counters + static_cast<size_t>(id) * DMS_NUM_COUNTERS, 0, sizeof(unsigned long long) * DMS_NUM_COUNTERS));
	DMS_CUDA(ctx, cudaMemset(ctx->d_hists + static_cast<size_t>(id) * DMS_NUM_HISTS * DMS_NUM_BINS, 0, sizeof(double) * DMS_NUM_HISTS * DMS_NUM_BINS));
	DMS_CUDA(ctx, cudaMemset(ctx->d_event_count + id, 0, sizeof(unsigned long long)));
	DMS_CUDA(ctx, cudaMemset(ctx->d_refl_count + id, 0, sizeof(unsigned long long)));
	if(point_id)
		*point_id = id;
	return DMS_OK;
}

int dms_num_points(const dms_ctx* ctx) { return ctx ? static_cast<int>(ctx->points.size()) : 0; }

int dms_set_rate_grid(dms_ctx* ctx, int point_id, const double* grid, uint32_t n)
{
	if(!ctx || !grid)
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "null argument");
	DMS_NOT_IN_FLIGHT(ctx);
	if(point_id < 0 || point_id >= static_cast<int>(ctx->points.size()))
		return Fail(ctx, DMS_ERR_NO_POINT, "no such point");
	if(ctx->points[point_id].grid_n == 0)
		return Fail(ctx, DMS_ERR_STATE, "the point has no rate grid (interpolation_points < 2)");
	if(static_cast<int>(n) != ctx->points[point_id].grid_n)
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "grid size does not match the point's interpolation_points");
	DMS_CUDA(ctx, cudaMemcpy(ctx->d_grids[point_id], grid, sizeof(double) * n * n, cudaMemcpyHostToDevice));
	ctx->grid_f_valid[point_id] = 0;
	return DMS_OK;
}

int dms_get_rate_grid(dms_ctx* ctx, int point_id, double* grid, uint32_t n)
{
	if(!ctx || !grid)
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "null argument");
	if(point_id < 0 || point_id >= static_cast<int>(ctx->points.size()))
		return Fail(ctx, DMS_ERR_NO_POINT, "no such point");
	if(ctx->points[point_id].grid_n == 0)
		return Fail(ctx, DMS_ERR_STATE, "the point has no rate grid (interpolation_points < 2)");
	if(static_cast<int>(n) != ctx->points[point_id].grid_n)
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "grid size does not match the point's interpolation_points");
	DMS_CUDA(ctx, cudaMemcpy(grid, ctx->d_grids[point_id], sizeof(double) * n * n, cudaMemcpyDeviceToHost));
	return DMS_OK;
}

int dms_rate(dms_ctx* ctx, int point_id, int interpolated, const double* r_km, const double* v_kms, double* rate_out, size_t n)
{
	if(!ctx || (n > 0 && (!r_km || !v_kms || !rate_out)))
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "null argument");
	DMS_NOT_IN_FLIGHT(ctx);
	if(point_id < 0 || point_id >= static_cast<int>(ctx->points.size()))
		return Fail(ctx, DMS_ERR_NO_POINT, "no such point");
	if(n == 0)
		return DMS_OK;
	double* d = nullptr;
	DMS_CUDA(ctx, cudaMalloc(&d, sizeof(double) * 3 * n));
	cudaError_t e = cudaMemcpy(d, r_km, sizeof(double) * n, cudaMemcpyHostToDevice);
	if(e == cudaSuccess)
		e = cudaMemcpy(d + n, v_kms, sizeof(double) * n, cudaMemcpyHostToDevice);
	if(e == cudaSuccess)
	{
		Launch_Rate_Query(ctx->dsolar, ctx->d_points + point_id, interpolated, d, d + n, d + 2 * n, n, ctx->stream);
		e = cudaStreamSynchronize(ctx->stream);
	}
	if(e == cudaSuccess)
		e = cudaMemcpy(rate_out, d + 2 * n, sizeof(double) * n, cudaMemcpyDeviceToHost);
	cudaFree(d);
	if(e != cudaSuccess)
		return Fail(ctx, DMS_ERR_CUDA, std::string("rate query: ") + cudaGetErrorString(e));
	return DMS_OK;
}

void dms_default_run_opts(dms_run_opts* o)
{
	if(!o)
		return;
	std::memset(o, 0, sizeof *o);
	o->seed = 1;
	o->capture_mode = 0;
	o->max_scatterings = 100000000000000ULL;   // DEFAULT_MAXIMUM_SCATTERINGS
	o->max_free_steps = 1000000000000ULL;      // DEFAULT_MAXIMUM_FREE_TIME_STEPS
	o->boundary_radius_rsun = 2.0;
	o->precision = DMS_PRECISION_FP64;
}

int dms_run(dms_ctx* ctx, const dms_run_opts* opts, const dms_work_range* ranges, int n_ranges)
{
	if(!ctx)
		return DMS_ERR_INVALID_ARGUMENT;
	DMS_NOT_IN_FLIGHT(ctx);
	int rc = Check_Run_Opts(ctx, opts);
	if(rc != DMS_OK)
		return rc;
	if(n_ranges <= 0 || !ranges)
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "no work ranges");
	DMS_CUDA(ctx, cudaSetDevice(ctx->device));
	std::vector<int32_t> pts(n_ranges);
	std::vector<uint64_t> firsts(n_ranges), offsets(n_ranges + 1);
	uint64_t total = 0;
	for(int k = 0; k < n_ranges; k++)
	{
		if(ranges[k].point_id < 0 || ranges[k].point_id >= static_cast<int>(ctx->points.size()))
			return Fail(ctx, DMS_ERR_NO_POINT, "work range names an unknown point");
		pts[k] = ranges[k].point_id;
		firsts[k] = ranges[k].first_trajectory;
		offsets[k] = total;
		total += ranges[k].count;
	}
	offsets[n_ranges] = total;
	if(total == 0)
		return DMS_OK;
	std::vector<char> buf(sizeof(int32_t) * n_ranges + sizeof(uint64_t) * (2 * n_ranges + 1) + 16);
	void* d = nullptr;
	DMS_CUDA(ctx, cudaMalloc(&d, buf.size()));
	char* dc = static_cast<char*>(d);
	const size_t off_first = 0, off_offset = sizeof(uint64_t) * n_ranges, off_point = sizeof(uint64_t) * (2 * n_ranges + 1);
	std::memcpy(buf.data() + off_first, firsts.data(), sizeof(uint64_t) * n_ranges);
	std::memcpy(buf.data() + off_offset, offsets.data(), sizeof(uint64_t) * (n_ranges + 1));
	std::memcpy(buf.data() + off_point, pts.data(), sizeof(int32_t) * n_ranges);
	cudaError_t e = cudaMemcpy(d, buf.data(), buf.size(), cudaMemcpyHostToDevice);
	if(e != cudaSuccess)
	{
		cudaFree(d);
		return Fail(ctx, DMS_ERR_CUDA, cudaGetErrorString(e));
	}
	RunParams p{};
	p.range_first = reinterpret_cast<const uint64_t*>(dc + off_first);
	p.range_offset = reinterpret_cast<const uint64_t*>(dc + off_offset);
	p.range_point = reinterpret_cast<const int32_t*>(dc + off_point);
	p.n_ranges = n_ranges;
	p.total = total;
	p.counters = ctx->d_counters;
	p.hists = ctx->d_hists;
	p.events = ctx->d_events;
	p.event_count = ctx->d_event_count;
	p.event_capacity = ctx->event_capacity;
	p.reflections = ctx->d_refl;
	p.reflection_count = ctx->d_refl_count;
	rc = Launch_And_Wait(ctx, opts, p);
	cudaFree(d);
	return rc;
}

// ---- autotuner ------------------------------------------------------------------------------
namespace
{
// One trial of the autotuner: a launch stopped after `seconds` over fresh ids (from 2^40) of the
// given points, its results in the scratch accumulators `scratch`; returns accepted free steps
// per second (finished and unfinished trajectories), or a negative value on failure.
struct TuneScratch
{
	unsigned long long* counters = nullptr;
	double* hists = nullptr;
	dms_evaporation_event* events = nullptr;
	unsigned long long* event_count = nullptr;
	dms_reflection* refl = nullptr;
	unsigned long long* refl_count = nullptr;
	uint64_t capacity = 256;
	void Free()
	{
		cudaFree(counters);
		cudaFree(hists);
		cudaFree(events);
		cudaFree(event_count);
		cudaFree(refl);
		cudaFree(refl_count);
	}
};

double Tune_Trial(dms_ctx* ctx, const dms_run_opts& o, const std::vector<int32_t>& pts, uint64_t per_point, uint64_t first,
                  const TuneScratch& t, void* d_ranges)
{
	const int n = static_cast<int>(pts.size());
	const size_t np = ctx->points.size();
	if(cudaMemsetAsync(t.counters, 0, sizeof(unsigned long long) * DMS_NUM_COUNTERS * np, ctx->stream) != cudaSuccess ||
	   cudaMemsetAsync(t.event_count, 0, sizeof(unsigned long long) * np, ctx->stream) != cudaSuccess ||
	   cudaMemsetAsync(t.refl_count, 0, sizeof(unsigned long long) * np, ctx->stream) != cudaSuccess)
		return -1.0;
	std::vector<uint64_t> firsts(n, first), offsets(n + 1);
	for(int k = 0; k <= n; k++) offsets[k] = per_point * static_cast<uint64_t>(k);
	char* dc = static_cast<char*>(d_ranges);
	const size_t off_offset = sizeof(uint64_t) * n, off_point = sizeof(uint64_t) * (2 * n + 1);
	std::vector<char> buf(off_point + sizeof(int32_t) * n);
	std::memcpy(buf.data(), firsts.data(), sizeof(uint64_t) * n);
	std::memcpy(buf.data() + off_offset, offsets.data(), sizeof(uint64_t) * (n + 1));
	std::memcpy(buf.data() + off_point, pts.data(), sizeof(int32_t) * n);
	if(cudaMemcpy(d_ranges, buf.data(), buf.size(), cudaMemcpyHostToDevice) != cudaSuccess)
		return -1.0;
	RunParams p{};
	p.range_first = reinterpret_cast<const uint64_t*>(dc);
	p.range_offset = reinterpret_cast<const uint64_t*>(dc + off_offset);
	p.range_point = reinterpret_cast<const int32_t*>(dc + off_point);
	p.n_ranges = n;
	p.total = per_point * static_cast<uint64_t>(n);
	p.counters = t.counters;
	p.hists = t.hists;
	p.events = t.events;
	p.event_count = t.event_count;
	p.event_capacity = t.capacity;
	p.reflections = t.refl;
	p.reflection_count = t.refl_count;
	const int rc = Launch_And_Wait(ctx, &o, p);
	if(rc != DMS_OK && rc != DMS_ERR_CANCELLED)
		return -1.0;
	std::vector<unsigned long long> c(DMS_NUM_COUNTERS * np);
	if(cudaMemcpy(c.data(), t.counters, sizeof(unsigned long long) * c.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
		return -1.0;
	double steps = 0.0;
	for(int32_t pt : pts)
	{
		const unsigned long long* q = c.data() + static_cast<size_t>(pt) * DMS_NUM_COUNTERS;
		steps += static_cast<double>(q[DMS_CNT_RK_STEPS] + q[DMS_CNT_UNFINISHED_RK_STEPS]);
	}
	return ctx->last_kernel_ms > 0.0 ? steps / (ctx->last_kernel_ms * 1.0e-3) : -1.0;
}
}	// namespace

int dms_autotune(dms_ctx* ctx, const dms_run_opts* base, const dms_work_range* ranges, int n_ranges, double trial_seconds,
                 dms_run_opts* tuned, int* trials)
{
	if(!ctx)
		return DMS_ERR_INVALID_ARGUMENT;
	DMS_NOT_IN_FLIGHT(ctx);
	int rc = Check_Run_Opts(ctx, base);
	if(rc != DMS_OK)
		return rc;
	if(!tuned || n_ranges <= 0 || !ranges || !(trial_seconds > 0.0) || trial_seconds > 60.0)
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "autotune: ranges, an output and a trial time in (0, 60] s are required");
	std::vector<int32_t> pts;
	for(int k = 0; k < n_ranges; k++)
	{
		if(ranges[k].point_id < 0 || ranges[k].point_id >= static_cast<int>(ctx->points.size()))
			return Fail(ctx, DMS_ERR_NO_POINT, "work range names an unknown point");
		if(std::find(pts.begin(), pts.end(), ranges[k].point_id) == pts.end())
			pts.push_back(ranges[k].point_id);
	}
	DMS_CUDA(ctx, cudaSetDevice(ctx->device));
	const size_t np = ctx->points.size();
	TuneScratch t;
	struct Guard
	{
		TuneScratch& t;
		void* ranges = nullptr;
		~Guard()
		{
			t.Free();
			cudaFree(ranges);
		}
	} guard{t};
	DMS_CUDA(ctx, cudaMalloc(&t.counters, sizeof(unsigned long long) * DMS_NUM_COUNTERS * np));
	DMS_CUDA(ctx, cudaMalloc(&t.hists, sizeof(double) * DMS_NUM_HISTS * DMS_NUM_BINS * np));
	DMS_CUDA(ctx, cudaMalloc(&t.events, sizeof(dms_evaporation_event) * t.capacity * np));
	DMS_CUDA(ctx, cudaMalloc(&t.event_count, sizeof(unsigned long long) * np));
	DMS_CUDA(ctx, cudaMalloc(&t.refl, sizeof(dms_reflection) * t.capacity * np));
	DMS_CUDA(ctx, cudaMalloc(&t.refl_count, sizeof(unsigned long long) * np));
	DMS_CUDA(ctx, cudaMalloc(&guard.ranges, (sizeof(uint64_t) * 2 + sizeof(int32_t)) * (pts.size() + 1)));
	// enough ids that no trial drains its queue: a million per point, fresh for every trial
	const uint64_t per_point = 1ULL << 20;
	dms_run_opts best = *base;
	best.time_limit_s = trial_seconds;
	best.iteration_budget = 0;
	int n_trials = 0;
	uint64_t next_first = 1ULL << 40;
	auto score = [&](const dms_run_opts& o) {
		n_trials++;
		const double v = Tune_Trial(ctx, o, pts, per_point, next_first, t, guard.ranges);
		next_first += per_point;
		return v;
	};
	double best_score = score(best);
	if(!(best_score > 0.0))
		return Fail(ctx, DMS_ERR_CUDA, "autotune: the first trial launch failed");
	struct Knob
	{
		uint32_t dms_run_opts::*field;
		std::vector<uint32_t> values;
	};
	const std::vector<Knob> knobs = {
		{&dms_run_opts::threads_per_block, {64, 96, 128}},
		{&dms_run_opts::blocks_per_sm, {2, 3, 4}},
		{&dms_run_opts::queue_chunk, {1, 2, 4}},
		{&dms_run_opts::scatter_batch, {8, 16, 24, 32}},
		{&dms_run_opts::scatter_wait, {16, 32, 64, 128}},
		{&dms_run_opts::final_batch, {4, 8, 16}},
		{&dms_run_opts::final_wait, {16, 32, 64}},
	};
	// coordinate descent: a value replaces the current one only when it is at least 2 % faster
	// (the run-to-run spread of a short trial)
	for(int pass = 0; pass < 2; pass++)
	{
		bool changed = false;
		for(const Knob& k : knobs)
			for(uint32_t v : k.values)
			{
				if(best.*(k.field) == v)
					continue;
				dms_run_opts trial = best;
				trial.*(k.field) = v;
				const double sc = score(trial);
				if(sc > 1.02 * best_score)
				{
					best = trial;
					best_score = sc;
					changed = true;
				}
			}
		if(!changed)
			break;
	}
	*tuned = *base;
	tuned->threads_per_block = best.threads_per_block;
	tuned->blocks_per_sm = best.blocks_per_sm;
	tuned->queue_chunk = best.queue_chunk;
	tuned->scatter_batch = best.scatter_batch;
	tuned->scatter_wait = best.scatter_wait;
	tuned->final_batch = best.final_batch;
	tuned->final_wait = best.final_wait;
	if(trials)
		*trials = n_trials;
	return DMS_OK;
}

int dms_run_records(dms_ctx* ctx, const dms_run_opts* opts, int point_id, uint64_t first, uint64_t count, dms_traj_record* records,
                    double* hist_dt, double* hist_v2dt)
{
	if(!ctx)
		return DMS_ERR_INVALID_ARGUMENT;
	DMS_NOT_IN_FLIGHT(ctx);
	int rc = Check_Run_Opts(ctx, opts);
	if(rc != DMS_OK)
		return rc;
	if(point_id < 0 || point_id >= static_cast<int>(ctx->points.size()))
		return Fail(ctx, DMS_ERR_NO_POINT, "no such point");
	if(count == 0)
		return DMS_OK;
	if(!records || ((hist_dt == nullptr) != (hist_v2dt == nullptr)))
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "records buffer required; histograms need both buffers");
	DMS_CUDA(ctx, cudaSetDevice(ctx->device));
	const bool want_hist = hist_dt != nullptr;
	const size_t hist_bytes = want_hist ? sizeof(double) * DMS_NUM_BINS * count : 0;
	const size_t rec_bytes = sizeof(dms_traj_record) * count;
	const size_t meta = 64;
	char* d = nullptr;
	DMS_CUDA(ctx, cudaMalloc(reinterpret_cast<void**>(&d), meta + rec_bytes + 2 * hist_bytes));
	struct Meta
	{
		uint64_t first, off0, off1;
		int32_t point;
	} m{first, 0, count, point_id};
	cudaError_t e = cudaMemcpy(d, &m, sizeof m, cudaMemcpyHostToDevice);
	if(e == cudaSuccess)
		e = cudaMemset(d + meta, 0, rec_bytes + 2 * hist_bytes);
	if(e != cudaSuccess)
	{
		cudaFree(d);
		return Fail(ctx, DMS_ERR_CUDA, cudaGetErrorString(e));
	}
	RunParams p{};
	p.range_first = reinterpret_cast<const uint64_t*>(d);
	p.range_offset = reinterpret_cast<const uint64_t*>(d + 8);
	p.range_point = reinterpret_cast<const int32_t*>(d + 24);
	p.n_ranges = 1;
	p.total = count;
	p.records = reinterpret_cast<dms_traj_record*>(d + meta);
	p.rec_hist_dt = want_hist ? reinterpret_cast<double*>(d + meta + rec_bytes) : nullptr;
	p.rec_hist_v2dt = want_hist ? reinterpret_cast<double*>(d + meta + rec_bytes + hist_bytes) : nullptr;
	p.counters = ctx->d_counters;
	p.hists = ctx->d_hists;
	p.events = ctx->d_events;
	p.event_count = ctx->d_event_count;
	p.event_capacity = ctx->event_capacity;
	p.reflections = ctx->d_refl;
	p.reflection_count = ctx->d_refl_count;
	rc = Launch_And_Wait(ctx, opts, p);
	if(rc == DMS_OK || rc == DMS_ERR_CANCELLED || rc == DMS_ERR_BUDGET)
	{
		e = cudaMemcpy(records, d + meta, rec_bytes, cudaMemcpyDeviceToHost);
		if(e == cudaSuccess && want_hist)
			e = cudaMemcpy(hist_dt, d + meta + rec_bytes, hist_bytes, cudaMemcpyDeviceToHost);
		if(e == cudaSuccess && want_hist)
			e = cudaMemcpy(hist_v2dt, d + meta + rec_bytes + hist_bytes, hist_bytes, cudaMemcpyDeviceToHost);
		if(e != cudaSuccess)
			rc = Fail(ctx, DMS_ERR_CUDA, cudaGetErrorString(e));
	}
	cudaFree(d);
	return rc;
}

int dms_get_results(dms_ctx* ctx, int point_id, dms_point_results* r)
{
	if(!ctx || !r)
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "null argument");
	if(point_id < 0 || point_id >= static_cast<int>(ctx->points.size()))
		return Fail(ctx, DMS_ERR_NO_POINT, "no such point");
	DMS_CUDA(ctx, cudaSetDevice(ctx->device));
	DMS_CUDA(ctx, cudaMemcpy(r->counters, ctx->d_counters + static_cast<size_t>(point_id) * DMS_NUM_COUNTERS,
	                         sizeof(unsigned long long) * DMS_NUM_COUNTERS, cudaMemcpyDeviceToHost));
	if(r->histograms)
		DMS_CUDA(ctx, cudaMemcpy(r->histograms, ctx->d_hists + static_cast<size_t>(point_id) * DMS_NUM_HISTS * DMS_NUM_BINS,
		                         sizeof(double) * DMS_NUM_HISTS * DMS_NUM_BINS, cudaMemcpyDeviceToHost));
	unsigned long long count = 0;
	DMS_CUDA(ctx, cudaMemcpy(&count, ctx->d_event_count + point_id, sizeof count, cudaMemcpyDeviceToHost));
	r->events_count = std::min<uint64_t>(count, ctx->event_capacity);
	if(r->events && r->events_capacity > 0)
	{
		const uint64_t n = std::min<uint64_t>(r->events_count, r->events_capacity);
		if(n > 0)
			DMS_CUDA(ctx, cudaMemcpy(r->events, ctx->d_events + static_cast<size_t>(point_id) * ctx->event_capacity,
			                         sizeof(dms_evaporation_event) * n, cudaMemcpyDeviceToHost));
	}
	unsigned long long nrefl = 0;
	DMS_CUDA(ctx, cudaMemcpy(&nrefl, ctx->d_refl_count + point_id, sizeof nrefl, cudaMemcpyDeviceToHost));
	r->reflections_count = std::min<uint64_t>(nrefl, ctx->event_capacity);
	if(r->reflections && r->reflections_capacity > 0)
	{
		const uint64_t n = std::min<uint64_t>(r->reflections_count, r->reflections_capacity);
		if(n > 0)
			DMS_CUDA(ctx, cudaMemcpy(r->reflections, ctx->d_refl + static_cast<size_t>(point_id) * ctx->event_capacity,
			                         sizeof(dms_reflection) * n, cudaMemcpyDeviceToHost));
	}
	return DMS_OK;
}

int dms_reset_results(dms_ctx* ctx, int point_id)
{
	if(!ctx)
		return DMS_ERR_INVALID_ARGUMENT;
	DMS_NOT_IN_FLIGHT(ctx);
	if(point_id < 0 || point_id >= static_cast<int>(ctx->points.size()))
		return Fail(ctx, DMS_ERR_NO_POINT, "no such point");
	DMS_CUDA(ctx, cudaSetDevice(ctx->device));
	DMS_CUDA(ctx, cudaMemset(ctx->d_counters + static_cast<size_t>(point_id) * DMS_NUM_COUNTERS, 0, sizeof(unsigned long long) * DMS_NUM_COUNTERS));
	DMS_CUDA(ctx, cudaMemset(ctx->d_hists + static_cast<size_t>(point_id) * DMS_NUM_HISTS * DMS_NUM_BINS, 0, sizeof(double) * DMS_NUM_HISTS * DMS_NUM_BINS));
	DMS_CUDA(ctx, cudaMemset(ctx->d_event_count + point_id, 0, sizeof(unsigned long long)));
	DMS_CUDA(ctx, cudaMemset(ctx->d_refl_count + point_id, 0, sizeof(unsigned long long)));
	DMS_CUDA(ctx, cudaMemset(ctx->d_events + static_cast<size_t>(point_id) * ctx->event_capacity, 0,
	                         sizeof(dms_evaporation_event) * ctx->event_capacity));
	return DMS_OK;
}

int dms_set_progress_callback(dms_ctx* ctx, dms_progress_fn fn, void* user, double interval_s)
{
	if(!ctx)
		return DMS_ERR_INVALID_ARGUMENT;
	if(fn && !(interval_s >= 0.0 && interval_s < 1e9))
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "progress interval must be finite and non-negative");
	ctx->progress_fn = fn;
	ctx->progress_user = fn ? user : nullptr;
	ctx->progress_interval_s = fn ? interval_s : 1.0;
	return DMS_OK;
}

int dms_peek_progress(dms_ctx* ctx, dms_progress* out)
{
	if(!ctx || !out)
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "null argument");
	std::memset(out, 0, sizeof *out);
	DMS_CUDA(ctx, cudaSetDevice(ctx->device));
	unsigned long long head = 0;
	DMS_CUDA(ctx, cudaMemcpyAsync(&head, ctx->d_queue, sizeof head, cudaMemcpyDeviceToHost, ctx->peek_stream));
	DMS_CUDA(ctx, cudaStreamSynchronize(ctx->peek_stream));
	out->running = ctx->running ? 1 : 0;
	out->total = ctx->launch_total;
	out->dispatched = std::min<uint64_t>(head, ctx->launch_total);
	out->elapsed_s = ctx->running ? std::chrono::duration<double>(std::chrono::steady_clock::now() - ctx->launch_start).count() : 0.0;
	return DMS_OK;
}

int dms_peek_results(dms_ctx* ctx, int point_id, dms_point_results* r)
{
	if(!ctx || !r)
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "null argument");
	if(point_id < 0 || point_id >= static_cast<int>(ctx->points.size()))
		return Fail(ctx, DMS_ERR_NO_POINT, "no such point");
	DMS_CUDA(ctx, cudaSetDevice(ctx->device));
	cudaStream_t s = ctx->peek_stream;
	unsigned long long count = 0;
	DMS_CUDA(ctx, cudaMemcpyAsync(r->counters, ctx->d_counters + static_cast<size_t>(point_id) * DMS_NUM_COUNTERS,
	                              sizeof(unsigned long long) * DMS_NUM_COUNTERS, cudaMemcpyDeviceToHost, s));
	if(r->histograms)
		DMS_CUDA(ctx, cudaMemcpyAsync(r->histograms, ctx->d_hists + static_cast<size_t>(point_id) * DMS_NUM_HISTS * DMS_NUM_BINS,
		                              sizeof(double) * DMS_NUM_HISTS * DMS_NUM_BINS, cudaMemcpyDeviceToHost, s));
	DMS_CUDA(ctx, cudaMemcpyAsync(&count, ctx->d_event_count + point_id, sizeof count, cudaMemcpyDeviceToHost, s));
	DMS_CUDA(ctx, cudaStreamSynchronize(s));
	r->events_count = std::min<uint64_t>(count, ctx->event_capacity);
	r->reflections_count = 0;
	if(r->events && r->events_capacity > 0)
	{
		const uint64_t n = std::min<uint64_t>(r->events_count, r->events_capacity);
		if(n > 0)
		{
			DMS_CUDA(ctx, cudaMemcpyAsync(r->events, ctx->d_events + static_cast<size_t>(point_id) * ctx->event_capacity,
			                              sizeof(dms_evaporation_event) * n, cudaMemcpyDeviceToHost, s));
			DMS_CUDA(ctx, cudaStreamSynchronize(s));
		}
		uint64_t k = 0;
		while(k < n && r->events[k].trajectory_id != 0)
			k++;
		r->events_count = k;
	}
	return DMS_OK;
}

}	// extern "C"

// ---- dms_run_records_noalloc -----------------------------------------------------------------
// Callers that cannot allocate device memory while they run trajectories: a host whose own
// caching allocator reserved the device's memory up front, or a service that fixes its memory
// budget before any work arrives and must not fail on an allocation later.  For them this
// entry point writes into the caller's device buffers and keeps its scratch in the array
// below, which is part of the library's device image: every device that loads the library
// holds these DMS_NOALLOC_SCRATCH_BYTES (4 104 448 bytes, about 3.9 MiB) until the process exits.
//
// Scratch layout (bytes): 0 work-queue head (u64), 8 status word (u32), 64 range start (u64),
// 72 range offsets {0, count} (2 x u64), 96 range point (i32); from 256 the initial states
// (64 bytes per trajectory); after them one 2000-bin (dt, v2dt) histogram row per lane,
// DMS_NOALLOC_MAX_TRAJECTORIES of each.
static __device__ __align__(256) unsigned char dms_noalloc_scratch[DMS_NOALLOC_SCRATCH_BYTES];

namespace
{
constexpr size_t NOALLOC_HEADER = 256;
constexpr size_t NOALLOC_ROWS = NOALLOC_HEADER + sizeof(InitState) * DMS_NOALLOC_MAX_TRAJECTORIES;
static_assert(DMS_NOALLOC_SCRATCH_BYTES == NOALLOC_ROWS + sizeof(double2) * DMS_NUM_BINS * DMS_NOALLOC_MAX_TRAJECTORIES,
              "scratch size must match its layout");

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};

// Address of the scratch array on the context's device (current), looked up once per device
// and kept for the life of the process.  A device reset (cudaDeviceReset) between calls would
// leave the kept address stale; the header states that such a reset is not supported.
int Noalloc_Scratch(dms_ctx* ctx, unsigned char** out)
{
	if(ctx->device < 0 || ctx->device >= NOALLOC_MAX_DEVICES)
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "dms_run_records_noalloc: device index out of range");
	std::lock_guard<std::mutex> lock(g_noalloc_mutex);
	if(g_noalloc_ptr[ctx->device] == nullptr)
	{
		unsigned char* ptr = nullptr;
		const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&ptr), dms_noalloc_scratch);
		if(e != cudaSuccess || ptr == nullptr)
			return Fail(ctx, DMS_ERR_CUDA, std::string("dms_run_records_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
		g_noalloc_ptr[ctx->device] = ptr;
	}
	*out = g_noalloc_ptr[ctx->device];
	return DMS_OK;
}

// The array keeps whatever the previous call left, so this clears everything the trajectory
// kernel expects to start at zero (queue head, status word, the lane rows in use) and the
// caller's outputs (records, histogram rows), and writes the work range.
__global__ void noalloc_prepare_kernel(unsigned char* scratch, uint64_t first, uint64_t count, int point, uint64_t lanes,
                                       unsigned char* records, double* hist_dt, double* hist_v2dt)
{
	const uint64_t tid = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
	const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	if(tid == 0)
	{
		*reinterpret_cast<unsigned long long*>(scratch + 0) = 0ULL;
		*reinterpret_cast<unsigned int*>(scratch + 8) = 0u;
		*reinterpret_cast<uint64_t*>(scratch + 64) = first;
		reinterpret_cast<uint64_t*>(scratch + 72)[0] = 0;
		reinterpret_cast<uint64_t*>(scratch + 72)[1] = count;
		*reinterpret_cast<int32_t*>(scratch + 96) = point;
	}
	double2* rows = reinterpret_cast<double2*>(scratch + NOALLOC_ROWS);
	for(uint64_t k = tid; k < lanes * DMS_NUM_BINS; k += stride) rows[k] = make_double2(0.0, 0.0);
	for(uint64_t k = tid; k < count * sizeof(dms_traj_record); k += stride) records[k] = 0;
	if(hist_dt != nullptr)
		for(uint64_t k = tid; k < count * DMS_NUM_BINS; k += stride)
		{
			hist_dt[k] = 0.0;
			hist_v2dt[k] = 0.0;
		}
}
}	// namespace

extern "C" {

int dms_run_records_noalloc(dms_ctx* ctx, const dms_run_opts* opts, int point_id, uint64_t first, uint64_t count,
                            dms_traj_record* d_records, double* d_hist_dt, double* d_hist_v2dt)
{
	if(!ctx)
		return DMS_ERR_INVALID_ARGUMENT;
	// from a progress callback this would clear the outer launch's cancel flag, re-record its
	// timing events and block the outer wait loop behind the running kernel
	DMS_NOT_IN_FLIGHT(ctx);
	int rc = Check_Run_Opts(ctx, opts);
	if(rc != DMS_OK)
		return rc;
	if(!(opts->max_trajectory_wall_time_s >= 0.0) || !std::isfinite(opts->max_trajectory_wall_time_s))
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "'max_trajectory_wall_time_sec' must be finite and non-negative");
	if(point_id < 0 || point_id >= static_cast<int>(ctx->points.size()))
		return Fail(ctx, DMS_ERR_NO_POINT, "no such point");
	if(count > DMS_NOALLOC_MAX_TRAJECTORIES)
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT,
		            "dms_run_records_noalloc: " + std::to_string(count) + " trajectories requested, at most " +
		                std::to_string(DMS_NOALLOC_MAX_TRAJECTORIES) + " fit the fixed device scratch of one call");
	if(count == 0)
		return DMS_OK;
	if(!d_records || ((d_hist_dt == nullptr) != (d_hist_v2dt == nullptr)))
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "records buffer required; histograms need both buffers");
	DMS_CUDA(ctx, cudaSetDevice(ctx->device));
	unsigned char* scratch = nullptr;
	rc = Noalloc_Scratch(ctx, &scratch);
	if(rc != DMS_OK)
		return rc;
	const int threads = 32;
	const int blocks = static_cast<int>((count + threads - 1) / threads);
	const uint64_t lanes = static_cast<uint64_t>(blocks) * threads;

	RunParams p{};
	p.S = ctx->dsolar;
	p.points = ctx->d_points;
	p.n_points = static_cast<int>(ctx->points.size());
	p.range_first = reinterpret_cast<const uint64_t*>(scratch + 64);
	p.range_offset = reinterpret_cast<const uint64_t*>(scratch + 72);
	p.range_point = reinterpret_cast<const int32_t*>(scratch + 96);
	p.n_ranges = 1;
	p.total = count;
	p.queue_head = reinterpret_cast<unsigned long long*>(scratch + 0);
	p.status = reinterpret_cast<unsigned int*>(scratch + 8);
	p.lane_hist = reinterpret_cast<double2*>(scratch + NOALLOC_ROWS);
	p.init = reinterpret_cast<InitState*>(scratch + NOALLOC_HEADER);
	p.seed = opts->seed;
	p.capture_mode = opts->capture_mode ? 1 : 0;
	p.max_scatterings = opts->max_scatterings;
	p.max_free_steps = opts->max_free_steps;
	p.boundary = opts->boundary_radius_rsun * DMS_RSUN_KM;
	p.iteration_budget = opts->iteration_budget ? opts->iteration_budget : ~0ULL;
	p.wall_limit_ns = static_cast<uint64_t>(opts->max_trajectory_wall_time_s * 1.0e9);
	if(opts->max_trajectory_wall_time_s > 0.0 && p.wall_limit_ns == 0)
		p.wall_limit_ns = 1;
	p.ic_max_attempts = 1 << 20;
	Apply_Lane_Options(p, opts);
	p.counters = ctx->d_counters;
	p.hists = ctx->d_hists;
	p.events = ctx->d_events;
	p.event_count = ctx->d_event_count;
	p.event_capacity = ctx->event_capacity;
	p.reflections = ctx->d_refl;
	p.reflection_count = ctx->d_refl_count;
	p.records = d_records;
	p.rec_hist_dt = d_hist_dt;
	p.rec_hist_v2dt = d_hist_v2dt;
	p.cancel = ctx->d_cancel;

#ifdef DMS_CHECKED
	(void)Take_Bounds_Status();   // bits of an earlier launch are not this call's
#endif
	*ctx->h_cancel = 0;
	noalloc_prepare_kernel<<<8, 256, 0, ctx->stream>>>(scratch, first, count, point_id, lanes, reinterpret_cast<unsigned char*>(d_records),
	                                                   d_hist_dt, d_hist_v2dt);
	DMS_CUDA(ctx, cudaGetLastError());
	DMS_CUDA(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
	Launch_Initial_States(p, ctx->stream);
	DMS_CUDA(ctx, cudaGetLastError());
	Launch_Trajectories(p, blocks, threads, ctx->stream);
	DMS_CUDA(ctx, cudaGetLastError());
	DMS_CUDA(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
	const auto start = std::chrono::steady_clock::now();
	bool cancelled_by_limit = false;
	for(;;)
	{
		const cudaError_t q = cudaStreamQuery(ctx->stream);
		if(q == cudaSuccess)
			break;
		if(q != cudaErrorNotReady)
			return Fail(ctx, DMS_ERR_CUDA, std::string("trajectory kernel: ") + cudaGetErrorString(q));
		if(opts->time_limit_s > 0.0 && !cancelled_by_limit &&
		   std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count() > opts->time_limit_s)
		{
			*reinterpret_cast<volatile int*>(ctx->h_cancel) = 1;
			cancelled_by_limit = true;
		}
		std::this_thread::sleep_for(std::chrono::microseconds(200));
	}
	float kernel_ms = 0.0f;
	DMS_CUDA(ctx, cudaEventElapsedTime(&kernel_ms, ctx->ev_start, ctx->ev_stop));
	ctx->last_kernel_ms = kernel_ms;
	unsigned int status = 0;
	DMS_CUDA(ctx, cudaMemcpy(&status, scratch + 8, sizeof status, cudaMemcpyDeviceToHost));
	if(status & STATUS_CANCELLED)
		return Fail(ctx, DMS_ERR_CANCELLED, cancelled_by_limit ? "run cancelled: wall-clock limit reached" : "run cancelled");
	if(status & STATUS_BUDGET)
		return Fail(ctx, DMS_ERR_BUDGET, "run stopped: per-lane iteration budget exhausted");
	if(status & STATUS_IC_REJECTION)
		ctx->error = "warning: an initial-condition rejection loop hit its attempt bound";
#ifdef DMS_CHECKED
	const unsigned int bounds = Take_Bounds_Status();
	if(bounds != 0)
		return Fail(ctx, DMS_ERR_STATE, "checked build: an index left its bounds (bits " + std::to_string(bounds) + ")");
#endif
	return DMS_OK;
}

}	// extern "C"

// ---- reflection spectrum -----------------------------------------------------------------
namespace
{
// Isoreflection_Ring_Angles (src/Simulation_Utilities.cpp:323-336): upper angles of n
// equal-area rings around the Sun's velocity
std::vector<double> Ring_Angles(uint32_t rings)
{
	std::vector<double> a;
	double theta = 0.0;
	for(uint32_t i = 0; i + 1 < rings; i++)
	{
		theta = std::acos(std::cos(theta) - 2.0 / rings);
		a.push_back(theta);
	}
	a.push_back(DMS_PI);
	return a;
}

// Speeds of the recorded reflected particles of one ring
int Ring_Speeds(dms_ctx* ctx, int point_id, uint32_t rings, uint32_t ring, std::vector<double>& speeds, uint64_t& trajectories)
{
	if(rings == 0 || ring >= rings)
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "isoreflection ring out of range");
	dms_point_results res;
	std::memset(&res, 0, sizeof res);
	int rc = dms_get_results(ctx, point_id, &res);
	if(rc != DMS_OK)
		return rc;
	std::vector<dms_reflection> all(res.reflections_count);
	res.reflections = all.data();
	res.reflections_capacity = all.size();
	rc = dms_get_results(ctx, point_id, &res);
	if(rc != DMS_OK)
		return rc;
	trajectories = res.counters[DMS_CNT_TRAJECTORIES];
	const std::vector<double> angles = Ring_Angles(rings);
	speeds.clear();
	for(const dms_reflection& r : all)
	{
		uint32_t k = 0;
		if(rings > 1)
		{
			const double c = r.cos_sun_velocity < -1.0 ? -1.0 : (r.cos_sun_velocity > 1.0 ? 1.0 : r.cos_sun_velocity);
			const double theta = std::acos(c);
			while(k + 1 < rings && theta > angles[k]) k++;
		}
		if(k == ring)
			speeds.push_back(r.speed_kms);
	}
	return DMS_OK;
}
}	// namespace

extern "C" {

int dms_get_reflection_spectrum(dms_ctx* ctx, int point_id, uint32_t rings, uint32_t ring, double dm_density_gev_cm3,
                                dms_reflection_spectrum* out)
{
	if(!ctx || !out)
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "null argument");
	if(point_id < 0 || point_id >= static_cast<int>(ctx->points.size()))
		return Fail(ctx, DMS_ERR_NO_POINT, "no such point");
	std::vector<double> speeds;
	uint64_t trajectories = 0;
	const int rc = Ring_Speeds(ctx, point_id, rings, ring, speeds, trajectories);
	if(rc != DMS_OK)
		return rc;
	const PointConstants& c = ctx->points[point_id];
	std::memset(out, 0, sizeof *out);
	out->trajectories = trajectories;
	out->reflections = speeds.size();
	out->reflection_ratio = trajectories > 0 ? static_cast<double>(speeds.size()) / trajectories : 0.0;
	// DM_Entering_Rate, src/Reflection_Spectrum.cpp:63-71: number density in 1/km^3, R_sun in km
	const double n_dm = dm_density_gev_cm3 / c.m_dm * 1.0e15;
	const double vesc2 = ctx->tables.vesc2.back();  // v_esc^2 at R_sun
	out->entering_rate_per_s = DMS_RSUN_KM * DMS_RSUN_KM * DMS_PI * n_dm * (c.avg_speed + vesc2 * c.eta0);
	out->reflection_rate_per_s = out->reflection_ratio * out->entering_rate_per_s;
	out->distance_au = 1.0;
	const double d_cm = DMS_AU_KM * 1.0e5;
	out->flux_per_s_cm2 = out->reflection_rate_per_s / (4.0 * DMS_PI * d_cm * d_cm) * rings;
	double vmax = 0.0, sum = 0.0;
	for(double v : speeds)
	{
		vmax = std::max(vmax, v);
		sum += v;
	}
	out->speed_min_kms = 0.0;  // 0.75 x the minimum speed threshold u_min = 0 of the run modes
	out->speed_max_kms = 1.05 * vmax;
	out->mean_speed_kms = speeds.empty() ? 0.0 : sum / speeds.size();
	return DMS_OK;
}

int dms_reflection_spectrum_pdf(dms_ctx* ctx, int point_id, uint32_t rings, uint32_t ring, const double* u_kms, size_t n, double* pdf)
{
	if(!ctx || (n > 0 && (!u_kms || !pdf)))
		return Fail(ctx, DMS_ERR_INVALID_ARGUMENT, "null argument");
	if(point_id < 0 || point_id >= static_cast<int>(ctx->points.size()))
		return Fail(ctx, DMS_ERR_NO_POINT, "no such point");
	std::vector<double> speeds;
	uint64_t trajectories = 0;
	const int rc = Ring_Speeds(ctx, point_id, rings, ring, speeds, trajectories);
	if(rc != DMS_OK)
		return rc;
	const size_t m = speeds.size();
	if(m < 2)
	{
		for(size_t i = 0; i < n; i++) pdf[i] = 0.0;
		return DMS_OK;
	}
	std::sort(speeds.begin(), speeds.end());
	double mean = 0.0, var = 0.0, vmax = speeds.back();
	for(double v : speeds) mean += v;
	mean /= m;
	for(double v : speeds) var += (v - mean) * (v - mean);
	const double sigma = std::sqrt(var / (m - 1));
	const double iqr = speeds[(3 * m) / 4] - speeds[m / 4];
	const double spread = iqr > 0.0 ? std::min(sigma, iqr / 1.34) : sigma;
	const double h = 0.9 * spread * std::pow(static_cast<double>(m), -0.2);
	const double lo = 0.0, hi = 1.05 * vmax;
	const double norm = 1.0 / (m * h * std::sqrt(2.0 * DMS_PI));
	for(size_t i = 0; i < n; i++)
	{
		const double u = u_kms[i];
		if(!(u >= lo && u <= hi) || !(h > 0.0))
		{
			pdf[i] = 0.0;
			continue;
		}
		double s = 0.0;
		for(double v : speeds)
		{
			const double a = (u - v) / h, b = (u + v - 2.0 * lo) / h;  // kernel and its mirror at lo
			s += std::exp(-0.5 * a * a) + std::exp(-0.5 * b * b);
		}
		pdf[i] = s * norm;
	}
	return DMS_OK;
}

int dms_print_reflection_summary(const dms_reflection_spectrum* s)
{
	if(!s)
		return DMS_ERR_INVALID_ARGUMENT;
	// Reflection_Spectrum::Print_Summary, src/Reflection_Spectrum.cpp:47-59
	const char* sep = "\n----------------------------------------\n";
	std::cout << sep << "Reflection spectrum" << std::endl
	          << "\tSpeed domain [km/sec]:\t\t\t[" << s->speed_min_kms << ", " << s->speed_max_kms << "]" << std::endl
	          << "\tReflected particles:\t\t\t" << s->reflections << " of " << s->trajectories << std::endl
	          << "\tMean speed at 1 AU [km/sec]:\t\t" << s->mean_speed_kms << std::endl
	          << "\tTotal DM entering rate [1/s]:\t\t" << s->entering_rate_per_s << std::endl
	          << "\tTotal reflection rate [1/s]:\t\t" << s->reflection_rate_per_s << std::endl
	          << "\tDistance from Sun [AU]:\t\t\t" << s->distance_au << std::endl
	          << "\tTotal reflection flux [1/s/cm^2]:\t" << s->flux_per_s_cm2 << sep;
	return DMS_OK;
}

}	// extern "C"
