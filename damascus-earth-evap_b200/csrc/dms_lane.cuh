// Lane state machine shared by the FP64 and the mixed-precision trajectory kernels: lane state,
// work claims, trajectory start, free-segment start, capture bookkeeping, termination and
// aggregation.  The free step itself (the Propagate_Freely loop body) is supplied by each form.
#pragma once

#include <type_traits>

#include "dms_kernels.cuh"

namespace dms
{
namespace lane
{

enum Phase : int
{
	PH_FETCH = 0,
	PH_SEGMENT = 1,
	PH_STEP = 2,
	PH_FINAL = 3,
	PH_DONE = 4,
	PH_SCATTER = 5,  // the committed event L.cur is a scattering point inside the Sun
};


// Trajectory state of a lane (TrajectoryBincount + Trajectory_Simulator members,
// include/Simulation_Trajectory.hpp:53-154).
template <class PropT, class EvT>
struct LaneT
{
	// the FP64 form bins by the reference's division; the mixed form multiplies by the
	// reciprocal bin width (a bin edge can then move by one ulp)
	static constexpr bool exact_bins = std::is_same<PropT, Prop>::value;
	uint64_t work;
	int point;
	Draws D;
	Event cur;           // absolute event at segment boundaries and at termination
	PropT pr;            // propagator of the current free segment (local time)
	EvT before;          // Event_In_3D of the propagator at the start of the step (cached)
	double origin;       // absolute time of the segment's local t = 0
	double tau;          // remaining optical depth to the next scattering (minus_log_xi)
	uint64_t seg_steps;
	uint64_t nscat;
	uint64_t steps;      // accepted free steps of the whole trajectory (work counter)
	uint64_t attempts;   // RK45 attempts of the whole trajectory (work counter)
	unsigned int retries;
	int before_valid;
	int in_rk;           // an RK45 step is in progress (retry pending)
	int rk_inner;        // passes of the current RK45 step
	double rate_before;  // scattering rate at the start of the step
	int next_valid;      // next_speed / next_rate hold the propagator's speed and rate (FP64 form, tail)
	double next_speed, next_rate;
	double b_time, b_radius, b_phi, b_vr, b_step;  // propagator fields at the start of the step
	int shift_ok;
	int reason;
	// capture / evaporation state
	int is_captured;
	int bound_state;
	double t_capture, t_last_bound, t_final_unbinding;
	double free_flight_E;
	double max_drift_eV, max_drift_rel;
	// bincount anchor (left-endpoint rule)
	double prev_time, prev_r, prev_v2;
	int bmin, bmax;
	// the bin being visited, held in registers until the trajectory leaves it
	int cbin;
	double2 cval;
	uint64_t wall_start;  // %globaltimer at the start of the trajectory (wall-clock limit only)
};
// Nanoseconds of the device's global timer, one clock for every SM.
__device__ __forceinline__ uint64_t global_timer_ns()
{
	uint64_t t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

// abort_if_wall_time_exceeded, src/Simulation_Trajectory.cpp:824-840: the trajectory's wall time
// since it started on its lane against max_trajectory_wall_time_sec (0 = no limit)
template <class Lane>
__device__ __forceinline__ bool wall_time_exceeded(const RunParams& R, const Lane& L)
{
	return R.wall_limit_ns != 0 && global_timer_ns() - L.wall_start > R.wall_limit_ns;
}

template <class Lane>
__device__ __forceinline__ void accumulate_bincount(Lane& L, double2* hist, double r, double v2, double dt)
{
	// Accumulate_Bincount_Step, src/Simulation_Trajectory.cpp:640-669
	if(!isfinite(dt) || dt <= 0.0)
		return;
	int bin = -1;
	if(isfinite(r) && r >= 0.0 && r < DMS_BIN_MAX_KM)
	{
		if constexpr(Lane::exact_bins)
			bin = static_cast<int>(r / DMS_BIN_WIDTH_KM);
		else
			bin = static_cast<int>(r * (1.0 / DMS_BIN_WIDTH_KM));
		if(bin < 0) bin = 0;
		if(bin >= DMS_NUM_BINS) bin = -1;
	}
	if(bin >= 0)
	{
		DMS_CHECK_INDEX(bin, 0, DMS_NUM_BINS, BOUNDS_BIN);
		// The row is read only when a visited bin is entered again and written when it is
		// left; the additions are the reference's, in its order.
		if(bin != L.cbin)
		{
			if(L.cbin >= 0)
				hist[L.cbin] = L.cval;
			L.cval = (bin >= L.bmin && bin <= L.bmax) ? hist[bin] : make_double2(0.0, 0.0);
			L.cbin = bin;
			L.bmin = bin < L.bmin ? bin : L.bmin;
			L.bmax = bin > L.bmax ? bin : L.bmax;
		}
		L.cval.x += dt;
		L.cval.y += v2 * dt;
	}
}

// Writes the bin being visited back to the lane's row (before the row is read out).
template <class Lane>
__device__ __forceinline__ void write_back_bin(Lane& L, double2* hist)
{
	if(L.cbin >= 0)
		hist[L.cbin] = L.cval;
	L.cbin = -1;
}

// Update_Capture_State, src/Simulation_Trajectory.cpp:689-760
template <class Lane>
__device__ __forceinline__ bool update_capture_state(const DevSolar& S, double m_dm, int capture_mode, Lane& L, double r, double v, double t, bool allow_new)
{
	if(capture_mode && !allow_new && !L.is_captured)
		return false;
	const double E = capture_energy_eV(S, m_dm, r, v);
	const bool negative = E < 0.0;
	if(!allow_new)
	{
		if(L.is_captured && isfinite(L.free_flight_E))
		{
			const double drift = fabs(E - L.free_flight_E);
			if(isfinite(drift) && drift > L.max_drift_eV)
				L.max_drift_eV = drift;
			const double ref = fabs(L.free_flight_E);
			const double scale = ref > DMS_FREE_ENERGY_DRIFT_REL_E_SCALE_EV ? ref : DMS_FREE_ENERGY_DRIFT_REL_E_SCALE_EV;
			const double rel = drift / scale;
			if(isfinite(rel) && rel > L.max_drift_rel)
				L.max_drift_rel = rel;
		}
		if(L.bound_state && L.is_captured)
			L.t_last_bound = t;
		return false;
	}
	const int was_bound = L.bound_state;
	L.bound_state = negative;
	L.free_flight_E = E;
	if(negative)
	{
		if(!L.is_captured)
		{
			L.is_captured = 1;
			L.t_capture = t;
			L.t_last_bound = t;
		}
		else if(!was_bound)
			L.t_final_unbinding = NAN;
		L.t_last_bound = t;
		return true;
	}
	if(was_bound && L.is_captured)
		L.t_final_unbinding = t;
	return false;
}

template <class Lane>
__device__ __forceinline__ bool uncaptured_bound(const DevSolar& S, double m_dm, const Lane& L, const Event& e)
{
	if(L.is_captured)
		return false;
	const double E = capture_energy_eV(S, m_dm, ev_radius(e), ev_speed(e));
	if(isfinite(E) && E >= 0.0)
		return false;
	return true;
}

template <class Lane>
__device__ __forceinline__ void set_final(Lane& L, const Event& local_or_abs, bool is_local, int reason)
{
	L.cur = local_or_abs;
	if(is_local)
		L.cur.t += L.origin;
	L.reason = reason;
}

__device__ __forceinline__ void init_propagator(Prop& p, const Event& e) { prop_init(p, e); }

// Start of a free segment: Simulate loop head + Propagate_Freely prologue,
// src/Simulation_Trajectory.cpp:1311-1313, 762-805
template <class Lane>
__device__ __forceinline__ int segment_start(const RunParams& R, const DevPoint* __restrict__ P, double m_dm, Lane& L)
{
	if(!(L.nscat < R.max_scatterings))
	{
		L.reason = DMS_REASON_MAX_SCATTERINGS;
		return PH_FINAL;
	}
	if(outward_escaping(R.S, L.cur, R.boundary))
	{
		L.reason = DMS_REASON_OUTWARD_ESCAPE;
		return PH_FINAL;
	}
	if(uncaptured_bound(R.S, m_dm, L, L.cur))
	{
		L.reason = DMS_REASON_NUMERICAL_FAILURE;
		return PH_FINAL;
	}
	L.origin = L.cur.t;
	Event local = L.cur;
	local.t = 0.0;
	init_propagator(L.pr, local);
	L.tau = -dms_log(L.D.positive_unit());
	L.seg_steps = 0;
	L.retries = 0;
	L.before_valid = 0;
	L.next_valid = 0;
	L.in_rk = 0;
	if(!R.capture_mode && L.prev_time >= 0.0)
		L.prev_time = 0.0;
	return PH_STEP;
}

__device__ __forceinline__ bool is_numerical_termination(int r)
{
	return r == DMS_REASON_NUMERICAL_FAILURE || r == DMS_REASON_NON_FINITE_STATE || r == DMS_REASON_SPEED_LIMIT ||
	       r == DMS_REASON_ENERGY_DRIFT_ESCAPE || r == DMS_REASON_UNKNOWN;
}

__device__ __forceinline__ bool is_computational_truncation(int r)
{
	return r == DMS_REASON_WALL_TIME_LIMIT || r == DMS_REASON_MAX_FREE_STEPS || r == DMS_REASON_MAX_SCATTERINGS;
}

// Termination: tail of Simulate (src/Simulation_Trajectory.cpp:1349-1399), classification and
// aggregation of simulate_one_trajectory (src/Data_Generation.cpp:745-861).
// The lane's histogram row still to be moved out at termination: copied into the record's
// histograms (records mode) or added with its squares to the per-point sums (accumulate mode),
// and zeroed either way.  Executed by the whole warp (cooperative_flush).
struct FlushJob
{
	double* dst0;  // records: dt row; accumulate: sum of dt
	double* dst1;  // records: v2dt row; accumulate: sum of v2dt
	double* dst2;  // accumulate: sum of dt^2
	double* dst3;  // accumulate: sum of v2dt^2
	int b0, b1;    // touched bins; b1 < b0 when there is nothing to do
	int mode;      // FLUSH_ZERO, FLUSH_COPY or FLUSH_ADD
};
constexpr int FLUSH_ZERO = 0, FLUSH_COPY = 1, FLUSH_ADD = 2;

template <class Lane>
__device__ __noinline__ void finalize(const RunParams& R, const DevPoint* __restrict__ P, double m_dm, Lane& L, FlushJob& job)
{
	const DevSolar& S = R.S;
	int reason = L.reason;
	int survival_valid = 1, event_observed = 0, boundary_escape = 0, invalid_escape = 0;
	double t_boundary = NAN;
	const double t_term = L.cur.t;
	uint32_t flags = 0;
	if(L.shift_ok)
	{
		flags |= DMS_REC_SHIFT_OK;
		if(L.is_captured)
		{
			const double r_f = ev_radius(L.cur), v_f = ev_speed(L.cur);
			const double vesc_f = solar_vesc(S, r_f);
			const double E_f = 0.5 * m_dm * ((v_f * v_f - vesc_f * vesc_f) / (DMS_C_KMS * DMS_C_KMS)) / 1.0e-9;
			if(reason == DMS_REASON_OUTWARD_ESCAPE && E_f >= 0.0)
			{
				if(isfinite(L.t_final_unbinding))
				{
					boundary_escape = 1;
					t_boundary = t_term;
					event_observed = 1;
				}
				else
				{
					reason = DMS_REASON_ENERGY_DRIFT_ESCAPE;
					survival_valid = 0;
					invalid_escape = 1;
				}
			}
		}
		switch(reason)
		{
			case DMS_REASON_ENERGY_DRIFT_ESCAPE:
			case DMS_REASON_NUMERICAL_FAILURE:
			case DMS_REASON_NON_FINITE_STATE:
			case DMS_REASON_SPEED_LIMIT:
			case DMS_REASON_WALL_TIME_LIMIT:
			case DMS_REASON_MAX_FREE_STEPS:
			case DMS_REASON_MAX_SCATTERINGS:
			case DMS_REASON_UNKNOWN: survival_valid = 0; break;
			default: break;
		}
		if(L.is_captured && !event_observed)
		{
			L.t_final_unbinding = NAN;
			if(reason != DMS_REASON_CAPTURE_MODE)
				survival_valid = 0;
		}
		if(L.is_captured) flags |= DMS_REC_CAPTURED;
		if(event_observed) flags |= DMS_REC_EVENT_OBSERVED;
		if(survival_valid) flags |= DMS_REC_SURVIVAL_VALID;
		if(boundary_escape) flags |= DMS_REC_BOUNDARY_ESCAPE;
		if(invalid_escape) flags |= DMS_REC_INVALID_ESCAPE;
		if(!L.is_captured && reason == DMS_REASON_OUTWARD_ESCAPE)
		{
			if(L.nscat == 0)
				flags |= DMS_REC_FREE;
			else
			{
				const double rf = ev_radius(L.cur);
				const double vesc = sqrt(2 * DMS_GMSUN_KM3S2 / rf);
				if(rf > DMS_RSUN_KM && ev_speed(L.cur) > vesc)
				{
					flags |= DMS_REC_REFLECTED;
					Event fin = L.cur;
					if(hyperbolic_kepler_shift(fin, DMS_AU_KM))
					{
						flags |= DMS_REC_REFLECT_SHIFT_OK;
						if(R.records == nullptr && R.reflections != nullptr)
						{
							// the reflection-spectrum sample, src/Data_Generation.cpp:829-840
							const double speed = ev_speed(fin);
							const double* vs = P->vel_obs;
							const double sun = sqrt(vs[0] * vs[0] + vs[1] * vs[1] + vs[2] * vs[2]);
							const double cosine = (fin.x.x * vs[0] + fin.x.y * vs[1] + fin.x.z * vs[2]) / ev_radius(fin) / sun;
							const unsigned long long k = atomicAdd(R.reflection_count + L.point, 1ULL);
							if(k < R.event_capacity)
							{
								dms_reflection rf;
								rf.trajectory_id = L.D.traj + 1;
								rf.speed_kms = speed;
								rf.cos_sun_velocity = cosine;
								R.reflections[static_cast<size_t>(L.point) * R.event_capacity + k] = rf;
							}
							else
								atomicAdd(R.counters + static_cast<size_t>(L.point) * DMS_NUM_COUNTERS + DMS_CNT_REFLECTIONS_DROPPED, 1ULL);
						}
					}
				}
			}
		}
	}
	else
	{
		reason = DMS_REASON_NUMERICAL_FAILURE;
		survival_valid = 0;
	}
	const bool invalid = invalid_escape || reason == DMS_REASON_ENERGY_DRIFT_ESCAPE;
	const bool valid = survival_valid && !invalid;
	const bool observed = valid && event_observed;
	const double life = observed ? L.t_final_unbinding - L.t_capture : -1.0;
	const double lifetime = (L.is_captured && isfinite(life) && life >= 0.0) ? life : -1.0;

	job.b0 = L.bmin;
	job.b1 = L.bmax;
	job.mode = FLUSH_ZERO;
	if(R.records != nullptr)
	{
		dms_traj_record& rec = R.records[L.work - 0];
		rec.number_of_scatterings = L.nscat;
		rec.number_of_draws = L.D.index;
		rec.termination_reason = static_cast<uint32_t>(reason);
		rec.flags = flags;
		rec.final_time = L.cur.t;
		rec.final_position[0] = L.cur.x.x;
		rec.final_position[1] = L.cur.x.y;
		rec.final_position[2] = L.cur.x.z;
		rec.final_velocity[0] = L.cur.v.x;
		rec.final_velocity[1] = L.cur.v.y;
		rec.final_velocity[2] = L.cur.v.z;
		rec.t_capture = L.shift_ok ? L.t_capture : -1.0;
		rec.t_last_bound = L.shift_ok ? L.t_last_bound : -1.0;
		rec.t_final_unbinding_scatter = L.shift_ok ? L.t_final_unbinding : NAN;
		rec.t_boundary_escape = t_boundary;
		rec.t_termination = L.shift_ok ? t_term : -1.0;
		rec.max_free_energy_drift_eV = L.max_drift_eV;
		rec.max_free_energy_drift_rel = L.max_drift_rel;
		rec.lifetime_unbinding = lifetime;
		if(R.rec_hist_dt != nullptr)
		{
			job.mode = FLUSH_COPY;
			job.dst0 = R.rec_hist_dt + L.work * DMS_NUM_BINS;
			job.dst1 = R.rec_hist_v2dt + L.work * DMS_NUM_BINS;
		}
	}
	else
	{
		unsigned long long* c = R.counters + static_cast<size_t>(L.point) * DMS_NUM_COUNTERS;
		atomicAdd(c + DMS_CNT_TRAJECTORIES, 1ULL);
		atomicAdd(c + DMS_CNT_TOTAL_SCATTERINGS, static_cast<unsigned long long>(L.nscat));
		atomicAdd(c + DMS_CNT_RK_STEPS, static_cast<unsigned long long>(L.steps));
		atomicAdd(c + DMS_CNT_RK_ATTEMPTS, static_cast<unsigned long long>(L.attempts));
		atomicAdd(c + DMS_CNT_REASON_BASE + reason, 1ULL);
		if(!L.shift_ok)
		{
			atomicAdd(c + DMS_CNT_INITIAL_SHIFT_FAILURES, 1ULL);
			atomicAdd(c + DMS_CNT_NUMERICAL_FAILURES, 1ULL);
		}
		else if(is_numerical_termination(reason))
			atomicAdd(c + DMS_CNT_NUMERICAL_FAILURES, 1ULL);
		if(is_computational_truncation(reason))
			atomicAdd(c + DMS_CNT_COMPUTATIONAL_TRUNCATIONS, 1ULL);
		int hist_slot = -1;
		if(L.is_captured)
		{
			atomicAdd(c + DMS_CNT_CAPTURED, 1ULL);
			if(!R.capture_mode)
			{
				atomicAdd(c + (event_observed ? DMS_CNT_COMPLETE_EVAPORATION : DMS_CNT_INVALID_SURVIVAL), 1ULL);
				hist_slot = 0;
				if(lifetime >= 0.0)
				{
					const unsigned long long k = atomicAdd(R.event_count + L.point, 1ULL);
					if(k < R.event_capacity)
					{
						// the lifetime is made visible before the id: a reader of a run in flight
						// takes a slot whose id is still 0 (ids start at 1) as not yet published
						dms_evaporation_event& ev = R.events[static_cast<size_t>(L.point) * R.event_capacity + k];
						ev.lifetime_unbinding = lifetime;
						__threadfence();
						*reinterpret_cast<volatile uint64_t*>(&ev.trajectory_id) = L.D.traj + 1;
					}
					else
						atomicAdd(c + DMS_CNT_EVENTS_DROPPED, 1ULL);
				}
			}
		}
		else if(reason == DMS_REASON_OUTWARD_ESCAPE)
		{
			atomicAdd(c + DMS_CNT_COMPLETED_OUTWARD, 1ULL);
			if(!R.capture_mode)
			{
				hist_slot = 2;
				if(flags & DMS_REC_FREE)
					atomicAdd(c + DMS_CNT_FREE, 1ULL);
				else if(flags & DMS_REC_REFLECTED)
				{
					atomicAdd(c + DMS_CNT_REFLECTED, 1ULL);
					if(!(flags & DMS_REC_REFLECT_SHIFT_OK))
					{
						atomicAdd(c + DMS_CNT_FINAL_REFLECTION_SHIFT_FAILURES, 1ULL);
						atomicAdd(c + DMS_CNT_NUMERICAL_FAILURES, 1ULL);
					}
				}
			}
		}
		if(hist_slot >= 0)
		{
			double* h = R.hists + static_cast<size_t>(L.point) * DMS_NUM_HISTS * DMS_NUM_BINS;
			job.mode = FLUSH_ADD;
			job.dst0 = h + (hist_slot + 0) * DMS_NUM_BINS;
			job.dst1 = h + (hist_slot + 1) * DMS_NUM_BINS;
			job.dst2 = h + (hist_slot + 4) * DMS_NUM_BINS;
			job.dst3 = h + (hist_slot + 5) * DMS_NUM_BINS;
		}
	}
}

// Moves the histogram rows of every lane of the group `grp` (the whole warp) that terminated in
// this iteration: all lanes of the group stride over one row at a time, so the row is read, the
// per-point sums are updated and the row is zeroed with coalesced accesses instead of one
// lane walking up to 2000 bins while the rest of its warp waits.
__device__ __forceinline__ void cooperative_flush(double2* hist, FlushJob& job, unsigned int grp)
{
	unsigned int pending = __ballot_sync(grp, job.b1 >= job.b0);
	if(pending == 0u)
		return;
	const int me = threadIdx.x & 31;
	const int rank = __popc(grp & ((1u << me) - 1u));
	const int size = __popc(grp);
	__syncwarp(grp);  // each owner's last write to its row is visible to the group
	while(pending != 0u)
	{
		const int leader = __ffs(pending) - 1;
		pending &= pending - 1u;
		double2* row = reinterpret_cast<double2*>(__shfl_sync(grp, reinterpret_cast<unsigned long long>(hist), leader));
		int b0 = __shfl_sync(grp, job.b0, leader);
		int b1 = __shfl_sync(grp, job.b1, leader);
		DMS_CHECK_INDEX(b0, 0, DMS_NUM_BINS, BOUNDS_ROW);
		DMS_CHECK_INDEX(b1, 0, DMS_NUM_BINS, BOUNDS_ROW);
		const int mode = __shfl_sync(grp, job.mode, leader);
		double* d0 = reinterpret_cast<double*>(__shfl_sync(grp, reinterpret_cast<unsigned long long>(job.dst0), leader));
		double* d1 = reinterpret_cast<double*>(__shfl_sync(grp, reinterpret_cast<unsigned long long>(job.dst1), leader));
		double* d2 = reinterpret_cast<double*>(__shfl_sync(grp, reinterpret_cast<unsigned long long>(job.dst2), leader));
		double* d3 = reinterpret_cast<double*>(__shfl_sync(grp, reinterpret_cast<unsigned long long>(job.dst3), leader));
		for(int b = b0 + rank; b <= b1; b += size)
		{
			const double2 x = row[b];
			if(mode == FLUSH_COPY)
			{
				d0[b] = x.x;
				d1[b] = x.y;
			}
			else if(mode == FLUSH_ADD && (x.x != 0.0 || x.y != 0.0))
			{
				atomicAdd(d0 + b, x.x);
				atomicAdd(d1 + b, x.y);
				atomicAdd(d2 + b, x.x * x.x);
				atomicAdd(d3 + b, x.y * x.y);
			}
			row[b] = make_double2(0.0, 0.0);
		}
	}
	__syncwarp(grp);  // the zeroed rows are visible to their owners before they are reused
	job.b1 = -1;
}

// Picks up work index `w`: the Simulate prologue (src/Simulation_Trajectory.cpp:1284-1308) from
// the initial state (Initial_Conditions + Hyperbolic_Kepler_Shift, src/Data_Generation.cpp:747-761)
// that initial_state_kernel computed for every work index before the launch.
template <class Lane>
__device__ __forceinline__ int start_trajectory(const RunParams& R, Lane& L, uint64_t w, const DevPoint*& P, double& m_dm)
{
	int k = find_range(R, w);
	DMS_CHECK_INDEX(k, 0, R.n_ranges, BOUNDS_RANGE);
	L.work = w;
	L.point = R.range_point[k];
	P = R.points + L.point;
	m_dm = __ldg(&P->m_dm);
	L.D.seed = R.seed;
	L.D.point = static_cast<uint32_t>(L.point);
	L.D.traj = R.range_first[k] + (w - R.range_offset[k]);
	L.D.index = 0;
	L.nscat = 0;
	L.steps = 0;
	L.attempts = 0;
	L.wall_start = R.wall_limit_ns != 0 ? global_timer_ns() : 0;
	L.is_captured = 0;
	L.bound_state = 0;
	L.t_capture = -1.0;
	L.t_last_bound = -1.0;
	L.t_final_unbinding = NAN;
	L.free_flight_E = NAN;
	L.max_drift_eV = 0.0;
	L.max_drift_rel = 0.0;
	L.prev_time = -1.0;
	L.prev_r = 0.0;
	L.prev_v2 = 0.0;
	L.bmin = DMS_NUM_BINS;
	L.bmax = -1;
	L.cbin = -1;
	L.reason = DMS_REASON_UNKNOWN;
	const InitState& init = R.init[w];
	const Event ic = init.ic;
	L.D.index = init.draws;
	L.shift_ok = (init.flags & INIT_SHIFT_OK) != 0u;
	L.cur = ic;
	if(R.records != nullptr)
	{
		dms_traj_record& rec = R.records[w];
		rec.trajectory_id = L.D.traj;
		rec.point = static_cast<uint32_t>(L.point);
		rec.reserved = 0;
		rec.initial_time = ic.t;
		rec.initial_position[0] = ic.x.x;
		rec.initial_position[1] = ic.x.y;
		rec.initial_position[2] = ic.x.z;
		rec.initial_velocity[0] = ic.v.x;
		rec.initial_velocity[1] = ic.v.y;
		rec.initial_velocity[2] = ic.v.z;
	}
	if(!L.shift_ok)
	{
		L.reason = DMS_REASON_NUMERICAL_FAILURE;
		return PH_FINAL;
	}
	return PH_SEGMENT;
}

// Sample_Target for every lane of the group `grp` (the whole warp) at a scattering point.  The 64
// channel rates of one scattering lane (63 isotopes + electrons, the dominant cost of a
// scatter) are evaluated by all lanes of the group in parallel into shared memory; the
// scattering lane then validates, sums and picks sequentially in the reference's order, so
// the target and the draws consumed are those of the one-lane form.  `rates` is this warp's
// DMS_NUM_TARGETS + 1 doubles of shared memory.
template <class Lane, class Step>
__device__ __forceinline__ void cooperative_targets(const RunParams& R, Lane& L, int phase, double* rates, int& target, const Step& step,
                                                    unsigned int grp)
{
	unsigned int pending = __ballot_sync(grp, phase == PH_SCATTER);
	if(pending == 0u)
		return;
	const int me = threadIdx.x & 31;
	const int rank = __popc(grp & ((1u << me) - 1u));
	const int size = __popc(grp);
	const bool mine = phase == PH_SCATTER;
	const double my_r = mine ? ev_radius(L.cur) : 0.0;
	const double my_v = mine ? ev_speed(L.cur) : 0.0;
	while(pending != 0u)
	{
		const int leader = __ffs(pending) - 1;
		pending &= pending - 1u;
		const double r = __shfl_sync(grp, my_r, leader);
		const double v = __shfl_sync(grp, my_v, leader);
		const int point = __shfl_sync(grp, L.point, leader);
		bool bad = !(isfinite(r) && isfinite(v));
		if(!bad)
		{
			const DevPoint* P = R.points + point;
			const int i = knot_index(R.S, r);
			const double dr = r - __ldg(R.S.r + i);
			const double T = __ldg(R.S.temp + i) + dr * __ldg(R.S.temp_s + i);
			for(int k = rank; k <= DMS_NUM_TARGETS; k += size)
			{
				const double x = step.channel(R.S, P, i, dr, T, v, k);
				bad = bad || !(isfinite(x) && x >= 0.0);
				rates[k] = x;
			}
		}
		// validation: every channel finite and >= 0 (the reference throws otherwise)
		bad = __any_sync(grp, bad);
		__syncwarp(grp);
		double total = 0.0;
		if(me == leader && !bad)
			total = channel_total(rates);
		total = __shfl_sync(grp, total, leader);
		const bool ok = !bad && isfinite(total) && total > 0.0;
		// the 64 divisions by the total, in parallel: each lane replaces its channels by
		// their fractions, exactly the quotients the sequential pick forms
		if(ok)
			for(int k = rank; k <= DMS_NUM_TARGETS; k += size) rates[k] = rates[k] / total;
		__syncwarp(grp);
		if(me == leader)
			target = ok ? pick_from_fractions(L.D, rates) : TARGET_FAILED;
		__syncwarp(grp);
	}
}

// Simulate after a scattering point (src/Simulation_Trajectory.cpp:1313-1346): target
// velocity, angle and kinematics, then capture bookkeeping and the bincount anchor.
template <class Lane, class Step>
__device__ __forceinline__ int finish_scatter(const RunParams& R, const DevPoint* __restrict__ P, double m_dm, Lane& L, int target, const Step& step)
{
	if(target != TARGET_FAILED)
		DMS_CHECK_INDEX(target, -1, DMS_NUM_TARGETS, BOUNDS_TARGET);
	if(target == TARGET_FAILED || !step.scatter(R.S, P, L.D, L.cur, target))
	{
		L.reason = DMS_REASON_NUMERICAL_FAILURE;
		return PH_FINAL;
	}
	L.nscat++;
	const bool captured = update_capture_state(R.S, m_dm, R.capture_mode, L, ev_radius(L.cur), ev_speed(L.cur), L.cur.t, true);
	if(!R.capture_mode)
	{
		// Reset_Bincount_Anchor, src/Simulation_Trajectory.cpp:671-680
		L.prev_time = L.cur.t;
		L.prev_r = ev_radius(L.cur);
		const double v = ev_speed(L.cur);
		L.prev_v2 = v * v;
	}
	if(R.capture_mode && captured)
	{
		L.reason = DMS_REASON_CAPTURE_MODE;
		return PH_FINAL;
	}
	return PH_SEGMENT;
}


// Position of the (n+1)-th set bit of m (n from 0); m must have more than n set bits.
__device__ __forceinline__ int nth_set_bit(unsigned int m, int n)
{
	for(int t = 0; t < n; t++) m &= m - 1u;
	return __ffs(m) - 1;
}

template <class Lane, class Step>
__device__ __forceinline__ void lane_loop(const RunParams& R, Step step)
{
	const int lane_id = blockIdx.x * blockDim.x + threadIdx.x;
	double2* hist = R.lane_hist + static_cast<size_t>(lane_id) * DMS_NUM_BINS;
	__shared__ double coop_rates[4][DMS_NUM_TARGETS + 1];  // blocks of at most 128 threads
	double* rates = coop_rates[threadIdx.x >> 5];
	// set once a lane of the block finds the work queue empty: the launch is in its tail, where
	// the lanes left run alone and the free step takes its shorter-chain form
	__shared__ int queue_drained;
	if(threadIdx.x == 0)
		queue_drained = 0;
	if constexpr(Step::pipeline)
		if(threadIdx.x == 0)
			step.pipe_init();
	__syncthreads();
	Lane L;
	FlushJob job;
	job.b0 = 0;
	job.b1 = -1;
	const DevPoint* P = R.points;
	double m_dm = 0.0;
	int phase = PH_FETCH;
	int scatter_wait = 0;
	int final_wait = 0;
	// the lane's claimed ids [q_next, q_end): R.queue_chunk ids per claim
	uint64_t q_next = 0, q_end = 0;
	const unsigned int lane_bit = 1u << (threadIdx.x & 31);
	// tail pipeline: this lane owns the block's helper warp; pipe_spec is the hand-over of the
	// next step's start made before the current finish (0 = none)
	bool pipe_owner = false;
	int pipe_spec = 0;
	// Every lane stays in the loop until its whole warp is done (a lane without work waits in
	// PH_DONE), and leaves only together with the others.  So the warp's collective steps
	// below (batching votes, cooperative target sampling into the warp's shared rates, the
	// histogram flush) always run with all 32 lanes, a fixed mask, instead of whichever lanes
	// happen to be converged at that point.
	constexpr unsigned int FULL_WARP = 0xffffffffu;
	for(uint64_t iter = 0;; iter++)
	{
		if(__all_sync(FULL_WARP, phase == PH_DONE))
		{
			if constexpr(Step::pipeline)
				if(R.wall_limit_ns == 0 && blockDim.x > 32)
					step.pipe_serve(R, L);  // the warp may stay as the block's helper
			break;
		}
#if DMS_RK_UNROLLED == 2 || DMS_RK_UNROLLED_MIXED == 2
		// a block whose lanes are all held by long trajectories learns of the drained queue from
		// the queue head itself (one read per warp every 64 iterations)
		if((iter & 63) == 63 && (threadIdx.x & 31) == 0 &&
		   *reinterpret_cast<volatile unsigned long long*>(R.queue_head) >= R.total)
			*reinterpret_cast<volatile int*>(&queue_drained) = 1;
#endif
		if((iter & 1023) == 1023)
		{
			if(__any_sync(FULL_WARP, *R.cancel != 0))
			{
				atomicOr(R.status, STATUS_CANCELLED);
				break;
			}
			if(iter > R.iteration_budget)
			{
				atomicOr(R.status, STATUS_BUDGET);
				break;
			}
		}
		if(phase == PH_FETCH)
		{
			// warp-aggregated claim of R.queue_chunk work indices per lane whose claimed ids
			// are used up
			const unsigned int mask = __activemask();
			const bool need = !(q_next < q_end);
			const unsigned int need_mask = __ballot_sync(mask, need);
			if(need_mask != 0u)
			{
				const int leader = __ffs(need_mask) - 1;
				const unsigned int rank = __popc(need_mask & (lane_bit - 1u));
				unsigned long long base = 0;
				if((threadIdx.x & 31) == leader)
					base = atomicAdd(R.queue_head, static_cast<unsigned long long>(__popc(need_mask)) * R.queue_chunk);
				base = __shfl_sync(mask, base, leader);
				if(need)
				{
					q_next = base + static_cast<uint64_t>(rank) * R.queue_chunk;
					q_end = q_next + R.queue_chunk;
				}
			}
			const uint64_t w = q_next++;
			if(w >= R.total)
			{
				*reinterpret_cast<volatile int*>(&queue_drained) = 1;
				phase = PH_DONE;
			}
			else
				phase = start_trajectory(R, L, w, P, m_dm);
		}
		if(phase == PH_SEGMENT)
			phase = segment_start(R, P, m_dm, L);
		if constexpr(Step::pairs)
		{
			// A step is opened per lane; its RK45 attempt then runs paired when at most half of
			// the warp is attempting: every attempting lane takes an idle lane of its warp as a
			// helper for the independent stages (rk45_attempt_pair), which shortens the dependent
			// chain of a lane that runs alone, the tail of a launch.  Same results either way.  With
			// Step::pipeline a lane that steps alone in its warp may instead hand its step head and
			// attempts to the block's helper warp (see PipeBox); such a lane is busy ("piped")
			// without attempting here.
			const int drained = *reinterpret_cast<volatile int*>(&queue_drained);
			bool want = false;
			bool piped = false;  // the step's head and attempts came from the helper warp
			int rk_piped = RK_RETRY;
			if constexpr(Step::pipeline)
			{
				// only a lane that steps alone in its warp owns the helper: an owner's waits hold its
				// whole warp.  An owner that ends its trajectory or stops being alone releases it.
				const unsigned int stepping = __ballot_sync(FULL_WARP, phase == PH_STEP);
				const bool alone = phase == PH_STEP && stepping == lane_bit;
				if(pipe_owner && !alone && phase != PH_SCATTER && phase != PH_SEGMENT)
				{
					step.pipe_release(pipe_spec);
					pipe_owner = false;
				}
				if(alone && !L.in_rk && drained && R.wall_limit_ns == 0)
				{
					if(!pipe_owner)
						pipe_owner = step.pipe_attach();
					if(pipe_owner)
					{
						const int r = step.pipe_step(P, L, pipe_spec, rk_piped);
						piped = r == 1;
						if(r < 0)
							pipe_owner = false;  // the helper did not answer: step alone
					}
				}
			}
			if(phase == PH_STEP)
			{
				if(piped)
					want = true;
				else
				{
					const int ph = step.begin(R, P, L);
					want = ph == PH_STEP;
					if(!want)
						phase = ph;
				}
			}
			if constexpr(Step::pipeline)
			{
				// hand over the next step's start now, so that it is made during this finish
				if(piped && rk_piped == RK_ACCEPTED)
					pipe_spec = step.pipe_post(P, L.pr, L.seg_steps + 1);
			}
			const unsigned int att = __ballot_sync(FULL_WARP, want && !piped);
			const unsigned int busy = __ballot_sync(FULL_WARP, want);
			const int n_att = __popc(att);
			// every attempting lane needs an idle lane (a piped lane is busy without attempting)
			if(busy != 0u && n_att <= DMS_PAIR_MAX_LANES && n_att + __popc(busy) <= 32 && (drained || !DMS_PAIR_ONLY_DRAINED))
			{
				const int me = threadIdx.x & 31;
				int role = 0, partner = me;
				const unsigned int below = lane_bit - 1u;
				if(want && !piped)
				{
					role = 1;
					partner = nth_set_bit(~busy, __popc(att & below));
				}
				else if(!want)
				{
					const int q = __popc(~busy & below);
					if(q < n_att)
					{
						role = 2;
						partner = nth_set_bit(att, q);
					}
				}
				// (a warp whose only busy lane was piped has no attempt to make)
				const int rk = n_att != 0 ? step.pair_attempt(R.S, L, role, partner) : RK_RETRY;
				// the finished steps' piece rates are formed by the whole warp
				const int ph = step.finish_warp(R, P, m_dm, L, hist, piped ? rk_piped : rk, want);
				if(want)
					phase = ph;
			}
			else if(want)
				phase = step.finish(R, P, m_dm, L, hist, piped ? rk_piped : step.attempt(R.S, L, drained));
		}
		else if(phase == PH_STEP)
			phase = step(R, P, m_dm, L, hist, *reinterpret_cast<volatile int*>(&queue_drained));
		// Scatterings wait until several lanes of the warp have one (or one has waited
		// R.scatter_wait iterations, or no lane is stepping), so that the scattering code
		// runs for many lanes at once.  A lane's draws do not depend on when it scatters.
		{
			const unsigned int grp = FULL_WARP;
			const unsigned int waiting = __ballot_sync(grp, phase == PH_SCATTER);
			if(waiting != 0u)
			{
				const unsigned int stepping = __ballot_sync(grp, phase == PH_STEP);
				const bool go = __popc(waiting) >= R.scatter_batch || stepping == 0u ||
				                __any_sync(grp, phase == PH_SCATTER && scatter_wait >= R.scatter_wait);
				if(go)
				{
					int target = TARGET_FAILED;
					cooperative_targets(R, L, phase, rates, target, step, grp);
					if(phase == PH_SCATTER)
					{
						phase = finish_scatter(R, P, m_dm, L, target, step);
						scatter_wait = 0;
					}
				}
				else if(phase == PH_SCATTER)
					scatter_wait++;
			}
		}
		// terminations are batched the same way
		{
			const unsigned int grp = FULL_WARP;
			const unsigned int ending = __ballot_sync(grp, phase == PH_FINAL);
			if(ending != 0u)
			{
				const unsigned int stepping = __ballot_sync(grp, phase == PH_STEP);
				const bool go = __popc(ending) >= R.final_batch || stepping == 0u ||
				                __any_sync(grp, phase == PH_FINAL && final_wait >= R.final_wait);
				if(go)
				{
					if(phase == PH_FINAL)
					{
						write_back_bin(L, hist);
						finalize(R, P, m_dm, L, job);
						phase = PH_FETCH;
						final_wait = 0;
					}
					cooperative_flush(hist, job, grp);
				}
				else if(phase == PH_FINAL)
					final_wait++;
			}
		}
	}
	const bool in_trajectory = phase != PH_FETCH && phase != PH_DONE;
	if(in_trajectory && L.bmax >= L.bmin)
		for(int b = L.bmin; b <= L.bmax; b++) hist[b] = make_double2(0.0, 0.0);
	if(in_trajectory && R.records == nullptr)
	{
		// stopped in mid-trajectory: count the work done so far
		unsigned long long* c = R.counters + static_cast<size_t>(L.point) * DMS_NUM_COUNTERS;
		atomicAdd(c + DMS_CNT_UNFINISHED_TRAJECTORIES, 1ULL);
		atomicAdd(c + DMS_CNT_UNFINISHED_SCATTERINGS, static_cast<unsigned long long>(L.nscat));
		atomicAdd(c + DMS_CNT_UNFINISHED_RK_STEPS, static_cast<unsigned long long>(L.steps));
		atomicAdd(c + DMS_CNT_UNFINISHED_RK_ATTEMPTS, static_cast<unsigned long long>(L.attempts));
	}
}

}	// namespace lane
}	// namespace dms
