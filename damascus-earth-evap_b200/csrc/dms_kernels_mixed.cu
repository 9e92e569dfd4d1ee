// Mixed-precision trajectory kernel (the batched-FP32 form).  Compiled with FMA contraction;
// shares the lane state machine (dms_lane.cuh) with the FP64 kernel.
#include "dms_device_mixed.cuh"
#include "dms_lane.cuh"

namespace dms
{
namespace mixed
{
// found by argument-dependent lookup from the lane state machine
__device__ __forceinline__ void init_propagator(PropF& p, const Event& e) { prop_init_f(p, e); }
}	// namespace mixed

namespace
{
using namespace lane;
using namespace mixed;
using MixedLane = LaneT<PropF, EventF>;

// commit_accepted_event (src/Simulation_Trajectory.cpp:842-874) for an FP32 event: bincount
// with FP64 times, capture energy in FP64.  Returns the energy when evaluated, NaN otherwise.
__device__ __forceinline__ double commit_event_mixed(const DevSolar& S, const DevSolarF& F, double m_dm, int capture_mode, MixedLane& L, double2* hist,
                                                     const EventF& local)
{
	const float rf = normf(local.x), vf = normf(local.v);
	const double r_now = static_cast<double>(rf);
	const double v_now = static_cast<double>(vf);
	if(!capture_mode)
	{
		if(L.prev_time >= 0.0)
			accumulate_bincount(L, hist, L.prev_r, L.prev_v2, local.t - L.prev_time);
		L.prev_time = local.t;
		L.prev_r = r_now;
		L.prev_v2 = v_now * v_now;
	}
	const double t_abs = local.t + L.origin;
	if(capture_mode && !L.is_captured)
		return NAN;
	const double E = capture_energy_eV_f(S, F, m_dm, rf, vf);
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
		L.t_last_bound = t_abs;
	return E;
}

// Mixed-precision form of the free step (see dms_kernels.cu for the FP64 form and
// dms_device_mixed.cuh for what stays FP64).  Propagate_Freely loop body,
// src/Simulation_Trajectory.cpp:876-1116, split at the
// RK45 retry loop: when no step is in progress the pre-step bounds are applied and a step is
// opened; every pass makes one RK45 attempt; only a finished step runs the optical-depth,
// boundary and commit logic.  Returns the next phase of the lane.
__device__ __forceinline__ int free_step_mixed(const RunParams& R, const DevPoint* __restrict__ P, double m_dm, MixedLane& L, double2* hist,
                                               int drained)
{
	const DevSolar& S = R.S;
	const DevSolarF F{R.sf_r, R.sf_gm, R.sf_gm_s, R.sf_vesc2, R.sf_vesc2_s};
	const float* grid = reinterpret_cast<const float*>(__ldg(reinterpret_cast<const unsigned long long*>(&P->grid_f)));
	const int capture_mode = R.capture_mode;
	const double tau_limit = capture_mode ? DMS_CAPTURE_MAX_OPTICAL_DEPTH_STEP : DMS_MAX_OPTICAL_DEPTH_STEP;
	if(!L.in_rk)
	{
		if(!(L.seg_steps < R.max_free_steps))
		{
			L.reason = DMS_REASON_MAX_FREE_STEPS;  // L.cur holds the last committed event
			return PH_FINAL;
		}
		if(wall_time_exceeded(R, L))  // "before_step", src/Simulation_Trajectory.cpp:873-874
		{
			set_final(L, to_event64(prop_event_f(L.pr)), true, DMS_REASON_WALL_TIME_LIMIT);
			return PH_FINAL;
		}
		if(!L.before_valid)
		{
			L.before = prop_event_f(L.pr);
			L.before_valid = 1;
		}
		const double r_before = prop_radius_f(L.pr);
		const double v_before = prop_speed_f(L.pr);
		L.rate_before = 0.0;
		if(r_before >= DMS_RSUN_KM)
		{
			const double cap = step_cap(r_before, v_before, R.boundary);
			const double ts = sanitized_step(L.pr.time_step);
			L.pr.time_step = ts < cap ? ts : cap;
			const double vr = (r_before > 0.0) ? static_cast<double>(dotf(L.before.x, L.before.v)) / r_before : 0.0;
			if(r_before > DMS_RSUN_KM && vr < 0.0)
			{
				const double est = (r_before - DMS_RSUN_KM) / (-vr);
				if(isfinite(est) && est > 0.0)
				{
					const double lim = est > DMS_RK45_ABS_MIN_STEP_S ? est : DMS_RK45_ABS_MIN_STEP_S;
					if(lim < L.pr.time_step) L.pr.time_step = lim;
				}
			}
		}
		else
		{
			L.pr.time_step = sanitized_step(L.pr.time_step);
			L.rate_before = rate_total_f(S, P, grid, static_cast<float>(r_before), static_cast<float>(v_before));
			if(!isfinite(L.rate_before) || L.rate_before < 0.0)
			{
				set_final(L, to_event64(prop_event_f(L.pr)), true, DMS_REASON_NUMERICAL_FAILURE);
				return PH_FINAL;
			}
			if(L.rate_before > 0.0)
			{
				const float lim = static_cast<float>(tau_limit) / static_cast<float>(L.rate_before);
				if(static_cast<double>(lim) < L.pr.time_step)
					L.pr.time_step = static_cast<double>(lim);
			}
		}
		// the RK step changes only these propagator fields
		L.b_time = L.pr.time;
		L.b_radius = L.pr.radius;
		L.b_phi = L.pr.phi;
		L.b_vr = L.pr.v_radial;
		L.b_step = L.pr.time_step;
		L.pr.time_step = sanitized_step(L.pr.time_step);  // head of Runge_Kutta_45_Step, :1489
		L.in_rk = 1;
		L.rk_inner = 0;
	}
	L.rk_inner++;
#if DMS_RK_UNROLLED_MIXED == 2
	const int rk = drained ? rk45_attempt_f<true>(S, F, L.pr, L.rk_inner) : rk45_attempt_f<false>(S, F, L.pr, L.rk_inner);
#else
	(void)drained;
	const int rk = rk45_attempt_f<DMS_RK_UNROLLED_MIXED == 1>(S, F, L.pr, L.rk_inner);
#endif
	if(rk == RK_RETRY)
		return PH_STEP;
	L.in_rk = 0;
	L.attempts += static_cast<uint64_t>(L.rk_inner);
	const EventF before = L.before;
	const double r_before = L.b_radius < 0.0 ? 0.0 : L.b_radius;
	const double rate_before = L.rate_before;
	const double actual_dt = L.pr.time - L.b_time;
	const double r_after = prop_radius_f(L.pr);
	const double v_after = prop_speed_f(L.pr);
	const EventF after = prop_event_f(L.pr);
	if(rk == RK_FORCED)
	{
		set_final(L, to_event64(after), true, DMS_REASON_NUMERICAL_FAILURE);
		return PH_FINAL;
	}
	if(!isfinite(r_after) || !isfinite(v_after) || !isfinite(actual_dt) || actual_dt <= 0.0)
	{
		set_final(L, to_event64(after), true, DMS_REASON_NON_FINITE_STATE);
		return PH_FINAL;
	}
	if(v_after > DMS_V_MAX_C * DMS_C_KMS)
	{
		set_final(L, to_event64(after), true, DMS_REASON_SPEED_LIMIT);
		return PH_FINAL;
	}
	if(wall_time_exceeded(R, L))  // "after_rk45_step", src/Simulation_Trajectory.cpp:953-954
	{
		set_final(L, to_event64(after), true, DMS_REASON_WALL_TIME_LIMIT);
		return PH_FINAL;
	}
	bool scattering = false, reflection = false;
	EventF accepted = after;
	float s0 = 0.0f, s1 = 0.0f;
	if(interior_interval_f(before, after, r_before, r_after, s0, s1))
	{
		// Build_Optical_Depth_Pieces, src/Simulation_Trajectory.cpp:347-414
		const int pieces = capture_mode ? DMS_CAPTURE_OPTICAL_DEPTH_PIECES : DMS_MAX_OPTICAL_DEPTH_PIECES;
		const bool use_cached = r_before < DMS_RSUN_KM && s0 <= 1.0e-12f;
		const float span = s1 - s0;
		const float adt = static_cast<float>(actual_dt);
		float fr[DMS_MAX_OPTICAL_DEPTH_PIECES + 1];
		float rt[DMS_MAX_OPTICAL_DEPTH_PIECES + 1];
		bool invalid = false;
		float dtau_f = 0.0f, tau2 = 0.0f;  // optical depths of one step (<= 0.1) in FP32
		if(s1 > s0 && actual_dt > 0.0)
		{
			// one loop over the piece boundaries, trapezoids formed as the rates arrive
			float fr_prev = 0.0f, rt_prev = 0.0f, fr_0 = 0.0f, rt_0 = 0.0f, fr_2 = 0.0f, rt_2 = 0.0f, tau2_a = 0.0f;
#pragma unroll 1
			for(int i = 0; i <= pieces; i++)
			{
				const float f = s0 + static_cast<float>(i) / static_cast<float>(pieces) * span;
				const float rate = (i == 0 && use_cached) ? static_cast<float>(rate_before) : rate_at_fraction_f(S, P, grid, before, after, f);
				fr[i] = f;
				rt[i] = rate;
				if(!isfinite(rate) || rate < 0.0f)
					invalid = true;
				if(i > 0 && f > fr_prev)
					dtau_f += 0.5f * (rt_prev + rate) * (adt * (f - fr_prev));
				if(pieces >= 4)
				{
					if(i == 0)
					{
						fr_0 = f;
						rt_0 = rate;
					}
					else if(i == 2)
					{
						fr_2 = f;
						rt_2 = rate;
						tau2_a = 0.5f * (rt_0 + rt_2) * (adt * (fr_2 - fr_0));
					}
					else if(i == 4)
						tau2 = tau2_a + 0.5f * (rt_2 + rate) * (adt * (f - fr_2));
				}
				else if(i > 0)
					tau2 += 0.5f * (rt_prev + rate) * (adt * (f - fr_prev));
				fr_prev = f;
				rt_prev = rate;
			}
		}
		const double dtau = static_cast<double>(dtau_f);
		if(invalid || !isfinite(dtau) || dtau < 0.0)
		{
			set_final(L, to_event64(after), true, DMS_REASON_NUMERICAL_FAILURE);
			return PH_FINAL;
		}
		const float scale = dtau_f > static_cast<float>(DMS_OPTICAL_DEPTH_ABS_TOL) ? dtau_f : static_cast<float>(DMS_OPTICAL_DEPTH_ABS_TOL);
		const double rel = static_cast<double>(fabsf(dtau_f - tau2) / scale);
		const bool reject_depth = dtau > tau_limit;
		const bool reject_acc = !capture_mode && rel > DMS_OPTICAL_DEPTH_REL_TOL;
		if(reject_depth || reject_acc)
		{
			L.retries++;
			if(L.retries > DMS_MAX_OPTICAL_DEPTH_RETRIES)
			{
				set_final(L, to_event64(before), true, DMS_REASON_NUMERICAL_FAILURE);
				return PH_FINAL;
			}
			L.pr.time = L.b_time;
			L.pr.radius = L.b_radius;
			L.pr.phi = L.b_phi;
			L.pr.v_radial = L.b_vr;
			L.pr.time_step = L.b_step;
			double factor = DMS_RK45_MAX_STEP_FACTOR;
			if(dtau > tau_limit && dtau > 0.0 && 0.8 * tau_limit / dtau < factor)
				factor = 0.8 * tau_limit / dtau;
			if(reject_acc && rel > 0.0 && 0.8 * sqrt(DMS_OPTICAL_DEPTH_REL_TOL / rel) < factor)
				factor = 0.8 * sqrt(DMS_OPTICAL_DEPTH_REL_TOL / rel);
			if(factor > 1.0) factor = 1.0;
			if(factor < DMS_RK45_MIN_STEP_FACTOR) factor = DMS_RK45_MIN_STEP_FACTOR;
			L.pr.time_step = sanitized_step(factor * actual_dt);
			return PH_STEP;  // L.before still describes the restored propagator
		}
		if(dtau >= L.tau)
		{
			double remaining = L.tau;
			for(int k = 0; k < pieces; k++)
			{
				if(!(fr[k + 1] > fr[k]))
					continue;
				const double pdt = actual_dt * static_cast<double>(fr[k + 1] - fr[k]);
				const double ptau = 0.5 * static_cast<double>(rt[k] + rt[k + 1]) * pdt;
				if(ptau >= remaining)
				{
					const double lf = solve_linear_rate(rt[k], rt[k + 1], pdt, remaining);
					const float f = fr[k] + static_cast<float>(lf) * (fr[k + 1] - fr[k]);
					accepted = interpolate_event_f(before, after, f);
					scattering = true;
					break;
				}
				remaining -= ptau;
			}
			if(!scattering)
			{
				accepted = interpolate_event_f(before, after, s1);
				scattering = true;
			}
		}
		else
			L.tau -= dtau;
	}
	if(!scattering)
	{
		EventF boundary_ev = after;
		double r_b = r_after, v_b = v_after;
		if(r_before < R.boundary && r_after >= R.boundary && r_after > r_before)
		{
			const double f = (R.boundary - r_before) / (r_after - r_before);
			boundary_ev = interpolate_event_f(before, after, static_cast<float>(f));
			r_b = normf(boundary_ev.x);
			v_b = normf(boundary_ev.v);
		}
		if(r_b >= R.boundary && r_b >= r_before && v_b > solar_vesc(S, r_b))
		{
			accepted = boundary_ev;
			reflection = true;
		}
		else if(r_b >= R.boundary && r_b >= r_before)
		{
			Event abs_b = to_event64(boundary_ev);
			abs_b.t += L.origin;
			if(uncaptured_bound(S, m_dm, L, abs_b))
			{
				set_final(L, abs_b, false, DMS_REASON_NUMERICAL_FAILURE);
				return PH_FINAL;
			}
			Event inbound;
			if(bound_kepler_return(to_event64(boundary_ev), inbound))
			{
				L.seg_steps++;
				L.steps++;
				L.retries = 0;
				commit_event_mixed(S, F, m_dm, capture_mode, L, hist, boundary_ev);
				// reset_propagator_at_absolute_event, src/Simulation_Trajectory.cpp:814-822
				L.cur = inbound;
				L.cur.t += L.origin;
				L.origin = L.cur.t;
				Event local = inbound;
				local.t = 0.0;
				prop_init_f(L.pr, local);
				L.before_valid = 0;
				if(!capture_mode && L.prev_time >= 0.0)
					L.prev_time = 0.0;
				return PH_STEP;
			}
		}
	}
	L.seg_steps++;
	L.steps++;
	L.retries = 0;
	double E = commit_event_mixed(S, F, m_dm, capture_mode, L, hist, accepted);
	L.cur = to_event64(accepted);
	L.cur.t += L.origin;
	if(!L.is_captured)
	{
		// abort_if_uncaptured_bound on the committed event, src/Simulation_Trajectory.cpp:767-778, 1108
		if(isnan(E))
			E = capture_energy_eV(S, m_dm, ev_radius(L.cur), ev_speed(L.cur));
		if(!(isfinite(E) && E >= 0.0))
		{
			L.reason = DMS_REASON_NUMERICAL_FAILURE;
			return PH_FINAL;
		}
	}
	if(reflection)
	{
		L.reason = DMS_REASON_OUTWARD_ESCAPE;
		return PH_FINAL;
	}
	if(scattering)
	{
		// Simulate, src/Simulation_Trajectory.cpp:1313-1346
		if(!(ev_radius(L.cur) < DMS_RSUN_KM))
		{
			L.reason = DMS_REASON_SCATTER;
			return PH_FINAL;
		}
		return PH_SCATTER;  // Sample_Target runs warp-cooperatively in the lane loop
	}
	L.before = after;
	return PH_STEP;
}

struct MixedStep
{
	static constexpr bool pairs = false;
	static constexpr bool pipeline = false;
	__device__ __forceinline__ int operator()(const RunParams& R, const DevPoint* __restrict__ P, double m_dm, MixedLane& L, double2* hist,
	                                          int drained) const
	{
		return free_step_mixed(R, P, m_dm, L, hist, drained);
	}
	__device__ __forceinline__ double channel(const DevSolar& S, const DevPoint* __restrict__ P, int i, double dr, double T, double v, int k) const
	{
		return channel_rate_f(S, P, i, dr, T, v, k);
	}
	__device__ __forceinline__ bool scatter(const DevSolar& S, const DevPoint* __restrict__ P, Draws& D, Event& e, int target) const
	{
		return scatter_with_target_f(S, P, D, e, target);
	}
};

__global__ void __launch_bounds__(128, DMS_TRAJ_MIN_BLOCKS_MIXED) trajectory_kernel_mixed(const RunParams R)
{
	lane_loop<MixedLane>(R, MixedStep());
}

__global__ void grid_to_float_kernel(const double* __restrict__ in, float* __restrict__ out, size_t n)
{
	for(size_t k = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; k < n; k += static_cast<size_t>(gridDim.x) * blockDim.x)
		out[k] = static_cast<float>(in[k]);
}

}	// namespace

void Launch_Trajectories_Mixed(const RunParams& p, int blocks, int threads, cudaStream_t stream)
{
	trajectory_kernel_mixed<<<blocks, threads, 0, stream>>>(p);
}

void Launch_To_Float(const double* in, float* out, size_t n, cudaStream_t stream)
{
	grid_to_float_kernel<<<148 * 4, 256, 0, stream>>>(in, out, n);
}

int Trajectory_Mixed_Max_Blocks_Per_SM(int threads)
{
	int n = 0;
	if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, trajectory_kernel_mixed, threads, 0) != cudaSuccess)
		return 0;
	return n;
}

unsigned int Take_Bounds_Status_Mixed()
{
#ifdef DMS_CHECKED
	unsigned int bits = 0;
	const unsigned int zero = 0;
	if(cudaMemcpyFromSymbol(&bits, dms_bounds_status, sizeof bits) != cudaSuccess ||
	   cudaMemcpyToSymbol(dms_bounds_status, &zero, sizeof zero) != cudaSuccess)
		return ~0u;
	return bits;
#else
	return 0;
#endif
}

}	// namespace dms
