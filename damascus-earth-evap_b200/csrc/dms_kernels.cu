// Kernels of the trajectory engine.
//
// trajectory_kernel: one persistent launch per dms_run.  Every thread is a lane that owns one
// trajectory at a time; lanes claim work indices from a global queue (one warp-aggregated
// atomic per claim), and refill as soon as their trajectory terminates, so trajectories of
// wildly different length (0 to 10^6 scatterings) never hold a whole batch back.  A lane's
// trajectory is a state machine whose common state is one outer step of Propagate_Freely
// (src/Simulation_Trajectory.cpp:876-1116); segment starts, scatterings and terminations are
// rare branches.  The time-weighted radial histogram of the running trajectory lives in a
// per-lane scratch row (touched bin range tracked) and is flushed once, at termination, into
// the per-point sums and sums of squares (src/Data_Generation.cpp:787-822).
#include "dms_lane.cuh"

namespace dms
{

namespace
{
using namespace lane;
using StrictLane = LaneT<Prop, Event>;

// The written-out attempt: with the certified straight-line division and square root
// (DMS_CERTIFIED_MATH = 1, the default; IEEE fallback per attempt) or with IEEE arithmetic.
__device__ __forceinline__ int rk45_attempt_written_out(const DevSolar& S, Prop& p, int inner)
{
#if DMS_CERTIFIED_MATH
	return rk45_attempt_certified(S, p, inner);
#else
	return rk45_attempt_unrolled(S, p, inner);
#endif
}

// commit_accepted_event, src/Simulation_Trajectory.cpp:842-874.  Returns the capture energy of
// the committed event when it was evaluated (NaN otherwise) so that the uncaptured-bound guard
// that follows the commit reuses the same value.
__device__ __forceinline__ double commit_event(const DevSolar& S, double m_dm, int capture_mode, StrictLane& L, double2* hist, const Event& local)
{
	const double r_now = ev_radius(local);
	const double v_now = ev_speed(local);
	if(!capture_mode)
	{
		const double v2 = v_now * v_now;
		if(L.prev_time >= 0.0)
			accumulate_bincount(L, hist, L.prev_r, L.prev_v2, local.t - L.prev_time);
		L.prev_time = local.t;
		L.prev_r = r_now;
		L.prev_v2 = v2;
	}
	const double t_abs = local.t + L.origin;
	// Update_Capture_State(..., allow_new_capture = false), src/Simulation_Trajectory.cpp:689-721
	if(capture_mode && !L.is_captured)
		return NAN;
	const double E = capture_energy_eV(S, m_dm, r_now, v_now);
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

// One pass of the Propagate_Freely loop body, src/Simulation_Trajectory.cpp:876-1116, split at the
// RK45 retry loop: when no step is in progress the pre-step bounds are applied and a step is
// opened (free_step_begin); every pass makes one RK45 attempt; only a finished step runs the
// optical-depth, boundary and commit logic (free_step_finish).  free_step_begin returns PH_STEP
// when an attempt is due, else the lane's next phase.
__device__ __forceinline__ int free_step_begin(const RunParams& R, const DevPoint* __restrict__ P, StrictLane& L)
{
	const DevSolar& S = R.S;
	const int capture_mode = R.capture_mode;
	const double tau_limit = capture_mode ? DMS_CAPTURE_MAX_OPTICAL_DEPTH_STEP : DMS_MAX_OPTICAL_DEPTH_STEP;
	if(!L.in_rk)
	{
		// speed and rate at the propagator's state, formed by the previous step's finish (tail of
		// a launch) from the same propagator
		const bool cached = L.next_valid != 0;
		L.next_valid = 0;
		if(!(L.seg_steps < R.max_free_steps))
		{
			L.reason = DMS_REASON_MAX_FREE_STEPS;  // L.cur holds the last committed event
			return PH_FINAL;
		}
		if(wall_time_exceeded(R, L))  // "before_step", src/Simulation_Trajectory.cpp:873-874
		{
			set_final(L, prop_event(L.pr), true, DMS_REASON_WALL_TIME_LIMIT);
			return PH_FINAL;
		}
		if(!L.before_valid)
		{
			L.before = prop_event(L.pr);
			L.before_valid = 1;
		}
		const double r_before = prop_radius(L.pr);
		const double v_before = cached ? L.next_speed : prop_speed(L.pr);
		L.rate_before = 0.0;
		if(r_before >= DMS_RSUN_KM)
		{
			const double cap = step_cap(r_before, v_before, R.boundary);
			const double ts = sanitized_step(L.pr.time_step);
			L.pr.time_step = ts < cap ? ts : cap;
			const double vr = (r_before > 0.0) ? dot3(L.before.x, L.before.v) / r_before : 0.0;
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
			L.rate_before = cached ? L.next_rate : rate_total(S, P, r_before, v_before);
			if(!isfinite(L.rate_before) || L.rate_before < 0.0)
			{
				set_final(L, prop_event(L.pr), true, DMS_REASON_NUMERICAL_FAILURE);
				return PH_FINAL;
			}
			if(L.rate_before > 0.0 && tau_limit / L.rate_before < L.pr.time_step)
				L.pr.time_step = tau_limit / L.rate_before;
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
	return PH_STEP;
}

// One RK45 attempt of the lane's open step (the lane alone).
__device__ __forceinline__ int free_step_attempt(const DevSolar& S, StrictLane& L, int drained)
{
	L.rk_inner++;
#if DMS_RK_UNROLLED == 2
	return drained ? rk45_attempt_written_out(S, L.pr, L.rk_inner) : rk45_attempt(S, L.pr, L.rk_inner);
#elif DMS_RK_UNROLLED == 1
	(void)drained;
	return rk45_attempt_written_out(S, L.pr, L.rk_inner);
#else
	(void)drained;
	return rk45_attempt(S, L.pr, L.rk_inner);
#endif
}

// The rest of the pass after an attempt with result rk: a retry keeps the step open; a
// finished step runs the optical-depth, boundary and commit logic.
// The trapezoid sums of the depth loop in free_step_finish over rates that are already formed:
// the same additions in the same order.
template <int PIECES>
__device__ __forceinline__ void depth_sums(const double (&fr)[DMS_MAX_OPTICAL_DEPTH_PIECES + 1], const double (&rt)[DMS_MAX_OPTICAL_DEPTH_PIECES + 1],
                                           double actual_dt, double& dtau, double& tau2, bool& invalid)
{
	double tau2_a = 0.0;
#pragma unroll
	for(int i = 0; i <= PIECES; i++)
	{
		const double f = fr[i], rate = rt[i];
		if(!isfinite(rate) || rate < 0.0)
			invalid = true;
		if(i > 0 && f > fr[i - 1])
			dtau += 0.5 * (rt[i - 1] + rate) * (actual_dt * (f - fr[i - 1]));
		if(PIECES >= 4)
		{
			if(i == 2)
				tau2_a = 0.5 * (rt[0] + rt[2]) * (actual_dt * (fr[2] - fr[0]));
			else if(i == 4)
				tau2 = tau2_a + 0.5 * (rt[2] + rate) * (actual_dt * (f - fr[2]));
		}
		else if(i > 0)
			tau2 += 0.5 * (rt[i - 1] + rate) * (actual_dt * (f - fr[i - 1]));
	}
}

// A finished RK45 step as the head of free_step_finish leaves it for the tail: the events and
// radii before and after it and its interior interval.
struct FinishCtx
{
	Event before, after;
	double r_before, rate_before, actual_dt, r_after, v_after, s0, s1;
	int interior;  // the chord enters the Sun (interior_interval)
	int depth;     // with a positive span and duration: the piece rates are formed
};

constexpr int PH_CONTINUE = -1;  // free_step_finish_head: the step goes on to its tail

// The checks after an attempt (src/Simulation_Trajectory.cpp:930-960) and the interior interval.
__device__ __forceinline__ int free_step_finish_head(const RunParams& R, StrictLane& L, int rk, FinishCtx& c)
{
	if(rk == RK_RETRY)
		return PH_STEP;
	L.in_rk = 0;
	L.attempts += static_cast<uint64_t>(L.rk_inner);
	c.before = L.before;
	c.r_before = L.b_radius < 0.0 ? 0.0 : L.b_radius;
	c.rate_before = L.rate_before;
	c.actual_dt = L.pr.time - L.b_time;
	c.r_after = prop_radius(L.pr);
	c.v_after = prop_speed(L.pr);
	c.after = prop_event(L.pr);
	if(rk == RK_FORCED)
	{
		set_final(L, c.after, true, DMS_REASON_NUMERICAL_FAILURE);
		return PH_FINAL;
	}
	if(!isfinite(c.r_after) || !isfinite(c.v_after) || !isfinite(c.actual_dt) || c.actual_dt <= 0.0)
	{
		set_final(L, c.after, true, DMS_REASON_NON_FINITE_STATE);
		return PH_FINAL;
	}
	if(c.v_after > DMS_V_MAX_C * DMS_C_KMS)
	{
		set_final(L, c.after, true, DMS_REASON_SPEED_LIMIT);
		return PH_FINAL;
	}
	if(wall_time_exceeded(R, L))  // "after_rk45_step", src/Simulation_Trajectory.cpp:953-954
	{
		set_final(L, c.after, true, DMS_REASON_WALL_TIME_LIMIT);
		return PH_FINAL;
	}
	c.s0 = 0.0;
	c.s1 = 0.0;
	c.interior = interior_interval(c.before, c.after, c.r_before, c.r_after, c.s0, c.s1) ? 1 : 0;
	c.depth = (c.interior && c.s1 > c.s0 && c.actual_dt > 0.0) ? 1 : 0;
	return PH_CONTINUE;
}

// The optical depth, boundary and commit logic of a finished step (src/Simulation_Trajectory.cpp:
// 960-1116) from its piece boundaries fr and rates rt, their trapezoid sums dtau (pieces) and
// tau2 (two-piece estimate) and whether a rate was invalid.  next_ok: next_rate is the scattering
// rate at the propagator's state (rate_total at r_after, v_after), for the next step's head.
__device__ __forceinline__ int free_step_finish_tail(const RunParams& R, double m_dm, StrictLane& L, double2* hist,
                                                     const FinishCtx& c, const double (&fr)[DMS_MAX_OPTICAL_DEPTH_PIECES + 1],
                                                     const double (&rt)[DMS_MAX_OPTICAL_DEPTH_PIECES + 1], double dtau, double tau2, bool invalid,
                                                     bool next_ok, double next_rate)
{
	const DevSolar& S = R.S;
	const int capture_mode = R.capture_mode;
	const double tau_limit = capture_mode ? DMS_CAPTURE_MAX_OPTICAL_DEPTH_STEP : DMS_MAX_OPTICAL_DEPTH_STEP;
	bool scattering = false, reflection = false;
	Event accepted = c.after;
	if(c.interior)
	{
		// Build_Optical_Depth_Pieces, src/Simulation_Trajectory.cpp:347-414
		const int pieces = capture_mode ? DMS_CAPTURE_OPTICAL_DEPTH_PIECES : DMS_MAX_OPTICAL_DEPTH_PIECES;
		if(invalid || !isfinite(dtau) || dtau < 0.0)
		{
			set_final(L, c.after, true, DMS_REASON_NUMERICAL_FAILURE);
			return PH_FINAL;
		}
		const double scale = dtau > DMS_OPTICAL_DEPTH_ABS_TOL ? dtau : DMS_OPTICAL_DEPTH_ABS_TOL;
		const double rel = fabs(dtau - tau2) / scale;
		const bool reject_depth = dtau > tau_limit;
		const bool reject_acc = !capture_mode && rel > DMS_OPTICAL_DEPTH_REL_TOL;
		if(reject_depth || reject_acc)
		{
			L.retries++;
			if(L.retries > DMS_MAX_OPTICAL_DEPTH_RETRIES)
			{
				set_final(L, c.before, true, DMS_REASON_NUMERICAL_FAILURE);
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
			L.pr.time_step = sanitized_step(factor * c.actual_dt);
			return PH_STEP;  // L.before still describes the restored propagator
		}
		if(dtau >= L.tau)
		{
			double remaining = L.tau;
			for(int k = 0; k < pieces; k++)
			{
				if(!(fr[k + 1] > fr[k]))
					continue;
				const double pdt = c.actual_dt * (fr[k + 1] - fr[k]);
				const double ptau = 0.5 * (rt[k] + rt[k + 1]) * pdt;
				if(ptau >= remaining)
				{
					const double lf = solve_linear_rate(rt[k], rt[k + 1], pdt, remaining);
					const double f = fr[k] + lf * (fr[k + 1] - fr[k]);
					accepted = interpolate_event(c.before, c.after, f);
					scattering = true;
					break;
				}
				remaining -= ptau;
			}
			if(!scattering)
			{
				accepted = interpolate_event(c.before, c.after, c.s1);
				scattering = true;
			}
		}
		else
			L.tau -= dtau;
	}
	if(!scattering)
	{
		Event boundary_ev = c.after;
		double r_b = c.r_after, v_b = c.v_after;
		if(c.r_before < R.boundary && c.r_after >= R.boundary && c.r_after > c.r_before)
		{
			const double f = (R.boundary - c.r_before) / (c.r_after - c.r_before);
			boundary_ev = interpolate_event(c.before, c.after, f);
			r_b = ev_radius(boundary_ev);
			v_b = ev_speed(boundary_ev);
		}
		if(r_b >= R.boundary && r_b >= c.r_before && v_b > solar_vesc(S, r_b))
		{
			accepted = boundary_ev;
			reflection = true;
		}
		else if(r_b >= R.boundary && r_b >= c.r_before)
		{
			Event abs_b = boundary_ev;
			abs_b.t += L.origin;
			if(uncaptured_bound(S, m_dm, L, abs_b))
			{
				set_final(L, abs_b, false, DMS_REASON_NUMERICAL_FAILURE);
				return PH_FINAL;
			}
			Event inbound;
			if(bound_kepler_return(boundary_ev, inbound))
			{
				L.seg_steps++;
				L.steps++;
				L.retries = 0;
				commit_event(S, m_dm, capture_mode, L, hist, boundary_ev);
				// reset_propagator_at_absolute_event, src/Simulation_Trajectory.cpp:814-822
				L.cur = inbound;
				L.cur.t += L.origin;
				L.origin = L.cur.t;
				Event local = inbound;
				local.t = 0.0;
				prop_init(L.pr, local);
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
	double E = commit_event(S, m_dm, capture_mode, L, hist, accepted);
	L.cur = accepted;
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
	L.before = c.after;
	// the propagator is left as the attempt made it: the next step starts from its speed and rate
	L.next_valid = next_ok ? 1 : 0;
	L.next_speed = c.v_after;
	L.next_rate = next_rate;
	return PH_STEP;
}

// A finished step on one lane: the piece rates one after another (one copy of the lookup).
__device__ __forceinline__ int free_step_finish(const RunParams& R, const DevPoint* __restrict__ P, double m_dm, StrictLane& L,
                                                double2* hist, int rk)
{
	const DevSolar& S = R.S;
	const int capture_mode = R.capture_mode;
	FinishCtx c;
	const int ph = free_step_finish_head(R, L, rk, c);
	if(ph != PH_CONTINUE)
		return ph;
	const int pieces = capture_mode ? DMS_CAPTURE_OPTICAL_DEPTH_PIECES : DMS_MAX_OPTICAL_DEPTH_PIECES;
	const bool use_cached = c.r_before < DMS_RSUN_KM && c.s0 <= 1.0e-12;
	const double span = c.s1 - c.s0;
	double fr[DMS_MAX_OPTICAL_DEPTH_PIECES + 1], rt[DMS_MAX_OPTICAL_DEPTH_PIECES + 1];
	bool invalid = false;
	double dtau = 0.0, tau2 = 0.0;
	if(c.depth)
	{
		// One loop over the piece boundaries (one copy of the rate lookup); the trapezoid
		// sums are formed as the rates arrive, in the reference's order.  The arrays keep
		// the boundaries for the scattering-point search, which is rare.
		double fr_prev = 0.0, rt_prev = 0.0, fr_0 = 0.0, rt_0 = 0.0, fr_2 = 0.0, rt_2 = 0.0, tau2_a = 0.0;
#pragma unroll 1
		for(int i = 0; i <= pieces; i++)
		{
			const double f = c.s0 + static_cast<double>(i) / static_cast<double>(pieces) * span;
			const double rate = (i == 0 && use_cached) ? c.rate_before : rate_at_fraction(S, P, c.before, c.after, f);
			fr[i] = f;
			rt[i] = rate;
			if(!isfinite(rate) || rate < 0.0)
				invalid = true;
			if(i > 0 && f > fr_prev)
				dtau += 0.5 * (rt_prev + rate) * (c.actual_dt * (f - fr_prev));
			if(pieces >= 4)
			{
				// two-piece estimate over [0, 2] and [2, 4]
				if(i == 0)
				{
					fr_0 = f;
					rt_0 = rate;
				}
				else if(i == 2)
				{
					fr_2 = f;
					rt_2 = rate;
					tau2_a = 0.5 * (rt_0 + rt_2) * (c.actual_dt * (fr_2 - fr_0));
				}
				else if(i == 4)
					tau2 = tau2_a + 0.5 * (rt_2 + rate) * (c.actual_dt * (f - fr_2));
			}
			else if(i > 0)
				tau2 += 0.5 * (rt_prev + rate) * (c.actual_dt * (f - fr_prev));
			fr_prev = f;
			rt_prev = rate;
		}
	}
	return free_step_finish_tail(R, m_dm, L, hist, c, fr, rt, dtau, tau2, invalid, false, 0.0);
}

// One piece-boundary rate of a step (rate_at_fraction at fraction f) or, for the job `next`, the
// scattering rate at the propagator's state after the step (rate_total at ra, va, as the next
// step's head forms it when ra is inside the Sun); the two share the code path, so that the lanes
// of a warp that form them run converged.
__device__ __forceinline__ double depth_job_rate(const DevSolar& S, const DevPoint* __restrict__ P, const Event& a, const Event& b, double f,
                                                 bool next, double ra, double va)
{
	f = clamp_unit(f);
	const double x = a.x.x + f * (b.x.x - a.x.x), vx = a.v.x + f * (b.v.x - a.v.x);
	const double y = a.x.y + f * (b.x.y - a.x.y), vy = a.v.y + f * (b.v.y - a.v.y);
	const double z = a.x.z + f * (b.x.z - a.x.z), vz = a.v.z + f * (b.v.z - a.v.z);
	double r2 = 0.0, v2 = 0.0;
	r2 += x * x;
	v2 += vx * vx;
	r2 += y * y;
	v2 += vy * vy;
	r2 += z * z;
	v2 += vz * vz;
	double r = sqrt(r2 > 0.0 ? r2 : 0.0), v = sqrt(v2 > 0.0 ? v2 : 0.0);
	if(next)
	{
		r = ra;
		v = va;
	}
	if(r >= DMS_RSUN_KM)
		return 0.0;
	return rate_total(S, P, r, v);
}

__device__ __forceinline__ double shfl_d(double v, int src) { return __shfl_sync(0xffffffffu, v, src); }

// The piece rates of every lane of the warp in `dm` (the lanes whose finished step needs them),
// formed by the whole warp at once: job j of a step (j = 0..PIECES, the boundaries; PIECES + 1,
// the next step's rate) runs on its own lane with the step's events broadcast from its owner,
// in as many rounds of 32 jobs as the steps need.  Each lookup is the function and arguments of
// the one-lane loop, so the rates are the same numbers.  Every lane of the warp calls this.
template <int PIECES>
__device__ __forceinline__ void coop_depth_rates(const RunParams& R, const DevPoint* __restrict__ P, const FinishCtx& c, bool depth,
                                                 unsigned int dm, double (&fr)[DMS_MAX_OPTICAL_DEPTH_PIECES + 1],
                                                 double (&rt)[DMS_MAX_OPTICAL_DEPTH_PIECES + 1], double& next_rate)
{
	constexpr int J = PIECES + 2;
	const int me = threadIdx.x & 31;
	const int jobs = __popc(dm) * J;
	const int rank = __popc(dm & ((1u << me) - 1u));  // among the lanes of dm (when depth)
	const double span = c.s1 - c.s0;
	for(int base = 0; base < jobs; base += 32)
	{
		const int job = base + me;
		const bool active = job < jobs;
		const int oi = active ? job / J : 0;
		const int j = active ? job - oi * J : 0;
		const int owner = nth_set_bit(dm, oi);
		Event a, b;
		a.x = mk(shfl_d(c.before.x.x, owner), shfl_d(c.before.x.y, owner), shfl_d(c.before.x.z, owner));
		a.v = mk(shfl_d(c.before.v.x, owner), shfl_d(c.before.v.y, owner), shfl_d(c.before.v.z, owner));
		b.x = mk(shfl_d(c.after.x.x, owner), shfl_d(c.after.x.y, owner), shfl_d(c.after.x.z, owner));
		b.v = mk(shfl_d(c.after.v.x, owner), shfl_d(c.after.v.y, owner), shfl_d(c.after.v.z, owner));
		const double s0 = shfl_d(c.s0, owner), sp = shfl_d(span, owner);
		const double ra = shfl_d(c.r_after, owner), va = shfl_d(c.v_after, owner);
		const DevPoint* Po = reinterpret_cast<const DevPoint*>(__shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(P), owner));
		double rate = 0.0;
		if(active)
			rate = depth_job_rate(R.S, Po, a, b, s0 + static_cast<double>(j) / static_cast<double>(PIECES) * sp, j == J - 1, ra, va);
#pragma unroll
		for(int jj = 0; jj < J; jj++)
		{
			const int src = rank * J + jj - base;
			const bool here = depth && src >= 0 && src < 32;
			const double v = shfl_d(rate, here ? src : me);
			if(here)
			{
				if(jj < J - 1)
					rt[jj] = v;
				else
					next_rate = v;
			}
		}
	}
	if(depth)
	{
#pragma unroll
		for(int i = 0; i <= PIECES; i++)
			fr[i] = c.s0 + static_cast<double>(i) / static_cast<double>(PIECES) * span;
		if(c.r_before < DMS_RSUN_KM && c.s0 <= 1.0e-12)
			rt[0] = c.rate_before;
	}
}

// A finished step on every lane of the warp that holds one (want), the piece rates formed by the
// whole warp (coop_depth_rates).  Every lane of the warp calls this; the others only help.
__device__ __forceinline__ int free_step_finish_warp(const RunParams& R, const DevPoint* __restrict__ P, double m_dm, StrictLane& L,
                                                     double2* hist, int rk, bool want)
{
	FinishCtx c = {};
	int ph = PH_STEP;
	if(want)
		ph = free_step_finish_head(R, L, rk, c);
	const bool depth = want && ph == PH_CONTINUE && c.depth;
	const unsigned int dm = __ballot_sync(0xffffffffu, depth);
	double fr[DMS_MAX_OPTICAL_DEPTH_PIECES + 1], rt[DMS_MAX_OPTICAL_DEPTH_PIECES + 1];
	double next_rate = 0.0, dtau = 0.0, tau2 = 0.0;
	bool invalid = false;
	if(dm != 0u)
	{
		if(R.capture_mode)
			coop_depth_rates<DMS_CAPTURE_OPTICAL_DEPTH_PIECES>(R, P, c, depth, dm, fr, rt, next_rate);
		else
			coop_depth_rates<DMS_MAX_OPTICAL_DEPTH_PIECES>(R, P, c, depth, dm, fr, rt, next_rate);
	}
	if(depth)
	{
		if(R.capture_mode)
			depth_sums<DMS_CAPTURE_OPTICAL_DEPTH_PIECES>(fr, rt, c.actual_dt, dtau, tau2, invalid);
		else
			depth_sums<DMS_MAX_OPTICAL_DEPTH_PIECES>(fr, rt, c.actual_dt, dtau, tau2, invalid);
	}
	if(want && ph == PH_CONTINUE)
		return free_step_finish_tail(R, m_dm, L, hist, c, fr, rt, dtau, tau2, invalid, depth, next_rate);
	return ph;
}

// Initial_Conditions + Hyperbolic_Kepler_Shift of every work index (src/Data_Generation.cpp:747-761,
// src/Simulation_Utilities.cpp:123-321), one thread each, ahead of the trajectory launch: the
// rejection loops of the halo sampler and the hyperbolic shift run here at full occupancy
// instead of inside the persistent kernel, where one starting lane would hold its warp.
__global__ void __launch_bounds__(128) initial_state_kernel(const RunParams R)
{
	const uint64_t w = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
	if(w >= R.total)
		return;
	int k = find_range(R, w);
	DMS_CHECK_INDEX(k, 0, R.n_ranges, BOUNDS_RANGE);
	const int point = R.range_point[k];
	Draws D;
	D.seed = R.seed;
	D.point = static_cast<uint32_t>(point);
	D.traj = R.range_first[k] + (w - R.range_offset[k]);
	D.index = 0;
	Event ic;
	const bool ok = initial_conditions(R.S, R.points + point, D, ic, R.ic_max_attempts);
	if(!ok)
		atomicOr(R.status, STATUS_IC_REJECTION);
	const bool shifted = ok && hyperbolic_kepler_shift(ic, R.boundary);
	InitState st;
	st.ic = ic;
	st.draws = static_cast<uint32_t>(D.index);
	st.flags = (ok ? INIT_IC_OK : 0u) | (shifted ? INIT_SHIFT_OK : 0u);
	R.init[w] = st;
}

// ---------------------------------------------------------------------------------------------
// Tail pipeline.  A lane that runs alone spends its step on one dependent chain, and the
// divergent paths of a warp do not overlap, but two warps do.  So once a block has drained, a
// warp whose lanes are all done stays as the block's helper: a stepping lane (the owner) hands it
// its propagator through shared memory, the helper makes the step's head (free_step_begin) and
// its RK45 attempts (paired on its lanes 0 and 1), and the owner adopts the result.  Right after
// adopting, the owner hands over the next step's start, computed as if the step it is about to
// finish ends plainly (the propagator unchanged, one more free step), and finishes the step
// meanwhile.  It adopts that speculative result only when its state is then bit for bit the one
// the speculation started from; otherwise it discards it and hands over its actual state.  The
// helper runs the same functions on the same values, so the results are the same.  One owner per
// block; every wait is bounded by the global timer, and a wait that runs out detaches the owner,
// which then steps on its own.
enum PipeState : int
{
	PIPE_NONE = 0,      // no helper
	PIPE_FREE = 1,      // a helper waits for an owner
	PIPE_ATTACHED = 2,
	PIPE_CLOSED = 3,
};

struct PipeBox
{
	int state, job, done;  // job / done: sequence numbers of the hand-over and of its result
	int begin_phase, rk, rk_inner;
	const DevPoint* P;
	uint64_t seg_in;
	Prop pr_in, pr_out;
	Event before_out;
	double b_time, b_radius, b_phi, b_vr, b_step, rate_before;
};

__device__ __forceinline__ PipeBox& pipe_box()
{
	__shared__ PipeBox box;
	return box;
}

// bounds of the waits, in SM clock cycles (about 2 GHz)
constexpr long long PIPE_WAIT_CYCLES = 2000000ll;            // an owner's wait for a result (~1 ms, 100 steps)
constexpr long long PIPE_IDLE_FREE_CYCLES = 400000ll;        // a helper without owner leaves after ~0.2 ms
constexpr long long PIPE_IDLE_ATTACHED_CYCLES = 10000000ll;  // ~5 ms (an owner hands over every step)

__device__ __forceinline__ bool pipe_wait(const PipeBox& b, int seq)
{
	const long long t0 = clock64();
	while(*reinterpret_cast<const volatile int*>(&b.done) != seq)
	{
		if(clock64() - t0 > PIPE_WAIT_CYCLES)
			return false;
		__nanosleep(32);  // leaves the issue slots to the other warps of the SM
	}
	__threadfence_block();
	return true;
}

__device__ __forceinline__ bool same_prop(const Prop& a, const Prop& b)
{
	auto eq = [](double x, double y) { return __double_as_longlong(x) == __double_as_longlong(y); };
	return eq(a.time, b.time) && eq(a.radius, b.radius) && eq(a.phi, b.phi) && eq(a.v_radial, b.v_radial) && eq(a.J, b.J) &&
	       eq(a.time_step, b.time_step) && eq(a.ax.x, b.ax.x) && eq(a.ax.y, b.ax.y) && eq(a.ax.z, b.ax.z) && eq(a.ay.x, b.ay.x) &&
	       eq(a.ay.y, b.ay.y) && eq(a.ay.z, b.ay.z) && a.radial_mode == b.radial_mode;
}

struct StrictStep
{
	// the lane loop runs a step as begin / attempt / finish and may pair the attempt of a lane
	// with an idle lane of its warp (rk45_attempt_pair)
	static constexpr bool pairs = DMS_PAIRED_ATTEMPTS != 0 && DMS_CERTIFIED_MATH != 0 && DMS_RK_UNROLLED >= 1;
	__device__ __forceinline__ int begin(const RunParams& R, const DevPoint* __restrict__ P, StrictLane& L) const
	{
		return free_step_begin(R, P, L);
	}
	__device__ __forceinline__ int attempt(const DevSolar& S, StrictLane& L, int drained) const
	{
		return free_step_attempt(S, L, drained);
	}
	// all lanes of the warp call this; role 1 = owner (its attempt), 2 = helper, 0 = neither
	__device__ __forceinline__ int pair_attempt(const DevSolar& S, StrictLane& L, int role, int partner) const
	{
		if(role == 1)
			L.rk_inner++;
		bool good = S.bucket_single_step != 0;
		const int rk = rk45_attempt_pair(S, L.pr, L.rk_inner, role, partner, good);
		if(role == 1 && !good)
			return rk45_attempt_ieee(S, L.pr, L.rk_inner);
		return rk;
	}
	__device__ __forceinline__ int finish(const RunParams& R, const DevPoint* __restrict__ P, double m_dm, StrictLane& L, double2* hist,
	                                      int rk) const
	{
		return free_step_finish(R, P, m_dm, L, hist, rk);
	}
	// the finish of the paired attempts: all lanes of the warp call this (want: the lane's own)
	__device__ __forceinline__ int finish_warp(const RunParams& R, const DevPoint* __restrict__ P, double m_dm, StrictLane& L, double2* hist,
	                                           int rk, bool want) const
	{
		return free_step_finish_warp(R, P, m_dm, L, hist, rk, want);
	}
	__device__ __forceinline__ int operator()(const RunParams& R, const DevPoint* __restrict__ P, double m_dm, StrictLane& L, double2* hist,
	                                          int drained) const
	{
		const int ph = begin(R, P, L);
		if(ph != PH_STEP)
			return ph;
		return finish(R, P, m_dm, L, hist, attempt(R.S, L, drained));
	}
	__device__ __forceinline__ double channel(const DevSolar& S, const DevPoint* __restrict__ P, int i, double dr, double T, double v, int k) const
	{
		return channel_rate(S, P, i, dr, T, v, k);
	}
	__device__ __forceinline__ bool scatter(const DevSolar& S, const DevPoint* __restrict__ P, Draws& D, Event& e, int target) const
	{
		return scatter_with_target(S, P, D, e, target);
	}

	// ---- tail pipeline (see PipeBox) ----
	static constexpr bool pipeline = DMS_TAIL_PIPELINE != 0 && pairs;
	__device__ __forceinline__ void pipe_init() const
	{
		PipeBox& b = pipe_box();
		b.state = PIPE_NONE;
		b.job = 0;
		b.done = 0;
	}
	// all lanes of a warp whose lanes are all done call this; it returns when the warp leaves
	// (it was not needed as the helper, or it has served its last owner)
	__device__ void pipe_serve(const RunParams& R, StrictLane& L) const
	{
		PipeBox& b = pipe_box();
		const int me = threadIdx.x & 31;
		int became = 0;
		if(me == 0)
			became = atomicCAS(&b.state, PIPE_NONE, PIPE_FREE) == PIPE_NONE ? 1 : 0;
		if(__shfl_sync(0xffffffffu, became, 0) == 0)
			return;
		// a helper that served before this one left every hand-over answered (done == job)
		int last = __shfl_sync(0xffffffffu, *reinterpret_cast<volatile int*>(&b.job), 0);
		long long idle_since = clock64();
		for(unsigned int poll = 0;; poll++)
		{
			const int job = __shfl_sync(0xffffffffu, *reinterpret_cast<volatile int*>(&b.job), 0);
			if(job != last)
			{
				__threadfence_block();
				pipe_job(R, L, b);
				__threadfence_block();
				if(me == 0)
					*reinterpret_cast<volatile int*>(&b.done) = job;
				last = job;
				idle_since = clock64();
				continue;
			}
			const int st = __shfl_sync(0xffffffffu, *reinterpret_cast<volatile int*>(&b.state), 0);
			const long long idle = clock64() - idle_since;
			// the cancel flag lives in host memory: read it rarely
			const bool cancelled = (poll & 4095u) == 4095u && __any_sync(0xffffffffu, *R.cancel != 0);
			if(cancelled || (st == PIPE_FREE && idle > PIPE_IDLE_FREE_CYCLES) || (st != PIPE_FREE && idle > PIPE_IDLE_ATTACHED_CYCLES))
			{
				int closed = 1;
				if(me == 0)
				{
					// without an owner the box is left for a warp that is done later; an owner may
					// attach meanwhile, and then the helper stays
					if(st == PIPE_FREE && !cancelled)
						closed = atomicCAS(&b.state, PIPE_FREE, PIPE_NONE) == PIPE_FREE ? 1 : 0;
					else
						atomicExch(&b.state, PIPE_CLOSED);
				}
				if(__shfl_sync(0xffffffffu, closed, 0))
					return;
				continue;
			}
			__nanosleep(64);
		}
	}
	// the helper's work for one hand-over: the step's head on lane 0 (its own lane state as
	// scratch), then the RK45 attempts paired on lanes 0 and 1 until one is not retried
	__device__ __forceinline__ void pipe_job(const RunParams& R, StrictLane& L, PipeBox& b) const
	{
		const int me = threadIdx.x & 31;
		int ph = PH_STEP;
		if(me == 0)
		{
			L.pr = b.pr_in;
			L.seg_steps = b.seg_in;
			L.before_valid = 0;  // the head forms Event_In_3D of the propagator (= the owner's cached one)
			L.next_valid = 0;
			L.in_rk = 0;
			ph = free_step_begin(R, b.P, L);
		}
		ph = __shfl_sync(0xffffffffu, ph, 0);
		int rk = RK_RETRY, passes = 0;
		if(ph == PH_STEP)
		{
			const int role = me == 0 ? 1 : (me == 1 ? 2 : 0);
			const int partner = me == 0 ? 1 : 0;
			while(rk == RK_RETRY && passes <= DMS_RK45_MAX_INNER_RETRIES + 1)
			{
				rk = __shfl_sync(0xffffffffu, pair_attempt(R.S, L, role, partner), 0);
				passes++;
			}
		}
		if(me == 0)
		{
			b.begin_phase = (ph == PH_STEP && rk == RK_RETRY) ? PH_FINAL : ph;  // a step that never ended: the owner steps alone
			b.rk = rk;
			b.rk_inner = L.rk_inner;
			b.pr_out = L.pr;
			b.before_out = L.before;
			b.b_time = L.b_time;
			b.b_radius = L.b_radius;
			b.b_phi = L.b_phi;
			b.b_vr = L.b_vr;
			b.b_step = L.b_step;
			b.rate_before = L.rate_before;
		}
	}
	__device__ __forceinline__ bool pipe_attach() const
	{
		PipeBox& b = pipe_box();
		return *reinterpret_cast<volatile int*>(&b.state) == PIPE_FREE && atomicCAS(&b.state, PIPE_FREE, PIPE_ATTACHED) == PIPE_FREE;
	}
	__device__ __forceinline__ int pipe_post(const DevPoint* __restrict__ P, const Prop& pr, uint64_t seg) const
	{
		PipeBox& b = pipe_box();
		b.P = P;
		b.pr_in = pr;
		b.seg_in = seg;
		__threadfence_block();
		const int seq = b.job + 1;
		*reinterpret_cast<volatile int*>(&b.job) = seq;
		return seq;
	}
	__device__ __forceinline__ void pipe_adopt(const PipeBox& b, StrictLane& L) const
	{
		L.pr = b.pr_out;
		L.before = b.before_out;
		L.before_valid = 1;
		L.next_valid = 0;
		L.b_time = b.b_time;
		L.b_radius = b.b_radius;
		L.b_phi = b.b_phi;
		L.b_vr = b.b_vr;
		L.b_step = b.b_step;
		L.rate_before = b.rate_before;
		L.in_rk = 1;
		L.rk_inner = b.rk_inner;
	}
	// the owner's step start: 1 = adopted (rk set), 0 = make the head here, -1 = detached
	__device__ __forceinline__ int pipe_step(const DevPoint* __restrict__ P, StrictLane& L, int& spec, int& rk) const
	{
		PipeBox& b = pipe_box();
		if(*reinterpret_cast<volatile int*>(&b.state) != PIPE_ATTACHED)
		{
			spec = 0;
			return -1;  // the helper has left
		}
		if(spec != 0)
		{
			const int s = spec;
			spec = 0;
			if(!pipe_wait(b, s))
				return -1;
			if(b.begin_phase == PH_STEP && b.P == P && b.seg_in == L.seg_steps && same_prop(b.pr_in, L.pr))
			{
				pipe_adopt(b, L);
				rk = b.rk;
				return 1;
			}
		}
		const int s = pipe_post(P, L.pr, L.seg_steps);
		if(!pipe_wait(b, s))
			return -1;
		if(b.begin_phase != PH_STEP)
			return 0;
		pipe_adopt(b, L);
		rk = b.rk;
		return 1;
	}
	__device__ __forceinline__ void pipe_release(int& spec) const
	{
		PipeBox& b = pipe_box();
		if(spec != 0)
			pipe_wait(b, spec);
		spec = 0;
		atomicCAS(&b.state, PIPE_ATTACHED, PIPE_FREE);
	}
};

__global__ void __launch_bounds__(128, DMS_TRAJ_MIN_BLOCKS) trajectory_kernel(const RunParams R)
{
	lane_loop<StrictLane>(R, StrictStep());
}

__global__ void rate_grid_kernel(const DevSolar S, const DevPoint* __restrict__ P, double* grid, int n)
{
	const size_t total = static_cast<size_t>(n) * n;
	for(size_t k = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; k < total; k += static_cast<size_t>(gridDim.x) * blockDim.x)
	{
		const int i = static_cast<int>(k / n), j = static_cast<int>(k % n);
		// src/Solar_Model.cpp:438-447: radius = R i/(N-1), speed = Linear_Space(0, 0.75, N)[j]
		const double radius = DMS_RSUN_KM * static_cast<double>(i) / static_cast<double>(n - 1);
		const double vstep_c = (DMS_V_MAX_C - 0.0) / (n - 1);
		const double speed = (0.0 + j * vstep_c) * DMS_C_KMS;
		grid[k] = rate_computed(S, P, radius, speed, nullptr, nullptr);
	}
}

__global__ void rate_query_kernel(const DevSolar S, const DevPoint* __restrict__ P, int interpolated, const double* r, const double* v, double* out, size_t n)
{
	const size_t k = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
	if(k >= n)
		return;
	out[k] = interpolated ? rate_total(S, P, r[k], v[k]) : rate_computed(S, P, r[k], v[k], nullptr, nullptr);
}

// Independent DFMA chains: 8 accumulators per thread, `iters` iterations.
__global__ void __launch_bounds__(256) fp64_fma_probe_kernel(double* out, int iters, double b, double c)
{
	double a0 = threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
	for(int i = 0; i < iters; i++)
	{
		a0 = fma(a0, b, c);
		a1 = fma(a1, b, c);
		a2 = fma(a2, b, c);
		a3 = fma(a3, b, c);
		a4 = fma(a4, b, c);
		a5 = fma(a5, b, c);
		a6 = fma(a6, b, c);
		a7 = fma(a7, b, c);
	}
	const double s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
	if(s == 1.2345)
		out[0] = s;
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t x)
{
	x += 0x9e3779b97f4a7c15ULL;
	x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
	x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
	return x ^ (x >> 31);
}

// A double with random significand and an exponent uniform in [lo, hi].
__device__ __forceinline__ double random_double(uint64_t bits, int lo, int hi)
{
	const int e = lo + static_cast<int>((bits >> 52) % static_cast<uint64_t>(hi - lo + 1));
	const uint64_t mant = bits & 0x000fffffffffffffULL;
	return __longlong_as_double(static_cast<long long>((static_cast<uint64_t>(e + 1023) << 52) | mant));
}

// Self-test of the certified division and square root against IEEE `/` and sqrt on n random
// operand pairs: out[0] quotients whose certificate held but whose bits differ from IEEE (must
// be 0), out[1] quotients whose certificate failed, out[2] and out[3] the same for the root.
// Operands: random exponents in the ranges of the trajectory arithmetic, arbitrary bit patterns
// (NaN, infinities, subnormals, zeros), quotients within a few ulp of representable values,
// and exact quotients (a power-of-two divisor).  Division and square root never land exactly
// halfway between two doubles, so round-to-nearest has no ties to test.
__global__ void certified_math_check_kernel(uint64_t n, uint64_t seed, unsigned long long* out)
{
	unsigned long long c[4] = {0, 0, 0, 0};
	for(uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < n; k += static_cast<uint64_t>(gridDim.x) * blockDim.x)
	{
		const uint64_t h1 = splitmix64(seed ^ (k * 0x2545f4914f6cdd1dULL)), h2 = splitmix64(h1), h3 = splitmix64(h2);
		double a, b;
		switch(k & 3)
		{
			case 0:  // the trajectory ranges: km, km/s, s, km^3/s^2
				a = random_double(h1, -40, 70);
				b = random_double(h2, -20, 40);
				break;
			case 1:  // any bit pattern
				a = __longlong_as_double(static_cast<long long>(h1));
				b = __longlong_as_double(static_cast<long long>(h2));
				break;
			case 2:
			{  // dividend a few ulp away from b * q for a random q
				b = random_double(h1, -30, 30);
				const double q = random_double(h2, -30, 30);
				const long long d = static_cast<long long>(h3 % 7) - 3;
				a = __longlong_as_double(__double_as_longlong(__dmul_rn(b, q)) + d);
				break;
			}
			default:
			{  // exact quotients: a power-of-two divisor
				const double m = random_double(h1, -10, 10);
				b = ldexp(1.0, static_cast<int>(h2 % 41) - 20);
				a = __dmul_rn(b, m);
				break;
			}
		}
		if(h3 & 1)
			a = -a;
		bool ok = true;
		const double q = fast::div(a, b, ok);
		const double ref = a / b;
		if(!ok)
			c[1]++;
		else if(__double_as_longlong(q) != __double_as_longlong(ref) && !(isnan(q) && isnan(ref)))
			c[0]++;
		const double x = fabs(a);
		bool ok2 = true;
		const double sq = fast::sqrt(x, ok2);
		const double sref = sqrt(x);
		if(!ok2)
			c[3]++;
		else if(__double_as_longlong(sq) != __double_as_longlong(sref) && !(isnan(sq) && isnan(sref)))
			c[2]++;
	}
	for(int i = 0; i < 4; i++)
		if(c[i])
			atomicAdd(out + i, c[i]);
}

}	// namespace

void Check_Certified_Math(uint64_t n, uint64_t seed, unsigned long long* out, int sm_count, cudaStream_t stream)
{
	certified_math_check_kernel<<<sm_count * 8, 256, 0, stream>>>(n, seed, out);
}

double Measure_FP64_Peak(int sm_count, cudaStream_t stream)
{
	double* d = nullptr;
	if(cudaMalloc(&d, sizeof(double)) != cudaSuccess)
		return -1.0;
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	const int blocks = sm_count * 8, threads = 256, iters = 1 << 16;
	fp64_fma_probe_kernel<<<blocks, threads, 0, stream>>>(d, 1024, 0.999999, 1e-9);
	cudaEventRecord(e0, stream);
	fp64_fma_probe_kernel<<<blocks, threads, 0, stream>>>(d, iters, 0.999999, 1e-9);
	cudaEventRecord(e1, stream);
	float ms = 0.0f;
	const bool ok = cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	cudaFree(d);
	if(!ok || ms <= 0.0f)
		return -1.0;
	const double flops = 2.0 * 8.0 * iters * static_cast<double>(blocks) * threads;
	return flops / (ms * 1.0e-3) / 1.0e12;
}

void Launch_Initial_States(const RunParams& p, cudaStream_t stream)
{
	const uint64_t blocks = (p.total + 127) / 128;
	if(blocks > 0)
		initial_state_kernel<<<static_cast<unsigned int>(blocks), 128, 0, stream>>>(p);
}

void Launch_Trajectories(const RunParams& p, int blocks, int threads, cudaStream_t stream)
{
	trajectory_kernel<<<blocks, threads, 0, stream>>>(p);
}

void Launch_Rate_Grid(const DevSolar& S, const DevPoint* point, double* grid, int n, cudaStream_t stream)
{
	rate_grid_kernel<<<148 * 8, 256, 0, stream>>>(S, point, grid, n);
}

void Launch_Rate_Query(const DevSolar& S, const DevPoint* point, int interpolated, const double* r, const double* v, double* out,
                       size_t n, cudaStream_t stream)
{
	const int threads = 128;
	const int blocks = static_cast<int>((n + threads - 1) / threads);
	if(blocks > 0)
		rate_query_kernel<<<blocks, threads, 0, stream>>>(S, point, interpolated, r, v, out, n);
}

int Trajectory_Max_Blocks_Per_SM(int threads)
{
	int n = 0;
	if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, trajectory_kernel, threads, 0) != cudaSuccess)
		return 0;
	return n;
}

int Trajectory_Kernel_Registers()
{
	cudaFuncAttributes a;
	if(cudaFuncGetAttributes(&a, trajectory_kernel) != cudaSuccess)
		return -1;
	return a.numRegs;
}

unsigned int Take_Bounds_Status()
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
