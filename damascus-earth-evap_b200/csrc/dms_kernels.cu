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
#include "dms_kernels.cuh"

namespace dms
{

namespace
{

enum Phase : int
{
	PH_FETCH = 0,
	PH_SEGMENT = 1,
	PH_STEP = 2,
	PH_FINAL = 3,
	PH_DONE = 4,
};

// Trajectory state of a lane (TrajectoryBincount + Trajectory_Simulator members,
// include/Simulation_Trajectory.hpp:53-154).
struct Lane
{
	uint64_t work;
	int point;
	Draws D;
	Event cur;           // absolute event at segment boundaries and at termination
	Prop pr;             // propagator of the current free segment (local time)
	Event before;        // Event_In_3D of the propagator at the start of the step (cached)
	double origin;       // absolute time of the segment's local t = 0
	double tau;          // remaining optical depth to the next scattering (minus_log_xi)
	uint64_t seg_steps;
	uint64_t nscat;
	uint64_t steps;      // accepted free steps of the whole trajectory (work counter)
	uint64_t attempts;   // RK45 attempts of the whole trajectory (work counter)
	unsigned int retries;
	int before_valid;
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
};

__device__ __forceinline__ void accumulate_bincount(Lane& L, double2* hist, double r, double v2, double dt)
{
	// Accumulate_Bincount_Step, src/Simulation_Trajectory.cpp:640-669
	if(!isfinite(dt) || dt <= 0.0)
		return;
	int bin = -1;
	if(isfinite(r) && r >= 0.0 && r < DMS_BIN_MAX_KM)
	{
		bin = static_cast<int>(r / DMS_BIN_WIDTH_KM);
		if(bin < 0) bin = 0;
		if(bin >= DMS_NUM_BINS) bin = -1;
	}
	if(bin >= 0)
	{
		double2 h = hist[bin];
		h.x += dt;
		h.y += v2 * dt;
		hist[bin] = h;
		L.bmin = bin < L.bmin ? bin : L.bmin;
		L.bmax = bin > L.bmax ? bin : L.bmax;
	}
}

// Update_Capture_State, src/Simulation_Trajectory.cpp:689-760
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

__device__ __forceinline__ bool uncaptured_bound(const DevSolar& S, double m_dm, const Lane& L, const Event& e)
{
	if(L.is_captured)
		return false;
	const double E = capture_energy_eV(S, m_dm, ev_radius(e), ev_speed(e));
	if(isfinite(E) && E >= 0.0)
		return false;
	return true;
}

// commit_accepted_event, src/Simulation_Trajectory.cpp:842-874
__device__ __forceinline__ void commit_event(const DevSolar& S, double m_dm, int capture_mode, Lane& L, double2* hist, const Event& local)
{
	if(!capture_mode)
	{
		const double r_now = ev_radius(local);
		const double v_now = ev_speed(local);
		const double v2 = v_now * v_now;
		if(L.prev_time >= 0.0)
			accumulate_bincount(L, hist, L.prev_r, L.prev_v2, local.t - L.prev_time);
		L.prev_time = local.t;
		L.prev_r = r_now;
		L.prev_v2 = v2;
	}
	Event abs_e = local;
	abs_e.t += L.origin;
	update_capture_state(S, m_dm, capture_mode, L, ev_radius(abs_e), ev_speed(abs_e), abs_e.t, false);
}

__device__ __forceinline__ void set_final(Lane& L, const Event& local_or_abs, bool is_local, int reason)
{
	L.cur = local_or_abs;
	if(is_local)
		L.cur.t += L.origin;
	L.reason = reason;
}

// One outer iteration of the Propagate_Freely loop, src/Simulation_Trajectory.cpp:876-1116.
// Returns the next phase of the lane.
__device__ __forceinline__ int free_step(const RunParams& R, const DevPoint* __restrict__ P, double m_dm, Lane& L, double2* hist)
{
	const DevSolar& S = R.S;
	const int capture_mode = R.capture_mode;
	if(!(L.seg_steps < R.max_free_steps))
	{
		L.reason = DMS_REASON_MAX_FREE_STEPS;  // L.cur holds the last committed event
		return PH_FINAL;
	}
	const double tau_limit = capture_mode ? DMS_CAPTURE_MAX_OPTICAL_DEPTH_STEP : DMS_MAX_OPTICAL_DEPTH_STEP;
	if(!L.before_valid)
	{
		L.before = prop_event(L.pr);
		L.before_valid = 1;
	}
	const Event before = L.before;
	const double r_before = prop_radius(L.pr);
	const double v_before = prop_speed(L.pr);
	double rate_before = 0.0;
	if(r_before >= DMS_RSUN_KM)
	{
		const double cap = step_cap(r_before, v_before, R.boundary);
		const double ts = sanitized_step(L.pr.time_step);
		L.pr.time_step = ts < cap ? ts : cap;
		const double vr = (r_before > 0.0) ? dot3(before.x, before.v) / r_before : 0.0;
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
		rate_before = rate_total(S, P, r_before, v_before);
		if(!isfinite(rate_before) || rate_before < 0.0)
		{
			set_final(L, prop_event(L.pr), true, DMS_REASON_NUMERICAL_FAILURE);
			return PH_FINAL;
		}
		if(rate_before > 0.0 && tau_limit / rate_before < L.pr.time_step)
			L.pr.time_step = tau_limit / rate_before;
	}
	// the RK step changes only these propagator fields
	const double b_time = L.pr.time, b_radius = L.pr.radius, b_phi = L.pr.phi, b_vr = L.pr.v_radial, b_step = L.pr.time_step;
	const int rk = rk45_step(S, L.pr);
	L.attempts += static_cast<uint64_t>(rk < 0 ? -rk : rk);
	const double actual_dt = L.pr.time - b_time;
	const double r_after = prop_radius(L.pr);
	const double v_after = prop_speed(L.pr);
	const Event after = prop_event(L.pr);
	if(rk < 0)
	{
		set_final(L, after, true, DMS_REASON_NUMERICAL_FAILURE);
		return PH_FINAL;
	}
	if(!isfinite(r_after) || !isfinite(v_after) || !isfinite(actual_dt) || actual_dt <= 0.0)
	{
		set_final(L, after, true, DMS_REASON_NON_FINITE_STATE);
		return PH_FINAL;
	}
	if(v_after > DMS_V_MAX_C * DMS_C_KMS)
	{
		set_final(L, after, true, DMS_REASON_SPEED_LIMIT);
		return PH_FINAL;
	}
	bool scattering = false, reflection = false;
	Event accepted = after;
	double s0 = 0.0, s1 = 0.0;
	if(interior_interval(before, after, r_before, r_after, s0, s1))
	{
		// Build_Optical_Depth_Pieces, src/Simulation_Trajectory.cpp:347-414
		const int pieces = capture_mode ? DMS_CAPTURE_OPTICAL_DEPTH_PIECES : DMS_MAX_OPTICAL_DEPTH_PIECES;
		const bool use_cached = r_before < DMS_RSUN_KM && s0 <= 1.0e-12;
		const double span = s1 - s0;
		double fr[DMS_MAX_OPTICAL_DEPTH_PIECES + 1], rt[DMS_MAX_OPTICAL_DEPTH_PIECES + 1];
		bool invalid = false;
		double dtau = 0.0, tau2 = 0.0;
		if(s1 > s0 && actual_dt > 0.0)
		{
#pragma unroll
			for(int i = 0; i <= DMS_MAX_OPTICAL_DEPTH_PIECES; i++)
			{
				if(i > pieces)
					break;
				fr[i] = s0 + static_cast<double>(i) / static_cast<double>(pieces) * span;
				rt[i] = (i == 0 && use_cached) ? rate_before : rate_at_fraction(S, P, before, after, fr[i]);
				if(!isfinite(rt[i]) || rt[i] < 0.0)
					invalid = true;
			}
			if(!invalid)
			{
				if(pieces >= 4)
					tau2 = 0.5 * (rt[0] + rt[2]) * (actual_dt * (fr[2] - fr[0])) + 0.5 * (rt[2] + rt[4]) * (actual_dt * (fr[4] - fr[2]));
				else
					for(int i = 0; i < pieces; i++) tau2 += 0.5 * (rt[i] + rt[i + 1]) * (actual_dt * (fr[i + 1] - fr[i]));
				for(int i = 0; i < pieces; i++)
					if(fr[i + 1] > fr[i])
						dtau += 0.5 * (rt[i] + rt[i + 1]) * (actual_dt * (fr[i + 1] - fr[i]));
			}
		}
		if(invalid || !isfinite(dtau) || dtau < 0.0)
		{
			set_final(L, after, true, DMS_REASON_NUMERICAL_FAILURE);
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
				set_final(L, before, true, DMS_REASON_NUMERICAL_FAILURE);
				return PH_FINAL;
			}
			L.pr.time = b_time;
			L.pr.radius = b_radius;
			L.pr.phi = b_phi;
			L.pr.v_radial = b_vr;
			L.pr.time_step = b_step;
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
				const double pdt = actual_dt * (fr[k + 1] - fr[k]);
				const double ptau = 0.5 * (rt[k] + rt[k + 1]) * pdt;
				if(ptau >= remaining)
				{
					const double lf = solve_linear_rate(rt[k], rt[k + 1], pdt, remaining);
					const double f = fr[k] + lf * (fr[k + 1] - fr[k]);
					accepted = interpolate_event(before, after, f);
					scattering = true;
					break;
				}
				remaining -= ptau;
			}
			if(!scattering)
			{
				accepted = interpolate_event(before, after, s1);
				scattering = true;
			}
		}
		else
			L.tau -= dtau;
	}
	if(!scattering)
	{
		Event boundary_ev = after;
		double r_b = r_after, v_b = v_after;
		if(r_before < R.boundary && r_after >= R.boundary && r_after > r_before)
		{
			const double f = (R.boundary - r_before) / (r_after - r_before);
			boundary_ev = interpolate_event(before, after, f);
			r_b = ev_radius(boundary_ev);
			v_b = ev_speed(boundary_ev);
		}
		if(r_b >= R.boundary && r_b >= r_before && v_b > solar_vesc(S, r_b))
		{
			accepted = boundary_ev;
			reflection = true;
		}
		else if(r_b >= R.boundary && r_b >= r_before)
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
	commit_event(S, m_dm, capture_mode, L, hist, accepted);
	L.cur = accepted;
	L.cur.t += L.origin;
	if(uncaptured_bound(S, m_dm, L, L.cur))
	{
		L.reason = DMS_REASON_NUMERICAL_FAILURE;
		return PH_FINAL;
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
		if(!scatter(S, P, L.D, L.cur))
		{
			L.reason = DMS_REASON_NUMERICAL_FAILURE;
			return PH_FINAL;
		}
		L.nscat++;
		const bool captured = update_capture_state(S, m_dm, capture_mode, L, ev_radius(L.cur), ev_speed(L.cur), L.cur.t, true);
		if(!capture_mode)
		{
			// Reset_Bincount_Anchor, src/Simulation_Trajectory.cpp:671-680
			L.prev_time = L.cur.t;
			L.prev_r = ev_radius(L.cur);
			const double v = ev_speed(L.cur);
			L.prev_v2 = v * v;
		}
		if(capture_mode && captured)
		{
			L.reason = DMS_REASON_CAPTURE_MODE;
			return PH_FINAL;
		}
		return PH_SEGMENT;
	}
	L.before = after;
	return PH_STEP;
}

// Start of a free segment: Simulate loop head + Propagate_Freely prologue,
// src/Simulation_Trajectory.cpp:1311-1313, 762-805
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
	prop_init(L.pr, local);
	L.tau = -dms_log(L.D.positive_unit());
	L.seg_steps = 0;
	L.retries = 0;
	L.before_valid = 0;
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
__device__ __noinline__ void finalize(const RunParams& R, const DevPoint* __restrict__ P, double m_dm, Lane& L, double2* hist)
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
						flags |= DMS_REC_REFLECT_SHIFT_OK;
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

	const int b0 = L.bmin, b1 = L.bmax;
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
			double* hd = R.rec_hist_dt + L.work * DMS_NUM_BINS;
			double* hv = R.rec_hist_v2dt + L.work * DMS_NUM_BINS;
			for(int b = b0; b <= b1; b++)
			{
				const double2 h = hist[b];
				hd[b] = h.x;
				hv[b] = h.y;
			}
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
						dms_evaporation_event ev;
						ev.trajectory_id = L.D.traj + 1;
						ev.lifetime_unbinding = lifetime;
						R.events[static_cast<size_t>(L.point) * R.event_capacity + k] = ev;
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
			double* h_dt = h + (hist_slot + 0) * DMS_NUM_BINS;
			double* h_v2 = h + (hist_slot + 1) * DMS_NUM_BINS;
			double* h_dt_sq = h + (hist_slot + 4) * DMS_NUM_BINS;
			double* h_v2_sq = h + (hist_slot + 5) * DMS_NUM_BINS;
			for(int b = b0; b <= b1; b++)
			{
				const double2 x = hist[b];
				if(x.x != 0.0 || x.y != 0.0)
				{
					atomicAdd(h_dt + b, x.x);
					atomicAdd(h_v2 + b, x.y);
					atomicAdd(h_dt_sq + b, x.x * x.x);
					atomicAdd(h_v2_sq + b, x.y * x.y);
				}
			}
		}
	}
	for(int b = b0; b <= b1; b++) hist[b] = make_double2(0.0, 0.0);
}

// Picks up work index `w`: trajectory start = Initial_Conditions + Hyperbolic_Kepler_Shift and the
// Simulate prologue (src/Data_Generation.cpp:747-761, src/Simulation_Trajectory.cpp:1284-1308).
__device__ __forceinline__ int start_trajectory(const RunParams& R, Lane& L, uint64_t w, const DevPoint*& P, double& m_dm)
{
	int k = 0;
	while(k + 1 < R.n_ranges && w >= R.range_offset[k + 1]) k++;
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
	L.reason = DMS_REASON_UNKNOWN;
	Event ic;
	const bool ic_ok = initial_conditions(R.S, P, L.D, ic, R.ic_max_attempts);
	if(!ic_ok)
		atomicOr(R.status, STATUS_IC_REJECTION);
	L.shift_ok = ic_ok && hyperbolic_kepler_shift(ic, R.boundary);
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

__global__ void __launch_bounds__(128) trajectory_kernel(const RunParams R)
{
	const int lane_id = blockIdx.x * blockDim.x + threadIdx.x;
	double2* hist = R.lane_hist + static_cast<size_t>(lane_id) * DMS_NUM_BINS;
	Lane L;
	const DevPoint* P = R.points;
	double m_dm = 0.0;
	int phase = PH_FETCH;
	const unsigned int lane_bit = 1u << (threadIdx.x & 31);
	for(uint64_t iter = 0;; iter++)
	{
		if((iter & 1023) == 1023)
		{
			if(*R.cancel != 0)
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
			// warp-aggregated claim of one work index per lane that needs one
			const unsigned int mask = __activemask();
			const int leader = __ffs(mask) - 1;
			const unsigned int rank = __popc(mask & (lane_bit - 1u));
			unsigned long long base = 0;
			if((threadIdx.x & 31) == leader)
				base = atomicAdd(R.queue_head, static_cast<unsigned long long>(__popc(mask)));
			base = __shfl_sync(mask, base, leader);
			const uint64_t w = base + rank;
			if(w >= R.total)
				break;
			phase = start_trajectory(R, L, w, P, m_dm);
		}
		if(phase == PH_SEGMENT)
			phase = segment_start(R, P, m_dm, L);
		if(phase == PH_STEP)
			phase = free_step(R, P, m_dm, L, hist);
		if(phase == PH_FINAL)
		{
			finalize(R, P, m_dm, L, hist);
			phase = PH_FETCH;
		}
	}
	if(phase != PH_FETCH && L.bmax >= L.bmin)
		for(int b = L.bmin; b <= L.bmax; b++) hist[b] = make_double2(0.0, 0.0);
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

}	// namespace

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

}	// namespace dms
