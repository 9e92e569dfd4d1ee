// Mixed-precision physics of the trajectory engine (the "batched FP32" form).
//
// Bulk arithmetic runs in FP32: RK45 stages (with FP32 copies of the G*M table), the 3-D event
// reconstruction, chord geometry, rate interpolation (FP32 copy of the rate grid) and the
// scattering kinematics.  FP64 is kept where the precision decides: the propagator's
// accumulated state (radius, radial speed, angle, time) is FP64 and receives the FP32
// increments; the RK45 error norm is formed in FP64 from the FP32 stage values (as a direct
// weighted sum of the stage differences, free of the r5 - r4 cancellation); the orbital energy
// whose sign decides capture and unbinding, the optical depth still to travel, and the
// histogram / evaporation accumulators are FP64.  Same algorithm and draw sequence as the FP64
// form; results agree statistically, not bit for bit.
#pragma once

#include "dms_device.cuh"

namespace dms
{
namespace mixed
{

struct F3
{
	float x, y, z;
};

__device__ __forceinline__ F3 f3(float a, float b, float c) { return F3{a, b, c}; }
__device__ __forceinline__ float dotf(const F3& a, const F3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float normf(const F3& a) { return sqrtf(dotf(a, a)); }

// Event with FP64 time and FP32 position / velocity (km, km/s) of one free segment.
struct EventF
{
	double t;
	F3 x, v;
};

// Propagator: FP64 accumulators, FP32 orbital-plane frame.
struct PropF
{
	double time, radius, phi, v_radial, time_step;
	float J;
	F3 ax, ay;
	int radial_mode;
};

// FP32 images of the tables the propagation reads every step.
struct DevSolarF
{
	const float* r;      // knots
	const float* gm;
	const float* gm_s;
	const float* vesc2;
	const float* vesc2_s;
};

__device__ __forceinline__ int knot_index_f(const DevSolar& S, const DevSolarF& F, float x)
{
	const int last = S.n - 2;
	if(x >= __ldg(F.r + last))
		return last;
	if(!(x >= 0.0f))
		return 0;
	int b = static_cast<int>(x * static_cast<float>(S.bucket_scale));
	b = b > S.nbuckets ? S.nbuckets : b;
	int i = __ldg(S.bucket + b);
	DMS_CHECK_INDEX(i, 0, last + 1, BOUNDS_KNOT);
	while(i > 0 && __ldg(F.r + i) > x) i--;
	while(i < last && __ldg(F.r + i + 1) <= x) i++;
	return i;
}

__device__ __forceinline__ float gm_f(const DevSolar& S, const DevSolarF& F, float r)
{
	r = r < 0.0f ? 0.0f : r;
	if(r > static_cast<float>(DMS_RSUN_KM))
		return static_cast<float>(DMS_GMSUN_KM3S2);
	const int i = knot_index_f(S, F, r);
	return __ldg(F.gm + i) + (r - __ldg(F.r + i)) * __ldg(F.gm_s + i);
}

// One RK45 stage's derivatives at radius r: dv_r/dt = J^2/r^3 - G M/r^2 (r clamped to >= 1 km)
// and dphi/dt = J/r^2, from one reciprocal.
__device__ __forceinline__ void stage_rates(const PropF& p, float r, float gm, float& dv, float& dp)
{
	const float inv = 1.0f / fmaxf(r, 1.0f);
	const float inv2 = inv * inv;
	dv = (p.J * p.J * inv - gm) * inv2;
	dp = (p.radial_mode || p.J == 0.0f || r <= 0.0f) ? 0.0f : p.J * inv2;
}

// Fehlberg weights in FP32 and the error weights (b5 - b4) in FP64
__constant__ float RKF_A_F[6][5] = {
	{0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
	{1.0f / 4.0f, 0.0f, 0.0f, 0.0f, 0.0f},
	{3.0f / 32.0f, 9.0f / 32.0f, 0.0f, 0.0f, 0.0f},
	{1932.0f / 2197.0f, -7200.0f / 2197.0f, 7296.0f / 2197.0f, 0.0f, 0.0f},
	{439.0f / 216.0f, -8.0f, 3680.0f / 513.0f, -845.0f / 4104.0f, 0.0f},
	{-8.0f / 27.0f, 2.0f, -3544.0f / 2565.0f, 1859.0f / 4104.0f, -11.0f / 40.0f}};
__constant__ float RKF_B4_F[6] = {25.0f / 216.0f, 0.0f, 1408.0f / 2565.0f, 2197.0f / 4104.0f, -1.0f / 5.0f, 0.0f};
__constant__ double RKF_E[6] = {16.0 / 135.0 - 25.0 / 216.0, 0.0, 6656.0 / 12825.0 - 1408.0 / 2565.0, 28561.0 / 56430.0 - 2197.0 / 4104.0,
                                -9.0 / 50.0 + 1.0 / 5.0, 2.0 / 55.0};

// One pass of the Runge_Kutta_45_Step retry loop (src/Simulation_Trajectory.cpp:1492-1600):
// FP32 stages, FP64 error norm and state update.  Unrolled: the six stages written out (a
// lane that runs alone takes 8 % less time per step); otherwise one loop over the stages
// (a shorter instruction stream while every lane is busy).  Both evaluate the same
// operations in the same order.
template <bool Unrolled>
__device__ __forceinline__ int rk45_attempt_f(const DevSolar& S, const DevSolarF& F, PropF& p, int inner)
{
	const float dt = static_cast<float>(p.time_step);
	const float r = static_cast<float>(p.radius), v = static_cast<float>(p.v_radial);
	// stages with accumulators for the later stages (see rk45_attempt); the 4th-order
	// increments in FP32, the (b5 - b4) error sums in FP64
	float R1 = r, R2 = r, R3 = r, R4 = r, R5 = r, V1 = v, V2 = v, V3 = v, V4 = v, V5 = v;
	float dr4 = 0.0f, dv4 = 0.0f, dp4 = 0.0f;
	double er = 0.0, ev = 0.0, ep = 0.0;
	auto stage = [&](int j) {
		const float ri = j == 0 ? r : j == 1 ? R1 : j == 2 ? R2 : j == 3 ? R3 : j == 4 ? R4 : R5;
		const float vi = j == 0 ? v : j == 1 ? V1 : j == 2 ? V2 : j == 3 ? V3 : j == 4 ? V4 : V5;
		float a, b;
		stage_rates(p, ri, gm_f(S, F, ri), a, b);
		const float kr = dt * vi, kv = dt * a, kp = dt * b;
		if(j < 1) { const float c = RKF_A_F[1][j]; R1 += c * kr; V1 += c * kv; }
		if(j < 2) { const float c = RKF_A_F[2][j]; R2 += c * kr; V2 += c * kv; }
		if(j < 3) { const float c = RKF_A_F[3][j]; R3 += c * kr; V3 += c * kv; }
		if(j < 4) { const float c = RKF_A_F[4][j]; R4 += c * kr; V4 += c * kv; }
		if(j < 5) { const float c = RKF_A_F[5][j]; R5 += c * kr; V5 += c * kv; }
		const float b4 = RKF_B4_F[j];
		dr4 += b4 * kr;
		dv4 += b4 * kv;
		dp4 += b4 * kp;
		const double c = RKF_E[j];
		er += c * static_cast<double>(kr);
		ev += c * static_cast<double>(kv);
		ep += c * static_cast<double>(kp);
	};
	if constexpr(Unrolled)
	{
#pragma unroll
		for(int j = 0; j < 6; j++) stage(j);
	}
	else
	{
#pragma unroll 1
		for(int j = 0; j < 6; j++) stage(j);
	}
	const double e0 = fabs(er), e1 = fabs(ev), e2 = fabs(ep);
	const bool finite_state = isfinite(dr4) && isfinite(dv4) && isfinite(dp4);
	// RK45_Next_Step_Size, src/Simulation_Trajectory.cpp:477-502
	double new_step;
	if(!isfinite(e0) || !isfinite(e1) || !isfinite(e2))
		new_step = DMS_RK45_MIN_STEP_FACTOR * p.time_step;
	else
	{
		float factor = static_cast<float>(DMS_RK45_MAX_STEP_FACTOR), c;
		if(e0 > 0.0)
		{
			c = 0.84f * sqrtf(sqrtf(static_cast<float>(DMS_RK45_TOL_R_KM) / static_cast<float>(e0)));
			if(isfinite(c) && c < factor) factor = c;
		}
		if(e1 > 0.0)
		{
			c = 0.84f * sqrtf(sqrtf(static_cast<float>(DMS_RK45_TOL_V_KMS) / static_cast<float>(e1)));
			if(isfinite(c) && c < factor) factor = c;
		}
		if(e2 > 0.0)
		{
			c = 0.84f * sqrtf(sqrtf(static_cast<float>(DMS_RK45_TOL_PHI) / static_cast<float>(e2)));
			if(isfinite(c) && c < factor) factor = c;
		}
		factor = factor < static_cast<float>(DMS_RK45_MIN_STEP_FACTOR) ? static_cast<float>(DMS_RK45_MIN_STEP_FACTOR) : factor;
		new_step = sanitized_step(static_cast<double>(factor) * p.time_step);
	}
	const bool within = isfinite(e0) && e0 <= DMS_RK45_TOL_R_KM && isfinite(e1) && e1 <= DMS_RK45_TOL_V_KMS && isfinite(e2) && e2 <= DMS_RK45_TOL_PHI;
	if(within)
	{
		p.time = p.time + p.time_step;
		const double r4 = p.radius + static_cast<double>(dr4);
		p.radius = r4 < 0.0 ? 0.0 : r4;
		p.v_radial = p.v_radial + static_cast<double>(dv4);
		p.phi = p.phi + static_cast<double>(dp4);
		p.time_step = new_step;
		return RK_ACCEPTED;
	}
	if(new_step < DMS_RK45_ABS_MIN_STEP_S || inner >= DMS_RK45_MAX_INNER_RETRIES)
	{
		p.time = p.time + DMS_RK45_ABS_MIN_STEP_S;
		if(finite_state)
		{
			const double r4 = p.radius + static_cast<double>(dr4);
			p.radius = r4 < 0.0 ? 0.0 : r4;
			p.v_radial = p.v_radial + static_cast<double>(dv4);
			p.phi = p.phi + static_cast<double>(dp4);
		}
		p.time_step = DMS_RK45_ABS_MIN_STEP_S;
		return RK_FORCED;
	}
	p.time_step = new_step;
	return RK_RETRY;
}

__device__ __forceinline__ double prop_radius_f(const PropF& p) { return p.radius < 0.0 ? 0.0 : p.radius; }

__device__ __forceinline__ double prop_speed_f(const PropF& p)
{
	const float r = static_cast<float>(p.radius < 0.0 ? 0.0 : p.radius);
	const float vr = static_cast<float>(p.v_radial);
	if(r == 0.0f || p.J == 0.0f)
		return fabs(p.v_radial);
	const float vt = p.J / r;
	return static_cast<double>(sqrtf(vr * vr + vt * vt));
}

// Capture_Energy_eV (src/Simulation_Trajectory.cpp:682-687) in FP32 for the per-step commit
// (free-flight drift and the uncaptured-bound check); the energy that decides capture and
// unbinding at a scattering stays FP64.
__device__ __forceinline__ double capture_energy_eV_f(const DevSolar& S, const DevSolarF& F, double m_dm, float r, float v)
{
	float vesc2;
	if(r > static_cast<float>(DMS_RSUN_KM))
		vesc2 = static_cast<float>(2.0 * DMS_GMSUN_KM3S2) / r;
	else
	{
		const float rr = r < 0.0f ? 0.0f : r;
		const int i = knot_index_f(S, F, rr);
		vesc2 = __ldg(F.vesc2 + i) + (rr - __ldg(F.r + i)) * __ldg(F.vesc2_s + i);
	}
	const float scale = static_cast<float>(0.5 * m_dm / (DMS_C_KMS * DMS_C_KMS) / 1.0e-9);
	return static_cast<double>(scale * (v * v - vesc2));
}

// Event_In_3D (src/Simulation_Trajectory.cpp:1715-1742) with the angle reduced in FP64 first
__device__ __forceinline__ EventF prop_event_f(const PropF& p)
{
	const double safe = (isfinite(p.radius) && p.radius > 0.0) ? p.radius : 0.0;
	EventF e;
	e.t = p.time;
	const float sr = static_cast<float>(safe), vr = static_cast<float>(p.v_radial);
	if(p.radial_mode || p.J == 0.0f || safe == 0.0)
	{
		e.x = f3(sr * p.ax.x, sr * p.ax.y, sr * p.ax.z);
		e.v = f3(vr * p.ax.x, vr * p.ax.y, vr * p.ax.z);
		return e;
	}
	const double turns = rint(p.phi * (1.0 / (2.0 * DMS_PI)));
	const float phi = static_cast<float>(p.phi - turns * (2.0 * DMS_PI));
	float sp, cp;
	sincosf(phi, &sp, &cp);
	const float vt = p.J / sr;
	const float vx = vr * cp - vt * sp;
	const float vy = vr * sp + vt * cp;
	e.x = f3(sr * (cp * p.ax.x + sp * p.ay.x), sr * (cp * p.ax.y + sp * p.ay.y), sr * (cp * p.ax.z + sp * p.ay.z));
	e.v = f3(vx * p.ax.x + vy * p.ay.x, vx * p.ax.y + vy * p.ay.y, vx * p.ax.z + vy * p.ay.z);
	return e;
}

// Free_Particle_Propagator constructor from an FP64 event (frame in FP32)
__device__ __forceinline__ void prop_init_f(PropF& q, const Event& e)
{
	Prop p;
	prop_init(p, e);
	q.time = p.time;
	q.radius = p.radius;
	q.phi = p.phi;
	q.v_radial = p.v_radial;
	q.time_step = p.time_step;
	q.J = static_cast<float>(p.J);
	q.ax = f3(static_cast<float>(p.ax.x), static_cast<float>(p.ax.y), static_cast<float>(p.ax.z));
	q.ay = f3(static_cast<float>(p.ay.x), static_cast<float>(p.ay.y), static_cast<float>(p.ay.z));
	q.radial_mode = p.radial_mode;
}

__device__ __forceinline__ Event to_event64(const EventF& e)
{
	Event o;
	o.t = e.t;
	o.x = mk(e.x.x, e.x.y, e.x.z);
	o.v = mk(e.v.x, e.v.y, e.v.z);
	return o;
}

// Total_DM_Scattering_Rate through the FP32 copy of the grid (src/Solar_Model.cpp:344-393);
// speeds above the grid fall back to the FP64 direct sum as in the reference.
__device__ __forceinline__ float rate_total_f(const DevSolar& S, const DevPoint* __restrict__ P, const float* __restrict__ grid, float r, float v)
{
	if(!isfinite(r) || !isfinite(v))
		return NAN;
	r = r < 0.0f ? 0.0f : r;
	v = v < 0.0f ? 0.0f : v;
	if(!(v <= static_cast<float>(__ldg(&P->grid_vmax))))
		return static_cast<float>(rate_computed(S, P, r, v, nullptr, nullptr));
	if(r > static_cast<float>(DMS_RSUN_KM))
		return 0.0f;
	const float rc = r * static_cast<float>(__ldg(&P->grid_inv_r));
	const float vc = v * static_cast<float>(__ldg(&P->grid_inv_v));
	const unsigned int N = static_cast<unsigned int>(__ldg(&P->grid_n));
	unsigned int ri = static_cast<unsigned int>(rc);
	unsigned int vi = static_cast<unsigned int>(vc);
	ri = ri > N - 2 ? N - 2 : ri;
	vi = vi > N - 2 ? N - 2 : vi;
	DMS_CHECK_INDEX(ri, 0u, N - 1, BOUNDS_GRID);
	DMS_CHECK_INDEX(vi, 0u, N - 1, BOUNDS_GRID);
	const float rf = rc - ri, vf = vc - vi;
	const size_t lower = static_cast<size_t>(ri) * N + vi;
	const float g00 = __ldg(grid + lower), g01 = __ldg(grid + lower + 1);
	const float g10 = __ldg(grid + lower + N), g11 = __ldg(grid + lower + N + 1);
	const float lo = g00 + vf * (g01 - g00);
	const float hi = g10 + vf * (g11 - g10);
	const float rate = lo + rf * (hi - lo);
	return isfinite(rate) ? (rate > 0.0f ? rate : 0.0f) : NAN;
}

__device__ __forceinline__ float rate_at_fraction_f(const DevSolar& S, const DevPoint* __restrict__ P, const float* __restrict__ grid,
                                                    const EventF& a, const EventF& b, float f)
{
	f = f < 0.0f ? 0.0f : (f > 1.0f ? 1.0f : f);
	const float x = a.x.x + f * (b.x.x - a.x.x), vx = a.v.x + f * (b.v.x - a.v.x);
	const float y = a.x.y + f * (b.x.y - a.x.y), vy = a.v.y + f * (b.v.y - a.v.y);
	const float z = a.x.z + f * (b.x.z - a.x.z), vz = a.v.z + f * (b.v.z - a.v.z);
	const float r = sqrtf(fmaxf(x * x + y * y + z * z, 0.0f));
	if(r >= static_cast<float>(DMS_RSUN_KM))
		return 0.0f;
	return rate_total_f(S, P, grid, r, sqrtf(fmaxf(vx * vx + vy * vy + vz * vz, 0.0f)));
}

__device__ __forceinline__ float radius_at_fraction_f(const EventF& a, const EventF& b, float f)
{
	f = f < 0.0f ? 0.0f : (f > 1.0f ? 1.0f : f);
	const float x = a.x.x + f * (b.x.x - a.x.x), y = a.x.y + f * (b.x.y - a.x.y), z = a.x.z + f * (b.x.z - a.x.z);
	return sqrtf(fmaxf(x * x + y * y + z * z, 0.0f));
}

// Solar_Interior_Fraction_Interval (src/Simulation_Trajectory.cpp:231-325); the quadratic's
// constant term |x|^2 - R^2 is formed in FP64 to avoid cancellation near the surface
__device__ __forceinline__ bool interior_interval_f(const EventF& a, const EventF& b, double ra, double rb, float& start, float& end)
{
	const bool a_in = ra < DMS_RSUN_KM, b_in = rb < DMS_RSUN_KM;
	if(a_in && b_in)
	{
		start = 0.0f;
		end = 1.0f;
		return true;
	}
	const float dx = b.x.x - a.x.x, dy = b.x.y - a.x.y, dz = b.x.z - a.x.z;
	const double qa = static_cast<double>(dx * dx + dy * dy + dz * dz);
	const double qb = 2.0 * static_cast<double>(a.x.x * dx + a.x.y * dy + a.x.z * dz);
	const double ax = a.x.x, ay = a.x.y, az = a.x.z;
	const double qc = (ax * ax + ay * ay + az * az) - DMS_RSUN_KM * DMS_RSUN_KM;
	bool has = false;
	float c1 = 0.0f, c2 = 0.0f;
	if(qa > 0.0)
	{
		const double disc = qb * qb - 4.0 * qa * qc;
		if(isfinite(disc) && disc >= 0.0)
		{
			const double sq = sqrt(disc);
			double f1 = (-qb - sq) / (2.0 * qa), f2 = (-qb + sq) / (2.0 * qa);
			if(f1 > f2)
			{
				const double t = f1;
				f1 = f2;
				f2 = t;
			}
			c1 = static_cast<float>(f1);
			c2 = static_cast<float>(f2);
			has = true;
		}
	}
	auto in_unit_f = [](float f) { return f >= -1.0e-12f && f <= 1.0f + 1.0e-6f; };
	auto clampf = [](float f) { return f < 0.0f ? 0.0f : (f > 1.0f ? 1.0f : f); };
	auto bisect = [&]() {
		float lower = 0.0f, upper = 1.0f;
		float r_lower = radius_at_fraction_f(a, b, lower) - static_cast<float>(DMS_RSUN_KM);
		for(int it = 0; it < 30; it++)
		{
			const float mid = 0.5f * (lower + upper);
			const float r_mid = radius_at_fraction_f(a, b, mid) - static_cast<float>(DMS_RSUN_KM);
			if((r_lower <= 0.0f && r_mid <= 0.0f) || (r_lower >= 0.0f && r_mid >= 0.0f))
			{
				lower = mid;
				r_lower = r_mid;
			}
			else
				upper = mid;
		}
		return clampf(0.5f * (lower + upper));
	};
	if(!a_in && b_in)
	{
		start = (has && in_unit_f(c1)) ? clampf(c1) : (has && in_unit_f(c2)) ? clampf(c2) : bisect();
		end = 1.0f;
		return end > start;
	}
	if(a_in && !b_in)
	{
		start = 0.0f;
		end = (has && in_unit_f(c2)) ? clampf(c2) : (has && in_unit_f(c1)) ? clampf(c1) : bisect();
		return end > start;
	}
	if(has && in_unit_f(c1) && in_unit_f(c2))
	{
		start = clampf(c1);
		end = clampf(c2);
		return end > start;
	}
	return false;
}

__device__ __forceinline__ EventF interpolate_event_f(const EventF& a, const EventF& b, float f)
{
	f = f < 0.0f ? 0.0f : (f > 1.0f ? 1.0f : f);
	EventF e;
	e.x = f3(a.x.x + f * (b.x.x - a.x.x), a.x.y + f * (b.x.y - a.x.y), a.x.z + f * (b.x.z - a.x.z));
	e.v = f3(a.v.x + f * (b.v.x - a.v.x), a.v.y + f * (b.v.y - a.v.y), a.v.z + f * (b.v.z - a.v.z));
	e.t = a.t + static_cast<double>(f) * (b.t - a.t);
	return e;
}

// ---- scattering in FP32 (the energy that decides capture stays FP64 in the caller) ----------

// Thermal_Averaged_Relative_Speed (src/Solar_Model.cpp:493-521) in FP32
__device__ __forceinline__ float thermal_relative_speed_f(float T, float m, float v)
{
	const float sqrt_pi = 1.7724538509055159f;
	if(!isfinite(T) || T <= 0.0f || !isfinite(m) || m <= 0.0f || !isfinite(v) || v < 0.0f)
		return NAN;
	const float kappa = sqrtf(m / (2.0f * T)) / static_cast<float>(DMS_C_KMS);
	if(!isfinite(kappa) || kappa <= 0.0f)
		return NAN;
	if(v == 0.0f)
		return 2.0f / sqrt_pi / kappa;
	const float x = kappa * v;
	if(!isfinite(x))
		return v;
	const float x2 = x * x;
	if(x < 1.0e-4f)
		return 2.0f / sqrt_pi / kappa * (1.0f + x2 / 3.0f - x2 * x2 / 30.0f + x2 * x2 * x2 / 210.0f);
	if(x > 26.0f)
		return v * (1.0f + 0.5f / x2);
	return v * ((1.0f + 2.0f * x2) * erff(x) / (2.0f * x2) + expf(-x2) / (sqrt_pi * x));
}

// One channel of Total_DM_Scattering_Rate_Computed (src/Solar_Model.cpp:263-303): density
// times cross section in FP64 (the factors alone exceed the FP32 range), the thermal average
// in FP32.  k == DMS_NUM_TARGETS is the electron channel.
__device__ __forceinline__ double channel_rate_f(const DevSolar& S, const DevPoint* __restrict__ P, int i, double dr, double T, double v, int k)
{
	double n_sigma;
	float m;
	if(k == DMS_NUM_TARGETS)
	{
		n_sigma = (__ldg(S.ne + i) + dr * __ldg(S.ne_s + i)) * channel_sigma(P, k, v);
		m = static_cast<float>(DMS_MELECTRON_GEV);
	}
	else
	{
		const size_t o = static_cast<size_t>(i) * DMS_NUM_TARGETS + k;
		n_sigma = (__ldg(S.nt + o) + dr * __ldg(S.nt_s + o)) * channel_sigma(P, k, v);
		m = static_cast<float>(__ldg(S.target_mass + k));
	}
	return n_sigma * static_cast<double>(thermal_relative_speed_f(static_cast<float>(T), m, static_cast<float>(v)));
}

// Unit_Vector_At_Angle_From_Axis (src/Simulation_Trajectory.cpp:109-128) in FP32
__device__ __forceinline__ bool unit_vector_at_angle_f(float cos_theta, float phi, const F3& axis, F3& out)
{
	if(!isfinite(cos_theta) || cos_theta < -1.0f - 1.0e-6f || cos_theta > 1.0f + 1.0e-6f || !isfinite(phi))
		return false;
	const float n = normf(axis);
	if(!isfinite(n) || n <= 0.0f)
		return false;
	const F3 e3 = f3(axis.x / n, axis.y / n, axis.z / n);
	const F3 ref = (fabsf(e3.z) < 0.9f) ? f3(0.0f, 0.0f, 1.0f) : f3(1.0f, 0.0f, 0.0f);
	F3 e1 = f3(ref.y * e3.z - ref.z * e3.y, ref.z * e3.x - ref.x * e3.z, ref.x * e3.y - ref.y * e3.x);
	const float n1 = normf(e1);
	e1 = f3(e1.x / n1, e1.y / n1, e1.z / n1);
	const F3 e2 = f3(e3.y * e1.z - e3.z * e1.y, e3.z * e1.x - e3.x * e1.z, e3.x * e1.y - e3.y * e1.x);
	cos_theta = fminf(fmaxf(cos_theta, -1.0f), 1.0f);
	const float st = sqrtf(fmaxf(1.0f - cos_theta * cos_theta, 0.0f));
	float sp, cp;
	sincosf(phi, &sp, &cp);
	out = f3(cos_theta * e3.x + st * cp * e1.x + st * sp * e2.x, cos_theta * e3.y + st * cp * e1.y + st * sp * e2.y,
	         cos_theta * e3.z + st * cp * e1.z + st * sp * e2.z);
	return true;
}

// Scatter once the target is known, in FP32: Sample_Target_Velocity (free-gas rejection),
// the isotropic angle and New_DM_Velocity, src/Simulation_Trajectory.cpp:1160-1269.  Same draw
// sequence as the FP64 form.  Returns false where the reference throws.
static __device__ __noinline__ bool scatter_with_target_f(const DevSolar& S, const DevPoint* __restrict__ P, Draws& D, Event& e, int target)
{
	const double r = ev_radius(e);
	const float m_target = target < 0 ? static_cast<float>(DMS_MELECTRON_GEV) : static_cast<float>(__ldg(S.target_mass + target));
	const float T = static_cast<float>(solar_temperature(S, r));
	if(!isfinite(T) || T <= 0.0f || !isfinite(m_target) || m_target <= 0.0f)
		return false;
	const float kappa = sqrtf(m_target / 2.0f / T) / static_cast<float>(DMS_C_KMS);
	const F3 vd = f3(static_cast<float>(e.v.x), static_cast<float>(e.v.y), static_cast<float>(e.v.z));
	const float vdm = normf(vd);
	if(!isfinite(kappa) || kappa <= 0.0f || !isfinite(vdm) || vdm <= 0.0f)
		return false;
	const float y = kappa * vdm;
	const float sqrt_pi = 1.7724538509055159f;
	float x = y, mu = 1.0f;
	unsigned long attempts = 0;
	for(;;)
	{
		const float raw = x * x + y * y - 2.0f * x * y * mu;
		const float den = x + y;
		if(!isfinite(x) || x < 0.0f || !isfinite(mu) || !isfinite(raw) || !isfinite(den) || den <= 0.0f)
			return false;
		const float ratio = sqrtf(fmaxf(raw, 0.0f)) / den;
		const float accept = ratio < 1.0f ? ratio : 1.0f;
		if(!(static_cast<double>(accept) < D.uniform(0.0, 1.0)))
			break;
		attempts++;
		if(attempts > DMS_TARGET_VELOCITY_MAX_REJECTIONS)
			return false;
		mu = static_cast<float>(D.uniform(-1.0, 1.0));
		const double xi1 = D.uniform(0.0, 1.0);
		if(xi1 < static_cast<double>(2.0f / (sqrt_pi * y + 2.0f)))
		{
			const float xi2 = static_cast<float>(D.positive_unit());
			const float xi3 = static_cast<float>(D.positive_unit());
			x = sqrtf(-logf(xi2) - logf(xi3));
		}
		else
		{
			const float xi2 = static_cast<float>(D.positive_unit());
			const float xi3 = static_cast<float>(D.uniform(0.0, 1.0));
			const float xi4 = static_cast<float>(D.positive_unit());
			const float c = cosf(1.5707963267948966f * xi3);
			x = sqrtf(-logf(xi2) - (c * c) * logf(xi4));
		}
	}
	const float vT = x / kappa;
	const float phi_t = static_cast<float>(D.uniform(0.0, 2.0 * DMS_PI));
	F3 unit_t;
	if(!unit_vector_at_angle_f(mu, phi_t, vd, unit_t))
		return false;
	const F3 vel_t = f3(vT * unit_t.x, vT * unit_t.y, vT * unit_t.z);
	const float cos_alpha = static_cast<float>(sample_cos_alpha(P, D, target, static_cast<double>(vdm)));
	const float md = static_cast<float>(__ldg(&P->m_dm));
	if(!isfinite(normf(vel_t)) || !isfinite(md) || md <= 0.0f)
		return false;
	const float phi_n = static_cast<float>(D.uniform(0.0, 2.0 * DMS_PI));
	F3 n;
	if(!unit_vector_at_angle_f(fminf(fmaxf(cos_alpha, -1.0f), 1.0f), phi_n, vd, n))
		return false;
	const F3 rel = f3(vel_t.x - vd.x, vel_t.y - vd.y, vel_t.z - vd.z);
	const float inv_m = 1.0f / (m_target + md);
	const float sc = m_target * normf(rel) * inv_m;
	const F3 out = f3(sc * n.x + (md * vd.x + m_target * vel_t.x) * inv_m, sc * n.y + (md * vd.y + m_target * vel_t.y) * inv_m,
	                  sc * n.z + (md * vd.z + m_target * vel_t.z) * inv_m);
	if(!isfinite(normf(out)))
		return false;
	e.v = mk(out.x, out.y, out.z);
	return true;
}

}	// namespace mixed
}	// namespace dms
