// Device-side physics of the trajectory engine: solar tables, scattering rates, the halo
// initial-condition sampler, Kepler maps, the RK45 propagator and the scatter kinematics.
// Each function restates the reference function cited beside it with the same operation
// order, so that the FP64 strict build (compiled without FMA contraction) reproduces the
// CPU oracle bit for bit.  Transcendentals that feed the trajectory state use the shared
// implementations of include/dms_math.h; exp/erf only enter rates and accept/reject tests.
#pragma once

#include <cstdint>

#include "../../include/dms.h"
#include "../../include/dms_constants.h"
#include "../../include/dms_math.h"
#include "../../include/dms_nuclear_data.h"
#include "../../include/dms_philox.h"
#include "dms_fastmath.cuh"

namespace dms
{

// ---------------------------------------------------------------------------------------------
// Checked build (-DDMS_CHECKED): every table, grid, histogram and work index is tested against
// its bounds before use; a failure sets a bit of this translation unit's status word and the
// index is clamped, so the kernel neither faults nor stops and the host reports the bits after
// the launch.  The bits: 1 solar-table knot, 2 rate-grid cell, 4 histogram bin, 8 flushed
// histogram row, 16 work range, 32 scattering target.  Without DMS_CHECKED the checks vanish.
enum : unsigned int
{
	BOUNDS_KNOT = 1u,
	BOUNDS_GRID = 2u,
	BOUNDS_BIN = 4u,
	BOUNDS_ROW = 8u,
	BOUNDS_RANGE = 16u,
	BOUNDS_TARGET = 32u,
};
#ifdef DMS_CHECKED
static __device__ unsigned int dms_bounds_status;
#define DMS_CHECK_INDEX(i, lo, hi, bit)                                  \
	do                                                                   \
	{                                                                    \
		if(!((i) >= (lo) && (i) < (hi)))                                 \
		{                                                                \
			atomicOr(&dms_bounds_status, (bit));                         \
			(i) = ((i) < (lo)) ? (lo) : (hi) - 1;                        \
		}                                                                \
	} while(0)
#else
#define DMS_CHECK_INDEX(i, lo, hi, bit) \
	do                                  \
	{                                   \
	} while(0)
#endif

// ---------------------------------------------------------------------------------------------
// Device images of the model
struct DevSolar
{
	int n;                 // knots
	int nbuckets;
	int bucket_single_step;  // 1: the knot interval of x is its bucket's base or the base + 1
	double bucket_scale;   // nbuckets / R_sun
	const double* r;
	const double* gm;
	const double* gm_s;
	const double* temp;
	const double* temp_s;
	const double* vesc2;
	const double* vesc2_s;
	const double* ne;
	const double* ne_s;
	const double* nt;      // node-major n x DMS_NUM_TARGETS
	const double* nt_s;
	const double* target_mass; // DMS_NUM_TARGETS isotope masses [GeV]
	const uint16_t* bucket;
};

struct DevPoint
{
	double m_dm;
	double sigma_e;
	double v0, vesc_halo, vobs;
	double vel_obs[3];
	double n_esc;
	double avg_speed, eta0;
	double grid_inv_r, grid_inv_v, grid_vmax;
	const double* grid;    // grid_n x grid_n, radius-major
	const float* grid_f;   // FP32 image of grid (mixed-precision kernel)
	int grid_n;
	int interaction;       // DMS_INTERACTION_*
	double ff_num, ff_m2;  // General form factor: (q_ref^2 + m^2)^2 / m^2, m^2 [GeV^2]
	double sigma_t[DMS_NUM_TARGETS];
	double q2c[DMS_NUM_TARGETS + 1];  // 4 mu_k^2 / c^2; [63] the electron
};

struct Vec3
{
	double x, y, z;
};

__device__ __forceinline__ Vec3 mk(double a, double b, double c) { return Vec3{a, b, c}; }
__device__ __forceinline__ double dot3(const Vec3& a, const Vec3& b)
{
	double s = 0.0;
	s += a.x * b.x;
	s += a.y * b.y;
	s += a.z * b.z;
	return s;
}
__device__ __forceinline__ double norm3(const Vec3& a) { return sqrt(dot3(a, a)); }
__device__ __forceinline__ Vec3 cross3(const Vec3& a, const Vec3& b)
{
	return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ Vec3 div3(const Vec3& a, double s) { return mk(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ Vec3 scale3(double s, const Vec3& a) { return mk(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ Vec3 add3(const Vec3& a, const Vec3& b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ Vec3 sub3(const Vec3& a, const Vec3& b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ Vec3 normalized3(const Vec3& a) { return div3(a, norm3(a)); }

struct Event
{
	double t;
	Vec3 x, v;
};

__device__ __forceinline__ double clamp_cos(double c) { return c < -1.0 ? -1.0 : (c > 1.0 ? 1.0 : c); }
__device__ __forceinline__ double clamp_unit(double c) { return c < 0.0 ? 0.0 : (c > 1.0 ? 1.0 : c); }

// ---------------------------------------------------------------------------------------------
// Tables: piecewise-linear, knot i = largest with r_i <= x clamped to [0, n-2]
__device__ __forceinline__ int knot_index(const DevSolar& S, double x)
{
	const int last = S.n - 2;
	if(S.bucket_single_step)
	{
		// one select, the same interval as the search below: x < 0 or NaN maps to bucket 0
		// (base 0, no step up), x beyond the last knot to a base of last - 1 or last
		const double xc = !(x >= 0.0) ? 0.0 : (x > DMS_RSUN_KM ? DMS_RSUN_KM : x);
		int b = static_cast<int>(xc * S.bucket_scale);
		b = b > S.nbuckets ? S.nbuckets : b;
		int i = __ldg(S.bucket + b);
		DMS_CHECK_INDEX(i, 0, last + 1, BOUNDS_KNOT);
		return i + ((i < last) & (__ldg(S.r + i + 1) <= x));
	}
	if(x >= __ldg(S.r + last))
		return last;
	if(!(x >= 0.0))
		return 0;
	int b = static_cast<int>(x * S.bucket_scale);
	b = b > S.nbuckets ? S.nbuckets : b;
	int i = __ldg(S.bucket + b);
	DMS_CHECK_INDEX(i, 0, last + 1, BOUNDS_KNOT);
	while(i > 0 && __ldg(S.r + i) > x) i--;
	while(i < last && __ldg(S.r + i + 1) <= x) i++;
	return i;
}

__device__ __forceinline__ double table_eval(const DevSolar& S, const double* y, const double* s, double x)
{
	const int i = knot_index(S, x);
	return __ldg(y + i) + (x - __ldg(S.r + i)) * __ldg(s + i);
}

// Solar_Model::Mass (as G*M), src/Solar_Model.cpp:168-179
__device__ __forceinline__ double solar_gm(const DevSolar& S, double r)
{
	if(S.bucket_single_step)
	{
		// without branches: both candidate intervals are loaded together with the bucket's
		// base, and the same interval and arithmetic as below are selected
		const double x = r < 0.0 ? 0.0 : r;
		const double xc = !(x >= 0.0) ? 0.0 : (x > DMS_RSUN_KM ? DMS_RSUN_KM : x);
		int b = static_cast<int>(xc * S.bucket_scale);
		b = b > S.nbuckets ? S.nbuckets : b;
		int i = __ldg(S.bucket + b);
		DMS_CHECK_INDEX(i, 0, S.n - 1, BOUNDS_KNOT);
		const double r0 = __ldg(S.r + i), r1 = __ldg(S.r + i + 1);
		const double y0 = __ldg(S.gm + i), y1 = __ldg(S.gm + i + 1);
		const double s0 = __ldg(S.gm_s + i), s1 = __ldg(S.gm_s + i + 1);
		const bool up = (i < S.n - 2) & (r1 <= x);
		const double v = up ? y1 + (x - r1) * s1 : y0 + (x - r0) * s0;
		return !isfinite(r) ? NAN : (r > DMS_RSUN_KM ? DMS_GMSUN_KM3S2 : v);
	}
	if(!isfinite(r))
		return NAN;
	if(r < 0.0)
		r = 0.0;
	if(r > DMS_RSUN_KM)
		return DMS_GMSUN_KM3S2;
	return table_eval(S, S.gm, S.gm_s, r);
}

// Solar_Model::Temperature [GeV], src/Solar_Model.cpp:194-202
__device__ __forceinline__ double solar_temperature(const DevSolar& S, double r)
{
	if(!isfinite(r))
		return NAN;
	if(r < 0.0)
		r = 0.0;
	return table_eval(S, S.temp, S.temp_s, r);
}

// Solar_Model::Local_Escape_Speed, src/Solar_Model.cpp:204-218
__device__ __forceinline__ double solar_vesc(const DevSolar& S, double r)
{
	if(!isfinite(r))
		return NAN;
	if(r < 0.0)
		r = 0.0;
	if(r > DMS_RSUN_KM)
		return sqrt(2 * DMS_GMSUN_KM3S2 / r);
	return sqrt(table_eval(S, S.vesc2, S.vesc2_s, r));
}

// Thermal_Averaged_Relative_Speed, src/Solar_Model.cpp:493-521 (T, m in GeV; v in km/s)
__device__ __forceinline__ double thermal_relative_speed(double temperature, double mass_target, double v)
{
	const double sqrt_pi = sqrt(DMS_PI);
	if(!isfinite(temperature) || temperature <= 0.0 || !isfinite(mass_target) || mass_target <= 0.0 || !isfinite(v) || v < 0.0)
		return NAN;
	const double kappa = sqrt(mass_target / (2.0 * temperature)) / DMS_C_KMS;
	if(!isfinite(kappa) || kappa <= 0.0)
		return NAN;
	if(v == 0.0)
		return 2.0 / sqrt_pi / kappa;
	const double x = kappa * v;
	if(!isfinite(x))
		return v;
	if(x < 1.0e-4)
	{
		const double x2 = x * x;
		return 2.0 / sqrt_pi / kappa * (1.0 + x2 / 3.0 - x2 * x2 / 30.0 + x2 * x2 * x2 / 210.0);
	}
	if(x > 26.0)
		return v * (1.0 + 0.5 / (x * x));
	const double x2 = x * x;
	return v * ((1.0 + 2.0 * x2) * erf(x) / (2.0 * x2) + exp(-x2) / (sqrt_pi * x));
}

// Sigma_Total_Nucleus / Sigma_Total_Electron of channel k (k = 63: the electron) at DM speed v:
// the contact cross section, times (q_ref^2 + m^2)^2 / (m^2 (m^2 + q_max^2)) for the dark
// photon's General form factor (src/Dark_Photon.cpp:167-229), q_max^2 = 4 mu_k^2 v^2 / c^2.
__device__ __forceinline__ double channel_sigma(const DevPoint* __restrict__ P, int k, double v)
{
	const double sigma = (k == DMS_NUM_TARGETS) ? __ldg(&P->sigma_e) : __ldg(&P->sigma_t[k]);
	if(__ldg(&P->interaction) != DMS_INTERACTION_DARK_PHOTON_GENERAL)
		return sigma;
	const double q2 = __ldg(&P->q2c[k]) * (v * v);
	return sigma * (__ldg(&P->ff_num) / (__ldg(&P->ff_m2) + q2));
}

// Total_DM_Scattering_Rate_Computed and its channels, src/Solar_Model.cpp:263-342; the
// per-target rates are written to rates[] when non-null (Sample_Target)
static __device__ __noinline__ double rate_computed(const DevSolar& S, const DevPoint* __restrict__ P, double r, double v, double* rates, double* rate_e)
{
	if(!isfinite(r) || !isfinite(v))
		return NAN;
	if(r < 0.0)
		r = 0.0;
	if(v < 0.0)
		v = 0.0;
	if(r > DMS_RSUN_KM)
	{
		if(rates)
			for(int k = 0; k < DMS_NUM_TARGETS; k++) rates[k] = 0.0;
		if(rate_e)
			*rate_e = 0.0;
		return 0.0;
	}
	const int i = knot_index(S, r);
	const double dr = r - __ldg(S.r + i);
	const double T = __ldg(S.temp + i) + dr * __ldg(S.temp_s + i);
	const double ne = __ldg(S.ne + i) + dr * __ldg(S.ne_s + i);
	double total = ne * channel_sigma(P, DMS_NUM_TARGETS, v) * thermal_relative_speed(T, DMS_MELECTRON_GEV, v);
	if(rate_e)
		*rate_e = total;
	const double* nt = S.nt + static_cast<size_t>(i) * DMS_NUM_TARGETS;
	const double* ns = S.nt_s + static_cast<size_t>(i) * DMS_NUM_TARGETS;
	for(int k = 0; k < DMS_NUM_TARGETS; k++)
	{
		const double n = __ldg(nt + k) + dr * __ldg(ns + k);
		const double m = __ldg(S.target_mass + k);
		const double rk = n * channel_sigma(P, k, v) * thermal_relative_speed(T, m, v);
		if(rates)
			rates[k] = rk;
		total += rk;
	}
	return total;
}

// Total_DM_Scattering_Rate (interpolated grid), src/Solar_Model.cpp:305-322, 344-393
__device__ __forceinline__ double rate_total(const DevSolar& S, const DevPoint* __restrict__ P, double r, double v)
{
	if(!isfinite(r) || !isfinite(v))
		return NAN;
	if(r < 0.0)
		r = 0.0;
	if(v < 0.0)
		v = 0.0;
	const double vmax = __ldg(&P->grid_vmax);
	if(!(v <= vmax))
		return rate_computed(S, P, r, v, nullptr, nullptr);
	if(r > DMS_RSUN_KM)
		return 0.0;
	const double rc = r * __ldg(&P->grid_inv_r);
	const double vc = v * __ldg(&P->grid_inv_v);
	const unsigned int N = static_cast<unsigned int>(__ldg(&P->grid_n));
	unsigned int ri = static_cast<unsigned int>(rc);
	unsigned int vi = static_cast<unsigned int>(vc);
	ri = ri > N - 2 ? N - 2 : ri;
	vi = vi > N - 2 ? N - 2 : vi;
	DMS_CHECK_INDEX(ri, 0u, N - 1, BOUNDS_GRID);
	DMS_CHECK_INDEX(vi, 0u, N - 1, BOUNDS_GRID);
	const double rf = rc - ri;
	const double vf = vc - vi;
	const double* g = reinterpret_cast<const double*>(__ldg(reinterpret_cast<const unsigned long long*>(&P->grid)));
	const size_t lower = static_cast<size_t>(ri) * N + vi;
	const size_t upper = lower + N;
	const double g00 = __ldg(g + lower), g01 = __ldg(g + lower + 1);
	const double g10 = __ldg(g + upper), g11 = __ldg(g + upper + 1);
	const double lower_rate = g00 + vf * (g01 - g00);
	const double upper_rate = g10 + vf * (g11 - g10);
	const double rate = lower_rate + rf * (upper_rate - lower_rate);
	return isfinite(rate) ? (rate > 0.0 ? rate : 0.0) : NAN;
}

// ---------------------------------------------------------------------------------------------
// Random draws: libphysica::Sample_Uniform semantics on the Philox stream
struct Draws
{
	uint32_t seed, point;
	uint64_t traj, index;
	__device__ __forceinline__ double uniform(double a, double b)
	{
		const double u = dms_draw_uniform(seed, point, traj, index++);
		return a + u * (b - a);
	}
	// Positive_Unit_Uniform, src/Simulation_Trajectory.cpp:103-107
	__device__ __forceinline__ double positive_unit()
	{
		const double u = uniform(0.0, 1.0);
		return u > 2.2250738585072014e-308 ? u : 2.2250738585072014e-308;
	}
};

// ---------------------------------------------------------------------------------------------
// Standard Halo Model and initial conditions, src/Simulation_Utilities.cpp:123-249
__device__ __forceinline__ double halo_pdf_speed(const DevPoint* __restrict__ P, double v)
{
	const double v0 = __ldg(&P->v0), vesc = __ldg(&P->vesc_halo), vobs = __ldg(&P->vobs);
	if(v < 0.0 || v > vesc + vobs)
		return 0.0;
	const double dm = v - vobs;
	const double dp = v + vobs;
	const double a = exp(-dm * dm / (v0 * v0));
	const double b = (dp <= vesc) ? exp(-dp * dp / (v0 * v0)) : exp(-vesc * vesc / (v0 * v0));
	return v / (__ldg(&P->n_esc) * sqrt(DMS_PI) * v0 * vobs) * (a - b);
}

__device__ __forceinline__ double halo_pdf_velocity(const DevPoint* __restrict__ P, const Vec3& vel)
{
	const double v0 = __ldg(&P->v0), vesc = __ldg(&P->vesc_halo);
	const Vec3 w = add3(vel, mk(__ldg(&P->vel_obs[0]), __ldg(&P->vel_obs[1]), __ldg(&P->vel_obs[2])));
	const double w2 = dot3(w, w);
	if(w2 > vesc * vesc)
		return 0.0;
	return exp(-w2 / (v0 * v0)) / (__ldg(&P->n_esc) * 5.5683279968317078453 * v0 * v0 * v0);
}

// libphysica::Spherical_Coordinates restated (stable frame about `axis`)
__device__ __forceinline__ Vec3 spherical_coordinates(double r, double theta, double phi, const Vec3& axis)
{
	const Vec3 e3 = div3(axis, norm3(axis));
	const Vec3 ref = (fabs(e3.z) < 0.9) ? mk(0.0, 0.0, 1.0) : mk(1.0, 0.0, 0.0);
	const Vec3 e1 = normalized3(cross3(ref, e3));
	const Vec3 e2 = normalized3(cross3(e3, e1));
	double st, ct, sp, cp;
	dms_sincos(theta, &st, &ct);
	dms_sincos(phi, &sp, &cp);
	return mk(r * (st * cp * e1.x + st * sp * e2.x + ct * e3.x), r * (st * cp * e1.y + st * sp * e2.y + ct * e3.y),
	          r * (st * cp * e1.z + st * sp * e2.z + ct * e3.z));
}

__device__ __forceinline__ double pdf_initial_speed(const DevSolar& S, const DevPoint* __restrict__ P, double v)
{
	if(v == 0.0)
		return 0.0;
	const double v_esc = solar_vesc(S, DMS_RSUN_KM);
	const double normalization = __ldg(&P->avg_speed) + v_esc * v_esc * __ldg(&P->eta0);
	const double f = halo_pdf_speed(P, v);
	return (f * v + (f / v) * v_esc * v_esc) / normalization;
}

__device__ __forceinline__ double pdf_cos_theta(const DevPoint* __restrict__ P, double cos_theta, double v)
{
	const double f = halo_pdf_speed(P, v);
	const double normalization = 2.0 * DMS_PI * v * v / f;
	const Vec3 vo = mk(__ldg(&P->vel_obs[0]), __ldg(&P->vel_obs[1]), __ldg(&P->vel_obs[2]));
	const Vec3 axis = (norm3(vo) > 0.0) ? vo : mk(0.0, 0.0, 1.0);
	const Vec3 vel = spherical_coordinates(v, dms_acos(cos_theta), 0.0, axis);
	return normalization * halo_pdf_velocity(P, vel);
}

// Initial_Conditions, src/Simulation_Utilities.cpp:176-249.  Returns false when a rejection
// loop exceeds `max_attempts` (the reference loops without bound).
static __device__ __noinline__ bool initial_conditions(const DevSolar& S, const DevPoint* __restrict__ P, Draws& D, Event& e, int max_attempts)
{
	const double y_max_speed = DMS_IC_SPEED_YMAX_NATURAL / DMS_C_KMS;
	const double v_max = __ldg(&P->vesc_halo) + __ldg(&P->vobs);
	double u = 0.0;
	bool ok = false;
	for(int a = 0; a < max_attempts; a++)
	{
		const double x = D.uniform(0.0, v_max);
		const double y = D.uniform(0.0, y_max_speed);
		if(y <= pdf_initial_speed(S, P, x))
		{
			u = x;
			ok = true;
			break;
		}
	}
	if(!ok)
		return false;
	const Vec3 vo = mk(__ldg(&P->vel_obs[0]), __ldg(&P->vel_obs[1]), __ldg(&P->vel_obs[2]));
	const double v_sun = norm3(vo);
	const double v_gal = v_max - v_sun;
	double cos_theta_max = (v_sun == 0.0) ? 1.0 : (v_gal * v_gal - v_sun * v_sun - u * u) / (2.0 * u * v_sun);
	if(cos_theta_max > 1.0)
		cos_theta_max = 1.0;
	const double y_max = pdf_cos_theta(P, -1.0, u);
	double cos_theta = 0.0;
	ok = false;
	for(int a = 0; a < max_attempts; a++)
	{
		const double x = D.uniform(-1.0, cos_theta_max);
		const double y = D.uniform(0.0, y_max);
		if(y <= pdf_cos_theta(P, x, u))
		{
			cos_theta = x;
			ok = true;
			break;
		}
	}
	if(!ok)
		return false;
	const double phi = D.uniform(0.0, 2.0 * DMS_PI);
	const Vec3 axis = (v_sun > 0.0) ? vo : mk(0.0, 0.0, 1.0);
	Vec3 velocity = spherical_coordinates(u, dms_acos(clamp_cos(cos_theta)), phi, axis);
	const double asymptotic_distance = DMS_IC_ASYMPTOTIC_DISTANCE_AU * DMS_AU_KM;
	const double vesc_asymptotic = solar_vesc(S, asymptotic_distance);
	const double v = sqrt(u * u + vesc_asymptotic * vesc_asymptotic);
	velocity = scale3(v, normalized3(velocity));
	const double v_esc = solar_vesc(S, DMS_RSUN_KM);
	const double b_max = sqrt(u * u + v_esc * v_esc) / v * DMS_RSUN_KM;
	const Vec3 e_z = scale3(-1.0, normalized3(velocity));
	const Vec3 ref = (fabs(e_z.z) < 0.9) ? mk(0.0, 0.0, 1.0) : mk(1.0, 0.0, 0.0);
	const Vec3 e_x = normalized3(cross3(ref, e_z));
	const Vec3 e_y = normalized3(cross3(e_z, e_x));
	const double phi_disk = D.uniform(0.0, 2.0 * DMS_PI);
	const double xi = D.uniform(0.0, 1.0);
	const double b = sqrt(xi) * b_max;
	double s, c;
	dms_sincos(phi_disk, &s, &c);
	e.t = 0.0;
	e.x = mk(asymptotic_distance * e_z.x + b * (c * e_x.x + s * e_y.x), asymptotic_distance * e_z.y + b * (c * e_x.y + s * e_y.y),
	         asymptotic_distance * e_z.z + b * (c * e_x.z + s * e_y.z));
	e.v = velocity;
	return true;
}

__device__ __forceinline__ bool finite_positive(double x) { return isfinite(x) && x > 0.0; }

// Hyperbolic_Kepler_Shift, src/Simulation_Utilities.cpp:252-321
static __device__ __noinline__ bool hyperbolic_kepler_shift(Event& e, double R_final)
{
	const double mu = DMS_GMSUN_KM3S2;
	const double R_initial = norm3(e.x);
	const double speed = norm3(e.v);
	if(R_final < DMS_RSUN_KM || R_initial < DMS_RSUN_KM)
		return false;
	if(!finite_positive(R_final) || !finite_positive(R_initial) || !finite_positive(speed))
		return false;
	if(fabs(R_final - R_initial) <= DMS_KEPLER_DOMAIN_TOLERANCE * (R_initial > R_final ? R_initial : R_final))
		return true;
	const double vr = dot3(e.x, e.v) / R_initial;
	if(!isfinite(vr) || vr == 0.0)
		return false;
	const double dir = (vr < 0.0) ? -1.0 : 1.0;
	if(dir < 0.0 && R_final > R_initial)
		return false;
	if(dir > 0.0 && R_final < R_initial)
		return false;
	const double energy = 0.5 * speed * speed - mu / R_initial;
	if(!finite_positive(energy))
		return false;
	const Vec3 r_hat = div3(e.x, R_initial);
	const Vec3 h_vec = cross3(e.x, e.v);
	const double h = norm3(h_vec);
	const double h_scale = R_initial * speed;
	if(!isfinite(h) || h <= DMS_KEPLER_DOMAIN_TOLERANCE * h_scale)
	{
		const double final_speed_sqr = 2.0 * (energy + mu / R_final);
		if(!finite_positive(final_speed_sqr))
			return false;
		e.x = scale3(R_final, r_hat);
		e.v = scale3(dir * sqrt(final_speed_sqr), r_hat);
		return true;
	}
	const double p = h * h / mu;
	const Vec3 ecc_vec = sub3(div3(cross3(e.v, h_vec), mu), r_hat);
	const double ecc = norm3(ecc_vec);
	if(!finite_positive(p) || !isfinite(ecc) || ecc <= 1.0)
		return false;
	const double cos_final = (p / R_final - 1.0) / ecc;
	if(!isfinite(cos_final) || cos_final > 1.0 + DMS_KEPLER_DOMAIN_TOLERANCE || cos_final < -1.0 - DMS_KEPLER_DOMAIN_TOLERANCE)
		return false;
	Vec3 ax = div3(ecc_vec, ecc);
	const Vec3 az = div3(h_vec, h);
	Vec3 ay = cross3(az, ax);
	const double ny = norm3(ay);
	if(!finite_positive(ny))
		return false;
	ay = div3(ay, ny);
	ax = normalized3(cross3(ay, az));
	const double theta = dir * dms_acos(clamp_cos(cos_final));
	double st, ct;
	dms_sincos(theta, &st, &ct);
	const double sq = sqrt(mu / p);
	e.x = mk(R_final * (ct * ax.x + st * ay.x), R_final * (ct * ax.y + st * ay.y), R_final * (ct * ax.z + st * ay.z));
	e.v = mk(sq * (-st * ax.x + (ecc + ct) * ay.x), sq * (-st * ax.y + (ecc + ct) * ay.y), sq * (-st * ax.z + (ecc + ct) * ay.z));
	return true;
}

// ---------------------------------------------------------------------------------------------
// Free_Particle_Propagator, src/Simulation_Trajectory.cpp:1403-1742
struct Prop
{
	double time, radius, phi, v_radial, J, time_step;
	Vec3 ax, ay;
	int radial_mode;
};

static __device__ __noinline__ void prop_init(Prop& p, const Event& e)
{
	p.time = e.t;
	p.radius = norm3(e.x);
	p.phi = 0.0;
	p.radial_mode = 0;
	p.time_step = DMS_RK45_DEFAULT_STEP_S;
	p.J = 0.0;
	const double speed = norm3(e.v);
	const double angular_scale = (p.radius * speed > 1.0) ? p.radius * speed : 1.0;
	const double angular_eps = 1.0e-12 * angular_scale;
	const Vec3 L = cross3(e.x, e.v);
	const double Ln = norm3(L);
	Vec3 ax;
	if(isfinite(p.radius) && p.radius > 1.0e-12)
	{
		ax = div3(e.x, p.radius);
		p.v_radial = dot3(e.x, e.v) / p.radius;
	}
	else if(isfinite(speed) && speed > 0.0)
	{
		ax = div3(e.v, speed);
		p.v_radial = speed;
		p.radius = 0.0;
		p.radial_mode = 1;
	}
	else
	{
		ax = mk(1.0, 0.0, 0.0);
		p.v_radial = 0.0;
		p.radius = 0.0;
		p.radial_mode = 1;
	}
	Vec3 ay = mk(0.0, 0.0, 0.0);
	if(!p.radial_mode && isfinite(Ln) && Ln > angular_eps)
	{
		const Vec3 az = div3(L, Ln);
		ay = cross3(az, ax);
		const double ny = norm3(ay);
		if(isfinite(ny) && ny > 0.0)
		{
			ay = div3(ay, ny);
			ax = normalized3(cross3(ay, az));
			p.J = Ln;
		}
		else
			p.radial_mode = 1;
	}
	else
		p.radial_mode = 1;
	if(p.radial_mode)
	{
		// Build_Stable_Orthonormal_Basis, src/Simulation_Trajectory.cpp:130-142
		const Vec3 e1 = div3(ax, norm3(ax));
		const Vec3 ref = (fabs(e1.z) < 0.9) ? mk(0.0, 0.0, 1.0) : mk(1.0, 0.0, 0.0);
		ax = e1;
		ay = normalized3(cross3(ref, e1));
		p.J = 0.0;
	}
	p.ax = ax;
	p.ay = ay;
}

__device__ __forceinline__ double dv_dt(double J, double r, double gm)
{
	if(r < 1.0)
		r = 1.0;
	return J * J / r / r / r - gm / r / r;
}

__device__ __forceinline__ double dphi_dt(const Prop& p, double r)
{
	if(p.radial_mode || p.J == 0.0 || r <= 0.0)
		return 0.0;
	return p.J / r / r;
}

__device__ __forceinline__ double sanitized_step(double step)
{
	if(!isfinite(step) || step <= 0.0)
		return DMS_RK45_DEFAULT_STEP_S;
	return step < DMS_RK45_ABS_MAX_STEP_S ? step : DMS_RK45_ABS_MAX_STEP_S;
}

// RK45_Next_Step_Size, src/Simulation_Trajectory.cpp:477-502
__device__ __forceinline__ double next_step_size(double current, double e0, double e1, double e2)
{
	if(!isfinite(e0) || !isfinite(e1) || !isfinite(e2))
		return DMS_RK45_MIN_STEP_FACTOR * current;
	double factor = DMS_RK45_MAX_STEP_FACTOR;
	double c;
	if(e0 > 0.0)
	{
		c = 0.84 * dms_pow_quarter(DMS_RK45_TOL_R_KM / e0);
		if(isfinite(c) && c < factor) factor = c;
	}
	if(e1 > 0.0)
	{
		c = 0.84 * dms_pow_quarter(DMS_RK45_TOL_V_KMS / e1);
		if(isfinite(c) && c < factor) factor = c;
	}
	if(e2 > 0.0)
	{
		c = 0.84 * dms_pow_quarter(DMS_RK45_TOL_PHI / e2);
		if(isfinite(c) && c < factor) factor = c;
	}
	if(factor > DMS_RK45_MAX_STEP_FACTOR) factor = DMS_RK45_MAX_STEP_FACTOR;
	if(factor < DMS_RK45_MIN_STEP_FACTOR) factor = DMS_RK45_MIN_STEP_FACTOR;
	return sanitized_step(factor * current);
}

// One pass of the while(!accepted) loop of Runge_Kutta_45_Step(Solar_Model&),
// src/Simulation_Trajectory.cpp:1492-1600, as its own unit so that lanes of a warp retry in
// lock-step.  `inner` is the pass number (1-based).  Returns RK_ACCEPTED, RK_RETRY (state
// unchanged, smaller time_step) or RK_FORCED (the minimum-step / retry-cap forced accept, for
// which the reference returns false).
enum RkResult : int
{
	RK_ACCEPTED = 0,
	RK_RETRY = 1,
	RK_FORCED = 2,
};

// Arithmetic policies of the RK45 attempt: IEEE division and square root as written, or the
// certified straight-line forms of dms_fastmath.cuh (bit-identical whenever `good` stays set;
// the caller repeats the attempt with IeeeMath otherwise).
struct IeeeMath
{
	struct Rcp
	{
		double b;
	};
	__device__ __forceinline__ Rcp rcp(double b) const { return Rcp{b}; }
	__device__ __forceinline__ double div(double a, const Rcp& d) const { return a / d.b; }
	__device__ __forceinline__ double div(double a, double b) const { return a / b; }
	__device__ __forceinline__ double root(double x) const { return sqrt(x); }
};

struct CertMath
{
	bool good = true;
	using Rcp = fast::Recip;
	__device__ __forceinline__ Rcp rcp(double b) const { return fast::recip(b); }
	__device__ __forceinline__ double div(double a, const Rcp& d) { return fast::div(a, d, good); }
	__device__ __forceinline__ double div(double a, double b) { return fast::div(a, b, good); }
	__device__ __forceinline__ double root(double x) { return fast::sqrt(x, good); }
};

// RK45_Next_Step_Size (src/Simulation_Trajectory.cpp:477-502) under an arithmetic policy;
// pow(c, 0.25) is sqrt(sqrt(c)) as in dms_pow_quarter.
template <class M>
__device__ __forceinline__ double next_step_size_t(M& m, double current, double e0, double e1, double e2)
{
	if(!isfinite(e0) || !isfinite(e1) || !isfinite(e2))
		return DMS_RK45_MIN_STEP_FACTOR * current;
	double factor = DMS_RK45_MAX_STEP_FACTOR;
	double c;
	if(e0 > 0.0)
	{
		c = 0.84 * m.root(m.root(m.div(DMS_RK45_TOL_R_KM, e0)));
		if(isfinite(c) && c < factor) factor = c;
	}
	if(e1 > 0.0)
	{
		c = 0.84 * m.root(m.root(m.div(DMS_RK45_TOL_V_KMS, e1)));
		if(isfinite(c) && c < factor) factor = c;
	}
	if(e2 > 0.0)
	{
		c = 0.84 * m.root(m.root(m.div(DMS_RK45_TOL_PHI, e2)));
		if(isfinite(c) && c < factor) factor = c;
	}
	if(factor > DMS_RK45_MAX_STEP_FACTOR) factor = DMS_RK45_MAX_STEP_FACTOR;
	if(factor < DMS_RK45_MIN_STEP_FACTOR) factor = DMS_RK45_MIN_STEP_FACTOR;
	return sanitized_step(factor * current);
}

// dv/dt and dphi/dt of one stage at radius r: J*J/r/r/r - gm/r/r with r clamped to >= 1 km, and
// J/r/r (0 in radial mode, for J = 0 or r <= 0), the reference's divisions in its order.  The
// quotients by the same r share one reciprocal under CertMath.
template <class M>
__device__ __forceinline__ void stage_rates(M& m, const Prop& p, double r, double gm, double& dv, double& dphi, bool want_phi)
{
	const double rc = r < 1.0 ? 1.0 : r;
	const auto R = m.rcp(rc);
	dv = m.div(m.div(m.div(p.J * p.J, R), R), R) - m.div(m.div(gm, R), R);
	dphi = 0.0;
	if(want_phi && !(p.radial_mode || p.J == 0.0 || r <= 0.0))
		dphi = r < 1.0 ? m.div(m.div(p.J, r), r) : m.div(m.div(p.J, R), R);
}

// The attempt with the six stages written out: a longer instruction stream (more
// instruction-cache pressure with many warps) but a shorter dependent chain for a lane that
// runs alone.
template <class M>
__device__ __forceinline__ int rk45_attempt_t(const DevSolar& S, Prop& p, int inner, M& m)
{
	{
		const double dt = p.time_step;
		double kr0, kr1, kr2, kr3, kr4, kr5, kv0, kv1, kv2, kv3, kv4, kv5, kp0, kp2, kp3, kp4, kp5, ri, a, b;
		kr0 = dt * p.v_radial;
		stage_rates(m, p, p.radius, solar_gm(S, p.radius), a, b, true);
		kv0 = dt * a;
		kp0 = dt * b;
		ri = p.radius + kr0 / 4.0;
		kr1 = dt * (p.v_radial + kv0 / 4.0);
		stage_rates(m, p, ri, solar_gm(S, ri), a, b, false);
		kv1 = dt * a;
		ri = p.radius + 3.0 / 32.0 * kr0 + 9.0 / 32.0 * kr1;
		kr2 = dt * (p.v_radial + 3.0 / 32.0 * kv0 + 9.0 / 32.0 * kv1);
		stage_rates(m, p, ri, solar_gm(S, ri), a, b, true);
		kv2 = dt * a;
		kp2 = dt * b;
		ri = p.radius + 1932.0 / 2197.0 * kr0 - 7200.0 / 2197.0 * kr1 + 7296.0 / 2197.0 * kr2;
		kr3 = dt * (p.v_radial + 1932.0 / 2197.0 * kv0 - 7200.0 / 2197.0 * kv1 + 7296.0 / 2197.0 * kv2);
		stage_rates(m, p, ri, solar_gm(S, ri), a, b, true);
		kv3 = dt * a;
		kp3 = dt * b;
		ri = p.radius + 439.0 / 216.0 * kr0 - 8.0 * kr1 + 3680.0 / 513.0 * kr2 - 845.0 / 4104.0 * kr3;
		kr4 = dt * (p.v_radial + 439.0 / 216.0 * kv0 - 8.0 * kv1 + 3680.0 / 513.0 * kv2 - 845.0 / 4104.0 * kv3);
		stage_rates(m, p, ri, solar_gm(S, ri), a, b, true);
		kv4 = dt * a;
		kp4 = dt * b;
		ri = p.radius - 8.0 / 27.0 * kr0 + 2.0 * kr1 - 3544.0 / 2565.0 * kr2 + 1859.0 / 4104.0 * kr3 - 11.0 / 40.0 * kr4;
		kr5 = dt * (p.v_radial - 8.0 / 27.0 * kv0 + 2.0 * kv1 - 3544.0 / 2565.0 * kv2 + 1859.0 / 4104.0 * kv3 - 11.0 / 40.0 * kv4);
		stage_rates(m, p, ri, solar_gm(S, ri), a, b, true);
		kv5 = dt * a;
		kp5 = dt * b;
		const double r4 = p.radius + 25.0 / 216.0 * kr0 + 1408.0 / 2565.0 * kr2 + 2197.0 / 4104.0 * kr3 - 1.0 / 5.0 * kr4;
		const double v4 = p.v_radial + 25.0 / 216.0 * kv0 + 1408.0 / 2565.0 * kv2 + 2197.0 / 4104.0 * kv3 - 1.0 / 5.0 * kv4;
		const double p4 = p.phi + 25.0 / 216.0 * kp0 + 1408.0 / 2565.0 * kp2 + 2197.0 / 4104.0 * kp3 - 1.0 / 5.0 * kp4;
		const double r5 = p.radius + 16.0 / 135.0 * kr0 + 6656.0 / 12825.0 * kr2 + 28561.0 / 56430.0 * kr3 - 9.0 / 50.0 * kr4 + 2.0 / 55.0 * kr5;
		const double v5 = p.v_radial + 16.0 / 135.0 * kv0 + 6656.0 / 12825.0 * kv2 + 28561.0 / 56430.0 * kv3 - 9.0 / 50.0 * kv4 + 2.0 / 55.0 * kv5;
		const double p5 = p.phi + 16.0 / 135.0 * kp0 + 6656.0 / 12825.0 * kp2 + 28561.0 / 56430.0 * kp3 - 9.0 / 50.0 * kp4 + 2.0 / 55.0 * kp5;
		const double e0 = fabs(r5 - r4), e1 = fabs(v5 - v4), e2 = fabs(p5 - p4);
		const double new_step = next_step_size_t(m, dt, e0, e1, e2);
		const bool within = isfinite(e0) && e0 <= DMS_RK45_TOL_R_KM && isfinite(e1) && e1 <= DMS_RK45_TOL_V_KMS && isfinite(e2) && e2 <= DMS_RK45_TOL_PHI;
		if(within)
		{
			p.time = p.time + dt;
			p.radius = r4 < 0.0 ? 0.0 : r4;
			p.v_radial = v4;
			p.phi = p4;
			p.time_step = new_step;
			return RK_ACCEPTED;
		}
		if(new_step < DMS_RK45_ABS_MIN_STEP_S || inner >= DMS_RK45_MAX_INNER_RETRIES)
		{
			const bool ok = isfinite(r4) && isfinite(v4) && isfinite(p4);
			p.time = p.time + DMS_RK45_ABS_MIN_STEP_S;
			if(ok)
			{
				p.radius = r4 < 0.0 ? 0.0 : r4;
				p.v_radial = v4;
				p.phi = p4;
			}
			p.time_step = DMS_RK45_ABS_MIN_STEP_S;
			return RK_FORCED;
		}
		p.time_step = new_step;
		return RK_RETRY;
	}
}

__device__ __forceinline__ int rk45_attempt_unrolled(const DevSolar& S, Prop& p, int inner)
{
	IeeeMath m;
	return rk45_attempt_t(S, p, inner, m);
}

// The IEEE attempt, out of line: the fallback of rk45_attempt_certified.
static __device__ __noinline__ int rk45_attempt_ieee(const DevSolar& S, Prop& p, int inner)
{
	IeeeMath m;
	return rk45_attempt_t(S, p, inner, m);
}

// Solar_Model::Mass as G*M for tables whose buckets hold at most one knot
// (S.bucket_single_step): both candidate intervals are loaded with the bucket's base and the
// interval of the search in knot_index is selected, so the lookup has no branch.  Same value
// as solar_gm.
__device__ __forceinline__ double solar_gm_select(const DevSolar& S, double r)
{
	const double x = r < 0.0 ? 0.0 : r;
	const double xc = !(x >= 0.0) ? 0.0 : (x > DMS_RSUN_KM ? DMS_RSUN_KM : x);
	int b = static_cast<int>(xc * S.bucket_scale);
	b = b > S.nbuckets ? S.nbuckets : b;
	int i = __ldg(S.bucket + b);
	DMS_CHECK_INDEX(i, 0, S.n - 1, BOUNDS_KNOT);
	const double r0 = __ldg(S.r + i), r1 = __ldg(S.r + i + 1);
	const double y0 = __ldg(S.gm + i), y1 = __ldg(S.gm + i + 1);
	const double s0 = __ldg(S.gm_s + i), s1 = __ldg(S.gm_s + i + 1);
	const bool up = (i < S.n - 2) & (r1 <= x);
	const double v = up ? y1 + (x - r1) * s1 : y0 + (x - r0) * s0;
	return !isfinite(r) ? NAN : (r > DMS_RSUN_KM ? DMS_GMSUN_KM3S2 : v);
}

// One stage's dv/dt = J*J/r/r/r - gm/r/r (r clamped to >= 1 km) and, when wanted,
// dphi/dt = J/r/r (0 in radial mode, for J = 0 or r <= 0), with the certified division and
// without branches: every quotient by r shares one reciprocal.  A stage with 0 < r < 1 km (where
// the reference divides J by the unclamped r) clears `good`, which hands the attempt to IEEE.
template <bool WANT_PHI>
__device__ __forceinline__ void cert_stage(const DevSolar& S, const Prop& p, double r, double& dv, double& dphi, bool& good)
{
	const double gm = solar_gm_select(S, r);
	const double rc = r < 1.0 ? 1.0 : r;
	const fast::Recip R = fast::recip(rc);
	const double jj = p.J * p.J;
	dv = fast::div(fast::div(fast::div(jj, R, good), R, good), R, good) - fast::div(fast::div(gm, R, good), R, good);
	dphi = 0.0;
	if(WANT_PHI)
	{
		const bool zero = (p.radial_mode != 0) | (p.J == 0.0) | (r <= 0.0);
		const double q = fast::div(fast::div(p.J, R, good), R, good);
		dphi = zero ? 0.0 : q;
		good &= zero | (r >= 1.0);
	}
}

// The factor of RK45_Next_Step_Size for one error component without branches: 0.84 (tol/e)^(1/4)
// when e > 0 and the result is finite, else +inf (no limit); e outside (0, inf) divides 1.
__device__ __forceinline__ double cert_step_factor(double tol, double e, bool& good)
{
	const bool use = (e > 0.0) & isfinite(e);
	const double c = 0.84 * fast::sqrt(fast::sqrt(fast::div(tol, use ? e : 1.0, good), good), good);
	return (use & isfinite(c)) ? c : INFINITY;
}

// The written-out attempt of rk45_attempt_t with the certified division and square root and
// no branch before its final accept / retry decision, so that the compiler can overlap the
// stages that do not depend on one another: the radius of stage j needs the slopes of stages
// up to j - 2 only, so stages 0 and 1, 2 and 3, 4 and 5 are independent pairs.  `good` is
// cleared when any certificate fails; p is then unchanged and the caller repeats the attempt
// with IEEE arithmetic.
__device__ __forceinline__ int rk45_attempt_cert(const DevSolar& S, Prop& p, int inner, bool& good)
{
	const double dt = p.time_step;
	double kr0, kr1, kr2, kr3, kr4, kr5, kv0, kv1, kv2, kv3, kv4, kv5, kp0, kp1, kp2, kp3, kp4, kp5, ri, a;
	kr0 = dt * p.v_radial;
	cert_stage<true>(S, p, p.radius, a, kp0, good);
	kv0 = dt * a;
	kp0 = dt * kp0;
	ri = p.radius + kr0 / 4.0;
	kr1 = dt * (p.v_radial + kv0 / 4.0);
	cert_stage<false>(S, p, ri, a, kp1, good);
	kv1 = dt * a;
	ri = p.radius + 3.0 / 32.0 * kr0 + 9.0 / 32.0 * kr1;
	kr2 = dt * (p.v_radial + 3.0 / 32.0 * kv0 + 9.0 / 32.0 * kv1);
	cert_stage<true>(S, p, ri, a, kp2, good);
	kv2 = dt * a;
	kp2 = dt * kp2;
	ri = p.radius + 1932.0 / 2197.0 * kr0 - 7200.0 / 2197.0 * kr1 + 7296.0 / 2197.0 * kr2;
	kr3 = dt * (p.v_radial + 1932.0 / 2197.0 * kv0 - 7200.0 / 2197.0 * kv1 + 7296.0 / 2197.0 * kv2);
	cert_stage<true>(S, p, ri, a, kp3, good);
	kv3 = dt * a;
	kp3 = dt * kp3;
	ri = p.radius + 439.0 / 216.0 * kr0 - 8.0 * kr1 + 3680.0 / 513.0 * kr2 - 845.0 / 4104.0 * kr3;
	kr4 = dt * (p.v_radial + 439.0 / 216.0 * kv0 - 8.0 * kv1 + 3680.0 / 513.0 * kv2 - 845.0 / 4104.0 * kv3);
	cert_stage<true>(S, p, ri, a, kp4, good);
	kv4 = dt * a;
	kp4 = dt * kp4;
	ri = p.radius - 8.0 / 27.0 * kr0 + 2.0 * kr1 - 3544.0 / 2565.0 * kr2 + 1859.0 / 4104.0 * kr3 - 11.0 / 40.0 * kr4;
	kr5 = dt * (p.v_radial - 8.0 / 27.0 * kv0 + 2.0 * kv1 - 3544.0 / 2565.0 * kv2 + 1859.0 / 4104.0 * kv3 - 11.0 / 40.0 * kv4);
	cert_stage<true>(S, p, ri, a, kp5, good);
	kv5 = dt * a;
	kp5 = dt * kp5;
	const double r4 = p.radius + 25.0 / 216.0 * kr0 + 1408.0 / 2565.0 * kr2 + 2197.0 / 4104.0 * kr3 - 1.0 / 5.0 * kr4;
	const double v4 = p.v_radial + 25.0 / 216.0 * kv0 + 1408.0 / 2565.0 * kv2 + 2197.0 / 4104.0 * kv3 - 1.0 / 5.0 * kv4;
	const double p4 = p.phi + 25.0 / 216.0 * kp0 + 1408.0 / 2565.0 * kp2 + 2197.0 / 4104.0 * kp3 - 1.0 / 5.0 * kp4;
	const double r5 = p.radius + 16.0 / 135.0 * kr0 + 6656.0 / 12825.0 * kr2 + 28561.0 / 56430.0 * kr3 - 9.0 / 50.0 * kr4 + 2.0 / 55.0 * kr5;
	const double v5 = p.v_radial + 16.0 / 135.0 * kv0 + 6656.0 / 12825.0 * kv2 + 28561.0 / 56430.0 * kv3 - 9.0 / 50.0 * kv4 + 2.0 / 55.0 * kv5;
	const double p5 = p.phi + 16.0 / 135.0 * kp0 + 6656.0 / 12825.0 * kp2 + 28561.0 / 56430.0 * kp3 - 9.0 / 50.0 * kp4 + 2.0 / 55.0 * kp5;
	const double e0 = fabs(r5 - r4), e1 = fabs(v5 - v4), e2 = fabs(p5 - p4);
	// RK45_Next_Step_Size (src/Simulation_Trajectory.cpp:477-502) as selects: the factor is
	// limited by each component in turn, clamped to [0.1, 4], and the step sanitised; non-finite
	// errors give 0.1 x the current step
	double factor = DMS_RK45_MAX_STEP_FACTOR;
	const double c0 = cert_step_factor(DMS_RK45_TOL_R_KM, e0, good);
	factor = c0 < factor ? c0 : factor;
	const double c1 = cert_step_factor(DMS_RK45_TOL_V_KMS, e1, good);
	factor = c1 < factor ? c1 : factor;
	const double c2 = cert_step_factor(DMS_RK45_TOL_PHI, e2, good);
	factor = c2 < factor ? c2 : factor;
	factor = factor > DMS_RK45_MAX_STEP_FACTOR ? DMS_RK45_MAX_STEP_FACTOR : factor;
	factor = factor < DMS_RK45_MIN_STEP_FACTOR ? DMS_RK45_MIN_STEP_FACTOR : factor;
	const double grown = factor * dt;
	const double sane = (!isfinite(grown) | (grown <= 0.0)) ? DMS_RK45_DEFAULT_STEP_S
	                    : (grown < DMS_RK45_ABS_MAX_STEP_S ? grown : DMS_RK45_ABS_MAX_STEP_S);
	const bool finite_err = isfinite(e0) & isfinite(e1) & isfinite(e2);
	const double new_step = finite_err ? sane : DMS_RK45_MIN_STEP_FACTOR * dt;
	const bool within = finite_err & (e0 <= DMS_RK45_TOL_R_KM) & (e1 <= DMS_RK45_TOL_V_KMS) & (e2 <= DMS_RK45_TOL_PHI);
	if(!good)
		return RK_RETRY;
	if(within)
	{
		p.time = p.time + dt;
		p.radius = r4 < 0.0 ? 0.0 : r4;
		p.v_radial = v4;
		p.phi = p4;
		p.time_step = new_step;
		return RK_ACCEPTED;
	}
	if(new_step < DMS_RK45_ABS_MIN_STEP_S || inner >= DMS_RK45_MAX_INNER_RETRIES)
	{
		const bool ok = isfinite(r4) && isfinite(v4) && isfinite(p4);
		p.time = p.time + DMS_RK45_ABS_MIN_STEP_S;
		if(ok)
		{
			p.radius = r4 < 0.0 ? 0.0 : r4;
			p.v_radial = v4;
			p.phi = p4;
		}
		p.time_step = DMS_RK45_ABS_MIN_STEP_S;
		return RK_FORCED;
	}
	p.time_step = new_step;
	return RK_RETRY;
}

// The attempt of rk45_attempt_cert computed by two lanes of a warp: an owner (role 1, the lane
// whose propagator steps) and a helper (role 2, an idle lane), `partner` being the other lane of
// the pair.  Every lane of the warp calls it (the exchanges are warp shuffles); lanes without a
// pair (role 0) compute nothing that is kept.  The radius of stage j needs the slopes of the
// stages up to j - 2 only, so the owner computes stages 0, 2, 4 and the helper 1, 3, 5, three
// rounds instead of six, exchanging the new slopes after each round; the owner then forms the
// solutions, the helper two of the three step-size factors.  Every value is formed by the same
// operations in the same order as in rk45_attempt_cert, so the result is the same bits.  Only
// the owner's p is changed; `good` (owner) is cleared when a certificate of either lane failed.
__device__ __forceinline__ int rk45_attempt_pair(const DevSolar& S, Prop& p, int inner, int role, int partner, bool& good)
{
	constexpr unsigned int FULL = 0xffffffffu;
	const int me = threadIdx.x & 31;
	const int src = role == 2 ? partner : me;
	Prop q = p;
	q.time_step = __shfl_sync(FULL, p.time_step, src);
	q.radius = __shfl_sync(FULL, p.radius, src);
	q.v_radial = __shfl_sync(FULL, p.v_radial, src);
	q.J = __shfl_sync(FULL, p.J, src);
	q.radial_mode = __shfl_sync(FULL, p.radial_mode, src);
	const bool odd = role == 2;
	const int other = role == 0 ? me : partner;
	const double dt = q.time_step;
	const double R = q.radius, V = q.v_radial;
	double a, b;
	const double kr0 = dt * V;
	// first pair: stage 0 (owner) | stage 1 (helper)
	const double r_s1 = R + kr0 / 4.0;
	cert_stage<true>(S, q, odd ? r_s1 : R, a, b, good);
	const double kv_m1 = dt * a, kp_m1 = dt * b;
	const double kv_o1 = __shfl_sync(FULL, kv_m1, other);
	const double kv0 = odd ? kv_o1 : kv_m1, kv1 = odd ? kv_m1 : kv_o1;
	const double kr1 = dt * (V + kv0 / 4.0);
	const double kr2 = dt * (V + 3.0 / 32.0 * kv0 + 9.0 / 32.0 * kv1);
	// second pair: stage 2 | stage 3
	const double r_s2 = R + 3.0 / 32.0 * kr0 + 9.0 / 32.0 * kr1;
	const double r_s3 = R + 1932.0 / 2197.0 * kr0 - 7200.0 / 2197.0 * kr1 + 7296.0 / 2197.0 * kr2;
	cert_stage<true>(S, q, odd ? r_s3 : r_s2, a, b, good);
	const double kv_m2 = dt * a, kp_m2 = dt * b;
	const double kv_o2 = __shfl_sync(FULL, kv_m2, other);
	const double kv2 = odd ? kv_o2 : kv_m2, kv3 = odd ? kv_m2 : kv_o2;
	const double kr3 = dt * (V + 1932.0 / 2197.0 * kv0 - 7200.0 / 2197.0 * kv1 + 7296.0 / 2197.0 * kv2);
	const double kr4 = dt * (V + 439.0 / 216.0 * kv0 - 8.0 * kv1 + 3680.0 / 513.0 * kv2 - 845.0 / 4104.0 * kv3);
	// third pair: stage 4 | stage 5
	const double r_s4 = R + 439.0 / 216.0 * kr0 - 8.0 * kr1 + 3680.0 / 513.0 * kr2 - 845.0 / 4104.0 * kr3;
	const double r_s5 = R - 8.0 / 27.0 * kr0 + 2.0 * kr1 - 3544.0 / 2565.0 * kr2 + 1859.0 / 4104.0 * kr3 - 11.0 / 40.0 * kr4;
	cert_stage<true>(S, q, odd ? r_s5 : r_s4, a, b, good);
	const double kv_m3 = dt * a, kp_m3 = dt * b;
	// both lanes gather every slope: the owner's kp of rounds 1-3 are kp0, kp2, kp4, the
	// helper's kp3, kp5 (its round-1 dphi belongs to stage 1, which has none)
	const double kv_o3 = __shfl_sync(FULL, kv_m3, other);
	const double kp_o1 = __shfl_sync(FULL, kp_m1, other);
	const double kp_o2 = __shfl_sync(FULL, kp_m2, other);
	const double kp_o3 = __shfl_sync(FULL, kp_m3, other);
	const double kv4 = odd ? kv_o3 : kv_m3, kv5 = odd ? kv_m3 : kv_o3;
	const double kp0 = odd ? kp_o1 : kp_m1;
	const double kp2 = odd ? kp_o2 : kp_m2, kp3 = odd ? kp_m2 : kp_o2;
	const double kp4 = odd ? kp_o3 : kp_m3, kp5 = odd ? kp_m3 : kp_o3;
	const double kr5 = dt * (V - 8.0 / 27.0 * kv0 + 2.0 * kv1 - 3544.0 / 2565.0 * kv2 + 1859.0 / 4104.0 * kv3 - 11.0 / 40.0 * kv4);
	const double r4 = R + 25.0 / 216.0 * kr0 + 1408.0 / 2565.0 * kr2 + 2197.0 / 4104.0 * kr3 - 1.0 / 5.0 * kr4;
	const double v4 = V + 25.0 / 216.0 * kv0 + 1408.0 / 2565.0 * kv2 + 2197.0 / 4104.0 * kv3 - 1.0 / 5.0 * kv4;
	const double p4 = p.phi + 25.0 / 216.0 * kp0 + 1408.0 / 2565.0 * kp2 + 2197.0 / 4104.0 * kp3 - 1.0 / 5.0 * kp4;
	const double r5 = R + 16.0 / 135.0 * kr0 + 6656.0 / 12825.0 * kr2 + 28561.0 / 56430.0 * kr3 - 9.0 / 50.0 * kr4 + 2.0 / 55.0 * kr5;
	const double v5 = V + 16.0 / 135.0 * kv0 + 6656.0 / 12825.0 * kv2 + 28561.0 / 56430.0 * kv3 - 9.0 / 50.0 * kv4 + 2.0 / 55.0 * kv5;
	const double p5 = p.phi + 16.0 / 135.0 * kp0 + 6656.0 / 12825.0 * kp2 + 28561.0 / 56430.0 * kp3 - 9.0 / 50.0 * kp4 + 2.0 / 55.0 * kp5;
	const double e0 = fabs(r5 - r4), e1 = fabs(v5 - v4), e2 = fabs(p5 - p4);
	// the step-size factors: c0 and c2 on the owner, c1 (and c2 again) on the helper, whose e2
	// needs the owner's phi
	const double phi_o = __shfl_sync(FULL, p.phi, src);
	const double p4h = phi_o + 25.0 / 216.0 * kp0 + 1408.0 / 2565.0 * kp2 + 2197.0 / 4104.0 * kp3 - 1.0 / 5.0 * kp4;
	const double p5h = phi_o + 16.0 / 135.0 * kp0 + 6656.0 / 12825.0 * kp2 + 28561.0 / 56430.0 * kp3 - 9.0 / 50.0 * kp4 + 2.0 / 55.0 * kp5;
	const double e2h = fabs(p5h - p4h);
	const double cA = cert_step_factor(odd ? DMS_RK45_TOL_V_KMS : DMS_RK45_TOL_R_KM, odd ? e1 : e0, good);
	const double cB = cert_step_factor(DMS_RK45_TOL_PHI, e2h, good);
	const double c1 = __shfl_sync(FULL, cA, other), c2 = cB;
	const int helper_good = __shfl_sync(FULL, static_cast<int>(good), other);
	if(role != 1)
		return RK_RETRY;
	good = good && helper_good != 0;
	const double c0 = cA;
	double factor = DMS_RK45_MAX_STEP_FACTOR;
	factor = c0 < factor ? c0 : factor;
	factor = c1 < factor ? c1 : factor;
	factor = c2 < factor ? c2 : factor;
	factor = factor > DMS_RK45_MAX_STEP_FACTOR ? DMS_RK45_MAX_STEP_FACTOR : factor;
	factor = factor < DMS_RK45_MIN_STEP_FACTOR ? DMS_RK45_MIN_STEP_FACTOR : factor;
	const double grown = factor * dt;
	const double sane = (!isfinite(grown) | (grown <= 0.0)) ? DMS_RK45_DEFAULT_STEP_S
	                    : (grown < DMS_RK45_ABS_MAX_STEP_S ? grown : DMS_RK45_ABS_MAX_STEP_S);
	const bool finite_err = isfinite(e0) & isfinite(e1) & isfinite(e2);
	const double new_step = finite_err ? sane : DMS_RK45_MIN_STEP_FACTOR * dt;
	const bool within = finite_err & (e0 <= DMS_RK45_TOL_R_KM) & (e1 <= DMS_RK45_TOL_V_KMS) & (e2 <= DMS_RK45_TOL_PHI);
	if(!good)
		return RK_RETRY;
	if(within)
	{
		p.time = p.time + dt;
		p.radius = r4 < 0.0 ? 0.0 : r4;
		p.v_radial = v4;
		p.phi = p4;
		p.time_step = new_step;
		return RK_ACCEPTED;
	}
	if(new_step < DMS_RK45_ABS_MIN_STEP_S || inner >= DMS_RK45_MAX_INNER_RETRIES)
	{
		const bool ok = isfinite(r4) && isfinite(v4) && isfinite(p4);
		p.time = p.time + DMS_RK45_ABS_MIN_STEP_S;
		if(ok)
		{
			p.radius = r4 < 0.0 ? 0.0 : r4;
			p.v_radial = v4;
			p.phi = p4;
		}
		p.time_step = DMS_RK45_ABS_MIN_STEP_S;
		return RK_FORCED;
	}
	p.time_step = new_step;
	return RK_RETRY;
}

// One attempt with the certified straight-line division and square root; when any certificate
// fails (or the tables' buckets can hold two knots), the attempt is repeated from the same
// state with IEEE arithmetic.  Either way the result is bit-identical with rk45_attempt_unrolled.
__device__ __forceinline__ int rk45_attempt_certified(const DevSolar& S, Prop& p, int inner)
{
	bool good = S.bucket_single_step != 0;
	if(good)
	{
		const int rk = rk45_attempt_cert(S, p, inner, good);
		if(good)
			return rk;
	}
	return rk45_attempt_ieee(S, p, inner);
}

// Runge-Kutta-Fehlberg 4(5) coefficients of src/Simulation_Trajectory.cpp:1492-1540: stage
// weights a[i][j] (stage i from the slopes of stages j < i) and the 4th / 5th order weights.
// Zero weights are absent from the reference's sums and are skipped here.
__constant__ double RKF_A[6][5] = {
	{0.0, 0.0, 0.0, 0.0, 0.0},
	{1.0 / 4.0, 0.0, 0.0, 0.0, 0.0},
	{3.0 / 32.0, 9.0 / 32.0, 0.0, 0.0, 0.0},
	{1932.0 / 2197.0, -(7200.0 / 2197.0), 7296.0 / 2197.0, 0.0, 0.0},
	{439.0 / 216.0, -8.0, 3680.0 / 513.0, -(845.0 / 4104.0), 0.0},
	{-(8.0 / 27.0), 2.0, -(3544.0 / 2565.0), 1859.0 / 4104.0, -(11.0 / 40.0)}};
__constant__ double RKF_B4[6] = {25.0 / 216.0, 0.0, 1408.0 / 2565.0, 2197.0 / 4104.0, -(1.0 / 5.0), 0.0};
__constant__ double RKF_B5[6] = {16.0 / 135.0, 0.0, 6656.0 / 12825.0, 28561.0 / 56430.0, -(9.0 / 50.0), 2.0 / 55.0};

__device__ __forceinline__ int rk45_attempt(const DevSolar& S, Prop& p, int inner)
{
	{
		const double dt = p.time_step;
		const double J = p.J;
		// The six stages run as one loop.  Every later stage's radius and radial speed, and the
		// two solutions, are accumulators that start at the step's initial value and receive
		// a * k as each slope becomes known: the same additions, in the same order, as the
		// reference's written-out sums (x + (-a) * k equals x - a * k exactly).
		double R1 = p.radius, R2 = p.radius, R3 = p.radius, R4 = p.radius, R5 = p.radius;
		double V1 = p.v_radial, V2 = p.v_radial, V3 = p.v_radial, V4 = p.v_radial, V5 = p.v_radial;
		double r4 = p.radius, v4 = p.v_radial, p4 = p.phi, r5 = p.radius, v5 = p.v_radial, p5 = p.phi;
#pragma unroll 1
		for(int j = 0; j < 6; j++)
		{
			const double ri = j == 0 ? p.radius : j == 1 ? R1 : j == 2 ? R2 : j == 3 ? R3 : j == 4 ? R4 : R5;
			const double vi = j == 0 ? p.v_radial : j == 1 ? V1 : j == 2 ? V2 : j == 3 ? V3 : j == 4 ? V4 : V5;
			const double kr = dt * vi;
			const double kv = dt * dv_dt(J, ri, solar_gm(S, ri));
			const double kp = dt * dphi_dt(p, ri);
			if(j < 1) { const double a = RKF_A[1][j]; R1 = R1 + a * kr; V1 = V1 + a * kv; }
			if(j < 2) { const double a = RKF_A[2][j]; R2 = R2 + a * kr; V2 = V2 + a * kv; }
			if(j < 3) { const double a = RKF_A[3][j]; R3 = R3 + a * kr; V3 = V3 + a * kv; }
			if(j < 4) { const double a = RKF_A[4][j]; R4 = R4 + a * kr; V4 = V4 + a * kv; }
			if(j < 5) { const double a = RKF_A[5][j]; R5 = R5 + a * kr; V5 = V5 + a * kv; }
			const double b4 = RKF_B4[j], b5 = RKF_B5[j];
			if(b4 != 0.0) { r4 = r4 + b4 * kr; v4 = v4 + b4 * kv; p4 = p4 + b4 * kp; }
			if(b5 != 0.0) { r5 = r5 + b5 * kr; v5 = v5 + b5 * kv; p5 = p5 + b5 * kp; }
		}
		const double e0 = fabs(r5 - r4), e1 = fabs(v5 - v4), e2 = fabs(p5 - p4);
		const double new_step = next_step_size(dt, e0, e1, e2);
		const bool within = isfinite(e0) && e0 <= DMS_RK45_TOL_R_KM && isfinite(e1) && e1 <= DMS_RK45_TOL_V_KMS && isfinite(e2) && e2 <= DMS_RK45_TOL_PHI;
		if(within)
		{
			p.time = p.time + dt;
			p.radius = r4 < 0.0 ? 0.0 : r4;
			p.v_radial = v4;
			p.phi = p4;
			p.time_step = new_step;
			return RK_ACCEPTED;
		}
		if(new_step < DMS_RK45_ABS_MIN_STEP_S || inner >= DMS_RK45_MAX_INNER_RETRIES)
		{
			const bool ok = isfinite(r4) && isfinite(v4) && isfinite(p4);
			p.time = p.time + DMS_RK45_ABS_MIN_STEP_S;
			if(ok)
			{
				p.radius = r4 < 0.0 ? 0.0 : r4;
				p.v_radial = v4;
				p.phi = p4;
			}
			p.time_step = DMS_RK45_ABS_MIN_STEP_S;
			return RK_FORCED;
		}
		p.time_step = new_step;
		return RK_RETRY;
	}
}

__device__ __forceinline__ double prop_radius(const Prop& p) { return p.radius < 0.0 ? 0.0 : p.radius; }

__device__ __forceinline__ double prop_speed(const Prop& p)
{
	const double r = p.radius < 0.0 ? 0.0 : p.radius;
	if(r == 0 || p.J == 0)
		return fabs(p.v_radial);
	return sqrt(p.v_radial * p.v_radial + p.J * p.J / r / r);
}

// Event_In_3D, src/Simulation_Trajectory.cpp:1715-1742
__device__ __forceinline__ Event prop_event(const Prop& p)
{
	const double safe = (isfinite(p.radius) && p.radius > 0.0) ? p.radius : 0.0;
	Event e;
	e.t = p.time;
	if(p.radial_mode || p.J == 0.0 || safe == 0.0)
	{
		e.x = scale3(safe, p.ax);
		e.v = scale3(p.v_radial, p.ax);
		return e;
	}
	double sp, cp;
	dms_sincos(p.phi, &sp, &cp);
	const double vt = p.J / safe;
	const double vx = p.v_radial * cp - vt * sp;
	const double vy = p.v_radial * sp + vt * cp;
	e.x = mk(safe * (cp * p.ax.x + sp * p.ay.x), safe * (cp * p.ax.y + sp * p.ay.y), safe * (cp * p.ax.z + sp * p.ay.z));
	e.v = mk(vx * p.ax.x + vy * p.ay.x, vx * p.ax.y + vy * p.ay.y, vx * p.ax.z + vy * p.ay.z);
	return e;
}

// ---------------------------------------------------------------------------------------------
// Chord geometry, src/Simulation_Trajectory.cpp:65-325
__device__ __forceinline__ double step_cap(double radius, double speed, double max_distance)
{
	double cap = DMS_RK45_ABS_MAX_STEP_S;
	const double safe_speed = fabs(speed) > 1.0e-12 ? fabs(speed) : 1.0e-12;
	const double crossing = (0.25 * max_distance > 10.0) ? 0.25 * max_distance : 10.0;
	if(crossing / safe_speed < cap) cap = crossing / safe_speed;
	const double safe_radius = radius > 1.0 ? radius : 1.0;
	const double dyn = sqrt(safe_radius * safe_radius * safe_radius / DMS_GMSUN_KM3S2);
	if(isfinite(dyn) && dyn > 0.0 && 0.1 * dyn < cap) cap = 0.1 * dyn;
	return cap > DMS_RK45_ABS_MIN_STEP_S ? cap : DMS_RK45_ABS_MIN_STEP_S;
}

__device__ __forceinline__ double ev_radius(const Event& e) { return norm3(e.x); }
__device__ __forceinline__ double ev_speed(const Event& e) { return norm3(e.v); }

__device__ __forceinline__ bool outward_escaping(const DevSolar& S, const Event& e, double boundary)
{
	const double r = ev_radius(e);
	if(r < boundary)
		return false;
	const double vr = (r > 0.0) ? dot3(e.x, e.v) / r : 0.0;
	return vr > 0.0 && ev_speed(e) > solar_vesc(S, r);
}

// Bound_Kepler_Return_At_Same_Radius, src/Simulation_Trajectory.cpp:152-201
static __device__ __noinline__ bool bound_kepler_return(const Event& out, Event& in)
{
	const double radius = ev_radius(out);
	const double speed = ev_speed(out);
	const double vr = (radius <= 0.0) ? 0.0 : dot3(out.x, out.v) / radius;
	if(!isfinite(radius) || !isfinite(speed) || !isfinite(vr) || radius <= DMS_RSUN_KM || speed <= 0.0 || vr <= 0.0)
		return false;
	const double mu = DMS_GMSUN_KM3S2;
	const double E = 0.5 * speed * speed - mu / radius;
	if(!isfinite(E) || E >= 0.0)
		return false;
	const double J = norm3(cross3(out.x, out.v));
	if(!isfinite(J))
		return false;
	const double a = -mu / (2.0 * E);
	if(!isfinite(a) || a <= 0.0)
		return false;
	double e2 = 1.0 + 2.0 * E * J * J / (mu * mu);
	if(!isfinite(e2) || e2 < 0.0)
		return false;
	e2 = e2 > 0.0 ? e2 : 0.0;
	const double ecc = sqrt(e2);
	if(ecc <= 1.0e-14 || ecc >= 1.0)
		return false;
	const double cosE = clamp_cos((1.0 - radius / a) / ecc);
	const double Eanom = dms_acos(cosE);
	const double one_minus = 1.0 - cosE * cosE;
	const double sinE = sqrt(one_minus > 0.0 ? one_minus : 0.0);
	const double n = sqrt(mu / (a * a * a));
	if(!isfinite(n) || n <= 0.0)
		return false;
	const double T = (2.0 * DMS_PI - 2.0 * Eanom + 2.0 * ecc * sinE) / n;
	if(!isfinite(T) || T <= 0.0)
		return false;
	const Vec3 rhat = div3(out.x, radius);
	in = out;
	in.t += T;
	in.v = sub3(out.v, scale3(2.0 * vr, rhat));
	return in.t > out.t && isfinite(ev_speed(in));
}

// Interpolate_Event, src/Simulation_Trajectory.cpp:203-216
__device__ __forceinline__ Event interpolate_event(const Event& a, const Event& b, double f)
{
	f = clamp_unit(f);
	Event e;
	e.x = mk(a.x.x + f * (b.x.x - a.x.x), a.x.y + f * (b.x.y - a.x.y), a.x.z + f * (b.x.z - a.x.z));
	e.v = mk(a.v.x + f * (b.v.x - a.v.x), a.v.y + f * (b.v.y - a.v.y), a.v.z + f * (b.v.z - a.v.z));
	e.t = a.t + f * (b.t - a.t);
	return e;
}

__device__ __forceinline__ double radius_at_fraction(const Event& a, const Event& b, double f)
{
	f = clamp_unit(f);
	const double x = a.x.x + f * (b.x.x - a.x.x);
	const double y = a.x.y + f * (b.x.y - a.x.y);
	const double z = a.x.z + f * (b.x.z - a.x.z);
	double r2 = 0.0;
	r2 += x * x;
	r2 += y * y;
	r2 += z * z;
	return sqrt(r2 > 0.0 ? r2 : 0.0);
}

__device__ __forceinline__ bool surface_crossings(const Event& a, const Event& b, double& first, double& second)
{
	const double dx = b.x.x - a.x.x, dy = b.x.y - a.x.y, dz = b.x.z - a.x.z;
	double qa = 0.0, qb = 0.0, qc = -DMS_RSUN_KM * DMS_RSUN_KM;
	qa += dx * dx;
	qb += 2.0 * a.x.x * dx;
	qc += a.x.x * a.x.x;
	qa += dy * dy;
	qb += 2.0 * a.x.y * dy;
	qc += a.x.y * a.x.y;
	qa += dz * dz;
	qb += 2.0 * a.x.z * dz;
	qc += a.x.z * a.x.z;
	if(qa <= 0.0)
		return false;
	const double disc = qb * qb - 4.0 * qa * qc;
	if(!isfinite(disc) || disc < 0.0)
		return false;
	const double sq = sqrt(disc > 0.0 ? disc : 0.0);
	first = (-qb - sq) / (2.0 * qa);
	second = (-qb + sq) / (2.0 * qa);
	if(first > second)
	{
		const double t = first;
		first = second;
		second = t;
	}
	return true;
}

__device__ __forceinline__ bool in_unit(double f) { return f >= -1.0e-12 && f <= 1.0 + 1.0e-12; }

static __device__ __noinline__ double find_crossing(const Event& a, const Event& b, double lower, double upper)
{
	double r_lower = radius_at_fraction(a, b, lower) - DMS_RSUN_KM;
	for(int it = 0; it < 60; it++)
	{
		const double mid = 0.5 * (lower + upper);
		const double r_mid = radius_at_fraction(a, b, mid) - DMS_RSUN_KM;
		if((r_lower <= 0.0 && r_mid <= 0.0) || (r_lower >= 0.0 && r_mid >= 0.0))
		{
			lower = mid;
			r_lower = r_mid;
		}
		else
			upper = mid;
	}
	return clamp_unit(0.5 * (lower + upper));
}

// Solar_Interior_Fraction_Interval, src/Simulation_Trajectory.cpp:282-325
__device__ __forceinline__ bool interior_interval(const Event& a, const Event& b, double ra, double rb, double& start, double& end)
{
	const bool a_in = ra < DMS_RSUN_KM, b_in = rb < DMS_RSUN_KM;
	if(a_in && b_in)
	{
		start = 0.0;
		end = 1.0;
		return true;
	}
	double c1 = 0.0, c2 = 0.0;  // the crossings matter only when a chord end is outside
	const bool has = surface_crossings(a, b, c1, c2);
	if(!a_in && b_in)
	{
		if(has && in_unit(c1))
			start = clamp_unit(c1);
		else if(has && in_unit(c2))
			start = clamp_unit(c2);
		else
			start = find_crossing(a, b, 0.0, 1.0);
		end = 1.0;
		return end > start;
	}
	if(a_in && !b_in)
	{
		start = 0.0;
		if(has && in_unit(c2))
			end = clamp_unit(c2);
		else if(has && in_unit(c1))
			end = clamp_unit(c1);
		else
			end = find_crossing(a, b, 0.0, 1.0);
		return end > start;
	}
	if(has && in_unit(c1) && in_unit(c2))
	{
		start = clamp_unit(c1);
		end = clamp_unit(c2);
		return end > start;
	}
	return false;
}

// Scattering_Rate_At_Fraction, src/Simulation_Trajectory.cpp:327-345
__device__ __forceinline__ double rate_at_fraction(const DevSolar& S, const DevPoint* __restrict__ P, const Event& a, const Event& b, double f)
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
	const double r = sqrt(r2 > 0.0 ? r2 : 0.0);
	if(r >= DMS_RSUN_KM)
		return 0.0;
	return rate_total(S, P, r, sqrt(v2 > 0.0 ? v2 : 0.0));
}

// Solve_Linear_Rate_Optical_Depth_Fraction, src/Simulation_Trajectory.cpp:416-464
static __device__ __noinline__ double solve_linear_rate(double r0, double r1, double dt, double target)
{
	if(target <= 0.0)
		return 0.0;
	if(!isfinite(target) || dt <= 0.0)
		return 1.0;
	if(!isfinite(r0) || !isfinite(r1) || r0 < 0.0 || r1 < 0.0)
		return 1.0;
	const double total = 0.5 * (r0 + r1) * dt;
	if(!isfinite(total) || total <= 0.0)
		return 1.0;
	if(target >= total)
		return 1.0;
	const double tg = target / dt;
	const double a = 0.5 * (r1 - r0);
	const double b = r0;
	if(fabs(a) < 1.0e-300)
		return (b > 0.0) ? clamp_unit(tg / b) : 1.0;
	const double disc = b * b + 4.0 * a * tg;
	if(isfinite(disc) && disc >= 0.0)
	{
		const double sq = sqrt(disc);
		const double root0 = (-b + sq) / (2.0 * a);
		if(isfinite(root0) && root0 >= 0.0 && root0 <= 1.0)
			return clamp_unit(root0);
		const double root1 = (-b - sq) / (2.0 * a);
		if(isfinite(root1) && root1 >= 0.0 && root1 <= 1.0)
			return clamp_unit(root1);
	}
	double lo = 0.0, hi = 1.0;
	for(int it = 0; it < 30; it++)
	{
		const double mid = 0.5 * (lo + hi);
		const double tm = dt * (r0 * mid + 0.5 * (r1 - r0) * mid * mid);
		if(tm < target)
			lo = mid;
		else
			hi = mid;
	}
	return clamp_unit(0.5 * (lo + hi));
}

// Unit_Vector_At_Angle_From_Axis, src/Simulation_Trajectory.cpp:109-128
__device__ __forceinline__ bool unit_vector_at_angle(double cos_theta, double phi, const Vec3& axis, Vec3& out)
{
	if(!isfinite(cos_theta) || cos_theta < -1.0 - 1.0e-12 || cos_theta > 1.0 + 1.0e-12 || !isfinite(phi))
		return false;
	const double n = norm3(axis);
	if(!isfinite(n) || n <= 0.0)
		return false;
	const Vec3 e3 = div3(axis, n);
	const Vec3 ref = (fabs(e3.z) < 0.9) ? mk(0.0, 0.0, 1.0) : mk(1.0, 0.0, 0.0);
	const Vec3 e1 = normalized3(cross3(ref, e3));
	const Vec3 e2 = normalized3(cross3(e3, e1));
	cos_theta = clamp_cos(cos_theta);
	const double st2 = 1.0 - cos_theta * cos_theta;
	const double st = sqrt(st2 > 0.0 ? st2 : 0.0);
	double sp, cp;
	dms_sincos(phi, &sp, &cp);
	out = mk(cos_theta * e3.x + st * cp * e1.x + st * sp * e2.x, cos_theta * e3.y + st * cp * e1.y + st * sp * e2.y,
	         cos_theta * e3.z + st * cp * e1.z + st * sp * e2.z);
	return true;
}

// One channel of Total_DM_Scattering_Rate_Computed (src/Solar_Model.cpp:263-303) at knot
// interval i, offset dr and temperature T: k < DMS_NUM_TARGETS the isotope k, k ==
// DMS_NUM_TARGETS the electrons.  Same expressions, in the same order, as rate_computed.
// The scattering angle of channel k (k < 0: the electron), one draw: isotropic for the contact
// interactions, the General form factor's closed form otherwise (src/Dark_Photon.cpp:286-325).
__device__ __forceinline__ double sample_cos_alpha(const DevPoint* __restrict__ P, Draws& D, int k, double v)
{
	if(__ldg(&P->interaction) != DMS_INTERACTION_DARK_PHOTON_GENERAL)
		return D.uniform(-1.0, 1.0);
	const double xi = D.uniform(0.0, 1.0);
	const double m2 = __ldg(&P->ff_m2);
	const double q2 = __ldg(&P->q2c[k < 0 ? DMS_NUM_TARGETS : k]) * (v * v);
	return (m2 * (2.0 * xi - 1.0) + q2 * xi) / (m2 + q2 * xi);
}

__device__ __forceinline__ double channel_rate(const DevSolar& S, const DevPoint* __restrict__ P, int i, double dr, double T, double v, int k)
{
	if(k == DMS_NUM_TARGETS)
	{
		const double ne = __ldg(S.ne + i) + dr * __ldg(S.ne_s + i);
		return ne * channel_sigma(P, k, v) * thermal_relative_speed(T, DMS_MELECTRON_GEV, v);
	}
	const size_t o = static_cast<size_t>(i) * DMS_NUM_TARGETS + k;
	const double n = __ldg(S.nt + o) + dr * __ldg(S.nt_s + o);
	return n * channel_sigma(P, k, v) * thermal_relative_speed(T, __ldg(S.target_mass + k), v);
}

constexpr int TARGET_FAILED = -2;

// Sample_Target (src/Simulation_Trajectory.cpp:1122-1158) works on the 64 channel rates
// rates[0..62] (isotopes) and rates[63] (electrons): every rate must be finite and >= 0 (the
// reference throws otherwise), the total is summed in the reference's order, and one uniform
// draw picks the channel by the cumulative sum of rate / total.  The result is -1 for an
// electron, the isotope index, or TARGET_FAILED.

// Total rate: the electron channel plus the 63 isotopes in order.
__device__ __forceinline__ double channel_total(const double* rates)
{
	double total = rates[DMS_NUM_TARGETS];
	for(int k = 0; k < DMS_NUM_TARGETS; k++) total += rates[k];
	return total;
}

// The cumulative pick from the fractions q[k] = rate_k / total (q[63] the electrons).
__device__ __forceinline__ int pick_from_fractions(Draws& D, const double* q)
{
	const double xi = D.uniform(0.0, 1.0);
	int target = -1;
	double sum = q[DMS_NUM_TARGETS];
	if(!(sum > xi))
	{
		for(int k = 0; k < DMS_NUM_TARGETS; k++)
		{
			sum += q[k];
			if(sum > xi || k == DMS_NUM_TARGETS - 1)
			{
				target = k;
				break;
			}
		}
	}
	return target;
}


// The rest of Scatter once the target is known: Sample_Target_Velocity, the scattering angle
// and New_DM_Velocity, src/Simulation_Trajectory.cpp:1160-1269.  Returns
// false where the reference throws.
static __device__ __noinline__ bool scatter_with_target(const DevSolar& S, const DevPoint* __restrict__ P, Draws& D, Event& e, int target)
{
	const double r = ev_radius(e);
	double m_target;
	if(target < 0)
		m_target = DMS_MELECTRON_GEV;
	else
		m_target = __ldg(S.target_mass + target);
	const double T = solar_temperature(S, r);
	if(!isfinite(T) || T <= 0.0 || !isfinite(m_target) || m_target <= 0.0)
		return false;
	const double kappa = sqrt(m_target / 2.0 / T) / DMS_C_KMS;
	const double vdm = norm3(e.v);
	if(!isfinite(kappa) || kappa <= 0.0 || !isfinite(vdm) || vdm <= 0.0)
		return false;
	const double y = kappa * vdm;
	double x = y, mu = 1.0;
	unsigned long attempts = 0;
	const double sqrt_pi = sqrt(DMS_PI);
	for(;;)
	{
		const double x2 = x * x, y2 = y * y;
		const double raw = x2 + y2 - 2.0 * x * y * mu;
		const double den = x + y;
		const double ax = fabs(x * y);
		const double rs = (1.0 > x2 + y2 + 2.0 * ax) ? 1.0 : x2 + y2 + 2.0 * ax;
		if(!isfinite(x) || x < 0.0 || !isfinite(y) || y <= 0.0 || !isfinite(mu) || mu < -1.0 || mu > 1.0 || !isfinite(raw) ||
		   raw < -1.0e-12 * rs || !isfinite(den) || den <= 0.0)
			return false;
		const double rel2 = raw > 0.0 ? raw : 0.0;
		const double ratio = sqrt(rel2) / den;
		if(!isfinite(ratio) || ratio < 0.0 || ratio > 1.0 + 1.0e-12)
			return false;
		const double accept = ratio < 1.0 ? ratio : 1.0;
		if(!(accept < D.uniform(0.0, 1.0)))
			break;
		attempts++;
		if(attempts > DMS_TARGET_VELOCITY_MAX_REJECTIONS)
			return false;
		mu = D.uniform(-1.0, 1.0);
		const double xi1 = D.uniform(0.0, 1.0);
		if(xi1 < 2.0 / (sqrt_pi * y + 2.0))
		{
			const double xi2 = D.positive_unit();
			const double xi3 = D.positive_unit();
			const double z = -dms_log(xi2) - dms_log(xi3);
			x = sqrt(z);
		}
		else
		{
			const double xi2 = D.positive_unit();
			const double xi3 = D.uniform(0.0, 1.0);
			const double xi4 = D.positive_unit();
			const double c = dms_cos(DMS_PI / 2.0 * xi3);
			const double z = -dms_log(xi2) - (c * c) * dms_log(xi4);
			x = sqrt(z);
		}
	}
	const double vT = x / kappa;
	const double phi_t = D.uniform(0.0, 2.0 * DMS_PI);
	Vec3 unit_t;
	if(!unit_vector_at_angle(mu, phi_t, e.v, unit_t))
		return false;
	const Vec3 vel_t = scale3(vT, unit_t);
	if(!isfinite(norm3(vel_t)))
		return false;
	const double cos_alpha = sample_cos_alpha(P, D, target, vdm);
	const double md = __ldg(&P->m_dm);
	if(!isfinite(cos_alpha) || cos_alpha < -1.0 - 1.0e-12 || cos_alpha > 1.0 + 1.0e-12 || !isfinite(md) || md <= 0.0 ||
	   !isfinite(norm3(e.v)) || !isfinite(norm3(vel_t)))
		return false;
	const double ca = clamp_cos(cos_alpha);
	const double phi_n = D.uniform(0.0, 2.0 * DMS_PI);
	Vec3 n;
	if(!unit_vector_at_angle(ca, phi_n, e.v, n))
		return false;
	const double rel_speed = norm3(sub3(vel_t, e.v));
	const double mt = m_target;
	const double sc = mt * rel_speed / (mt + md);
	const Vec3 out = mk(sc * n.x + (md * e.v.x + mt * vel_t.x) / (mt + md), sc * n.y + (md * e.v.y + mt * vel_t.y) / (mt + md),
	                    sc * n.z + (md * e.v.z + mt * vel_t.z) / (mt + md));
	if(!isfinite(norm3(out)))
		return false;
	e.v = out;
	return true;
}

// Capture_Energy_eV, src/Simulation_Trajectory.cpp:682-687
__device__ __forceinline__ double capture_energy_eV(const DevSolar& S, double m_dm, double r, double v)
{
	const double vesc = solar_vesc(S, r);
	const double E = 0.5 * m_dm * ((v * v - vesc * vesc) / (DMS_C_KMS * DMS_C_KMS));
	return E / 1.0e-9;
}

}	// namespace dms
