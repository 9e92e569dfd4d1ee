/*
 * dms_oracle.c — CPU oracle of the DaMaSCUS-SUN trajectory Monte Carlo (TEST INFRASTRUCTURE).
 *
 * Plain-C restatement of the reference's per-trajectory path in km/s units.  Every function
 * cites the reference lines it follows (paths relative to the reference checkout).  Only
 * tests/, the smoke check and bench.py's CPU-baseline leg use this file, and only as the
 * checker: the engine never links or calls it.
 *
 * Third-party numerics that the reference takes from libphysica/obscura follow the same
 * restatements as the shims in oracle/shim (piecewise-linear tables, escape-speed quadrature,
 * SI contact cross sections, isotropic angles, Standard Halo Model), so this file, the reference
 * build in oracle/_ref and the CUDA engine start from the same numbers.
 */
#define _GNU_SOURCE
#include "dms_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../include/dms_constants.h"
#include "../include/dms_math.h"
#include "../include/dms_nuclear_data.h"
#include "../include/dms_philox.h"

#define PI 3.14159265358979323846

/* Work-unit marks for the op-counting build (oracle/opcount.hpp); no-ops otherwise. */
#ifndef DMS_OPS_MARK
#define DMS_OPS_MARK(kind)
#define DMS_OPS_PHASE(kind)
#endif
#define SQRT_PI sqrt(PI) /* as the reference: sqrt(M_PI), not the rounded literal */
#define PI_1_5 5.5683279968317078453

/* ------------------------------------------------------------------------------------------
 * 3-vectors and events (libphysica::Vector semantics, oracle/shim/libphysica/Linear_Algebra.hpp)
 */
typedef struct
{
	double x[3];
} vec3;

static vec3 v3(double a, double b, double c)
{
	vec3 r = {{a, b, c}};
	return r;
}
static double v_dot(vec3 a, vec3 b)
{
	double s = 0.0;
	for(int i = 0; i < 3; i++) s += a.x[i] * b.x[i];
	return s;
}
static double v_norm(vec3 a) { return sqrt(v_dot(a, a)); }
static vec3 v_cross(vec3 a, vec3 b)
{
	return v3(a.x[1] * b.x[2] - a.x[2] * b.x[1], a.x[2] * b.x[0] - a.x[0] * b.x[2], a.x[0] * b.x[1] - a.x[1] * b.x[0]);
}
static vec3 v_div(vec3 a, double s) { return v3(a.x[0] / s, a.x[1] / s, a.x[2] / s); }
static vec3 v_scale(double s, vec3 a) { return v3(s * a.x[0], s * a.x[1], s * a.x[2]); }
static vec3 v_add(vec3 a, vec3 b) { return v3(a.x[0] + b.x[0], a.x[1] + b.x[1], a.x[2] + b.x[2]); }
static vec3 v_sub(vec3 a, vec3 b) { return v3(a.x[0] - b.x[0], a.x[1] - b.x[1], a.x[2] - b.x[2]); }
static vec3 v_normalized(vec3 a) { return v_div(a, v_norm(a)); }

typedef struct
{
	double time;
	vec3 position, velocity;
} event_t;

static double ev_radius(const event_t* e) { return v_norm(e->position); }
static double ev_speed(const event_t* e) { return v_norm(e->velocity); }

/* ------------------------------------------------------------------------------------------
 * Tabulated functions (libphysica::Interpolation restated: piecewise linear,
 * oracle/shim/libphysica/Numerics.hpp)
 */
typedef struct
{
	int n;
	const double* x;   /* knots (shared) */
	double* y;
	double* s;         /* slopes */
} table1d;

static void table_slopes(table1d* t)
{
	for(int i = 0; i + 1 < t->n; i++) t->s[i] = (t->y[i + 1] - t->y[i]) / (t->x[i + 1] - t->x[i]);
}

static int table_index(const table1d* t, double x)
{
	int lo = 0, hi = t->n - 1;
	if(x >= t->x[hi - 1])
		return hi - 1;
	while(hi - lo > 1)
	{
		const int mid = (lo + hi) / 2;
		if(t->x[mid] <= x)
			lo = mid;
		else
			hi = mid;
	}
	return lo;
}

static double table_eval(const table1d* t, double x)
{
	const int i = table_index(t, x);
	return t->y[i] + (x - t->x[i]) * t->s[i];
}

/* ------------------------------------------------------------------------------------------
 * Oracle state
 */
struct dms_oracle
{
	char error[256];
	int n;                 /* radial knots (1970 for AGSS09) */
	double* r;             /* knots [km] */
	table1d gm, temp, vesc2, n_e;
	table1d targets[DMS_NUM_TARGETS];
	double target_mass_gev[DMS_NUM_TARGETS];
	/* point */
	int has_point;
	double m_dm;                       /* GeV */
	double sigma_target[DMS_NUM_TARGETS]; /* km^2 */
	double sigma_e;                    /* km^2 */
	unsigned int interaction;          /* DMS_INTERACTION_* */
	double ff_num, ff_m2;              /* General form factor: (q_ref^2 + m^2)^2 / m^2 and m^2 [GeV^2] */
	double q2c[DMS_NUM_TARGETS + 1];   /* 4 mu_k^2 / c^2 [GeV^2 s^2/km^2], [63] the electron */
	double v0, vesc_halo, vobs;        /* km/s */
	vec3 vel_obs;
	double n_esc;
	double halo_avg_speed, halo_eta0;
	int grid_n;
	double* grid;
	double grid_inv_r, grid_inv_v, grid_vmax;
	/* per-trajectory draw stream */
	uint32_t seed, point;
	uint64_t traj, draw_index;
	/* per-trajectory scatter trace */
	double* trace;
	size_t trace_capacity, trace_length;
	/* reflection-spectrum sample of the current trajectory (speed at 1 AU, cosine to the Sun's
	 * velocity), or NULL */
	double* reflection;
	double* reflection_base;
	/* when non-NULL: 7 doubles (t, x, v) per trajectory that replace the event after the initial
	 * Kepler shift (the initial conditions still run, for their draws) */
	const double* start_base;
};

static double next_uniform(dms_oracle* o) { return dms_draw_uniform(o->seed, o->point, o->traj, o->draw_index++); }

/* libphysica::Sample_Uniform restated (oracle/shim/libphysica/Statistics.hpp) */
static double sample_uniform(dms_oracle* o, double a, double b)
{
	const double u = next_uniform(o);
	return a + u * (b - a);
}

/* Positive_Unit_Uniform, src/Simulation_Trajectory.cpp:103-107 */
static double positive_unit_uniform(dms_oracle* o)
{
	const double u = sample_uniform(o, 0.0, 1.0);
	return u > DBL_MIN ? u : DBL_MIN;
}

/* ------------------------------------------------------------------------------------------
 * Solar model: import and tables, src/Solar_Model.cpp:43-166
 */
static int load_solar(dms_oracle* o, const char* path)
{
	FILE* f = fopen(path, "r");
	if(!f)
	{
		snprintf(o->error, sizeof o->error, "cannot open %s", path);
		return -1;
	}
	char line[4096];
	for(int i = 0; i < DMS_SOLAR_DATA_SKIP_LINES; i++)
		if(!fgets(line, sizeof line, f))
			break;
	size_t cap = 2048, rows = 0;
	double* raw = (double*)malloc(cap * DMS_SOLAR_COLUMNS * sizeof(double));
	while(fgets(line, sizeof line, f))
	{
		double vals[DMS_SOLAR_COLUMNS];
		int k = 0;
		char* p = line;
		char* end;
		while(k < DMS_SOLAR_COLUMNS)
		{
			const double v = strtod(p, &end);
			if(end == p)
				break;
			vals[k++] = v;
			p = end;
		}
		if(k == 0)
			continue;
		if(k != DMS_SOLAR_COLUMNS)
		{
			snprintf(o->error, sizeof o->error, "malformed solar model row %zu", rows);
			free(raw);
			fclose(f);
			return -1;
		}
		if(rows + 2 >= cap)
		{
			cap *= 2;
			raw = (double*)realloc(raw, cap * DMS_SOLAR_COLUMNS * sizeof(double));
		}
		memcpy(raw + (rows + 1) * DMS_SOLAR_COLUMNS, vals, sizeof vals);
		rows++;
	}
	fclose(f);
	if(rows < 2)
	{
		snprintf(o->error, sizeof o->error, "solar model has too few rows");
		free(raw);
		return -1;
	}
	/* padding rows, src/Solar_Model.cpp:47-65 (values in file units here) */
	const int n = (int)rows + 2;
	double* first = raw;
	double* last = raw + (n - 1) * DMS_SOLAR_COLUMNS;
	const double* front = raw + DMS_SOLAR_COLUMNS;
	const double* back = raw + (n - 2) * DMS_SOLAR_COLUMNS;
	for(int i = 0; i < DMS_SOLAR_COLUMNS; i++)
	{
		first[i] = (i == 0 || i == 1) ? 0.0 : front[i];
		last[i] = back[i];
	}
	last[0] = 1.0;
	last[1] = 1.0;
	last[2] = DMS_PHOTOSPHERE_T_K;
	last[3] = DMS_PHOTOSPHERE_RHO_GCM3;

	o->n = n;
	o->r = (double*)malloc(n * sizeof(double));
	for(int i = 0; i < n; i++) o->r[i] = raw[i * DMS_SOLAR_COLUMNS + 1] * DMS_RSUN_KM;

	table1d* tabs[4] = {&o->gm, &o->temp, &o->vesc2, &o->n_e};
	for(int k = 0; k < 4; k++)
	{
		tabs[k]->n = n;
		tabs[k]->x = o->r;
		tabs[k]->y = (double*)calloc(n, sizeof(double));
		tabs[k]->s = (double*)calloc(n, sizeof(double));
	}
	/* mass -> gravitational parameter G*M(r) [km^3/s^2]; temperature in GeV (natural) */
	for(int i = 0; i < n; i++)
	{
		o->gm.y[i] = raw[i * DMS_SOLAR_COLUMNS + 0] * DMS_GMSUN_KM3S2;
		o->temp.y[i] = raw[i * DMS_SOLAR_COLUMNS + 2] * DMS_KB_GEV_PER_K;
	}
	table_slopes(&o->gm);
	table_slopes(&o->temp);

	/* escape speed, Create_Escape_Speed_Table src/Solar_Model.cpp:79-96, integrand Mass(x)/x^2
	 * with integrand(0) = 0; quadrature restated in oracle/shim/libphysica/Integration.hpp */
	for(int k = 0; k < n; k++)
	{
		const double rk = o->r[k];
		double integral;
		if(rk < DMS_RSUN_KM)
		{
			integral = 0.0;
			for(int j = k; j + 1 < n; j++)
			{
				const double lo = o->r[j], hi = o->r[j + 1];
				const double f_lo = (lo == 0.0) ? 0.0 : table_eval(&o->gm, lo) / lo / lo;
				const double f_hi = (hi == 0.0) ? 0.0 : table_eval(&o->gm, hi) / hi / hi;
				if(lo == 0.0)
				{
					integral += 0.5 * (hi - lo) * (f_lo + f_hi);
					continue;
				}
				const double g_lo = f_lo * lo * lo, g_hi = f_hi * hi * hi;
				const double h = hi - lo;
				const double s = (g_hi - g_lo) / h;
				integral += g_lo * h / (lo * hi) + s * (log1p(h / lo) - h / hi);
			}
		}
		else
			integral = DMS_GMSUN_KM3S2 * (1.0 / rk - 1.0 / DMS_RSUN_KM);
		o->vesc2.y[k] = 2.0 * DMS_GMSUN_KM3S2 / DMS_RSUN_KM * (1.0 + DMS_RSUN_KM / DMS_GMSUN_KM3S2 * integral);
	}
	table_slopes(&o->vesc2);

	/* isotope number densities, Create_Number_Density_Table src/Solar_Model.cpp:98-110 and
	 * the target list :143-163; n = f rho / m, then Multiply(abundance) */
	for(int t = 0; t < DMS_NUM_TARGETS; t++)
	{
		const dms_target_isotope* iso = &DMS_TARGET_ISOTOPES[t];
		const double m_gev = (iso->A == 1) ? DMS_MPROTON_GEV : iso->A * DMS_MNUCLEON_GEV;
		const double m_kg = m_gev / DMS_GEV_PER_KG;
		o->target_mass_gev[t] = m_gev;
		table1d* tb = &o->targets[t];
		tb->n = n;
		tb->x = o->r;
		tb->y = (double*)calloc(n, sizeof(double));
		tb->s = (double*)calloc(n, sizeof(double));
		for(int i = 0; i < n; i++)
		{
			const double rho = raw[i * DMS_SOLAR_COLUMNS + 3] * 1.0e12; /* g/cm^3 -> kg/km^3 */
			const double frac = raw[i * DMS_SOLAR_COLUMNS + 6 + iso->element_index];
			tb->y[i] = frac * rho / m_kg;
		}
		if(iso->element_index >= 10)
			for(int i = 0; i < n; i++) tb->y[i] *= iso->abundance;
		table_slopes(tb);
	}
	/* electrons, Create_Number_Density_Table_Electron src/Solar_Model.cpp:112-126 */
	for(int t = 0; t < DMS_NUM_TARGETS; t++)
		for(int i = 0; i < n; i++)
		{
			const double ri = o->r[i];
			const double nt = (ri > DMS_RSUN_KM) ? 0.0 : table_eval(&o->targets[t], ri < 0.0 ? 0.0 : ri);
			o->n_e.y[i] += (double)DMS_TARGET_ISOTOPES[t].Z * nt;
		}
	table_slopes(&o->n_e);
	free(raw);
	return 0;
}

/* Solar_Model::Mass as G*M, src/Solar_Model.cpp:168-179 */
static double solar_gm(const dms_oracle* o, double r)
{
	if(!isfinite(r))
		return NAN;
	if(r < 0.0)
		r = 0.0;
	if(r > DMS_RSUN_KM)
		return DMS_GMSUN_KM3S2;
	return table_eval(&o->gm, r);
}

/* Solar_Model::Temperature [GeV], src/Solar_Model.cpp:194-202 */
static double solar_temperature(const dms_oracle* o, double r)
{
	if(!isfinite(r))
		return NAN;
	if(r < 0.0)
		r = 0.0;
	return table_eval(&o->temp, r);
}

/* Solar_Model::Local_Escape_Speed, src/Solar_Model.cpp:204-218 */
static double solar_vesc(const dms_oracle* o, double r)
{
	if(!isfinite(r))
		return NAN;
	if(r < 0.0)
		r = 0.0;
	if(r > DMS_RSUN_KM)
		return sqrt(2 * DMS_GMSUN_KM3S2 / r);
	return sqrt(table_eval(&o->vesc2, r));
}

/* Solar_Isotope::Number_Density / Number_Density_Electron, src/Solar_Model.cpp:28-39, 250-261 */
static double solar_density(const table1d* t, double r)
{
	if(!isfinite(r))
		return NAN;
	if(r < 0.0)
		r = 0.0;
	if(r > DMS_RSUN_KM)
		return 0.0;
	return table_eval(t, r);
}

/* Thermal_Averaged_Relative_Speed, src/Solar_Model.cpp:493-521; T in GeV, m in GeV, v in km/s.
 * kappa is converted from 1/c to s/km. */
static double thermal_relative_speed(double temperature, double mass_target, double v)
{
	if(!isfinite(temperature) || temperature <= 0.0 || !isfinite(mass_target) || mass_target <= 0.0 || !isfinite(v) || v < 0.0)
		return NAN;
	const double kappa = sqrt(mass_target / (2.0 * temperature)) / DMS_C_KMS;
	if(!isfinite(kappa) || kappa <= 0.0)
		return NAN;
	if(v == 0.0)
		return 2.0 / SQRT_PI / kappa;
	const double x = kappa * v;
	if(!isfinite(x))
		return v;
	if(x < 1.0e-4)
	{
		const double x2 = x * x;
		return 2.0 / SQRT_PI / kappa * (1.0 + x2 / 3.0 - x2 * x2 / 30.0 + x2 * x2 * x2 / 210.0);
	}
	if(x > 26.0)
		return v * (1.0 + 0.5 / (x * x));
	const double x2 = x * x;
	return v * ((1.0 + 2.0 * x2) * erf(x) / (2.0 * x2) + exp(-x2) / (SQRT_PI * x));
}

/* Sigma_Total_Nucleus / Sigma_Total_Electron at DM speed v [km/s] of channel k (k = 63: the
 * electron): the contact cross section, times (q_ref^2 + m^2)^2 / (m^2 (m^2 + q_max^2)) for the
 * dark photon's General form factor (src/Dark_Photon.cpp:190-229), q_max^2 = 4 mu_k^2 v^2 / c^2. */
static double channel_sigma(const dms_oracle* o, int k, double v)
{
	const double sigma = (k == DMS_NUM_TARGETS) ? o->sigma_e : o->sigma_target[k];
	if(o->interaction != DMS_INTERACTION_DARK_PHOTON_GENERAL)
		return sigma;
	const double q2 = o->q2c[k] * (v * v);
	return sigma * (o->ff_num / (o->ff_m2 + q2));
}

/* DM_Scattering_Rate_Electron / _Nucleus, src/Solar_Model.cpp:263-303 */
static double rate_electron(const dms_oracle* o, double r, double v)
{
	if(!isfinite(r) || !isfinite(v))
		return NAN;
	if(r < 0.0)
		r = 0.0;
	if(v < 0.0)
		v = 0.0;
	if(r > DMS_RSUN_KM)
		return 0.0;
	const double vrel = thermal_relative_speed(solar_temperature(o, r), DMS_MELECTRON_GEV, v);
	return solar_density(&o->n_e, r) * channel_sigma(o, DMS_NUM_TARGETS, v) * vrel;
}

static double rate_nucleus(const dms_oracle* o, double r, double v, int t)
{
	if(!isfinite(r) || !isfinite(v))
		return NAN;
	if(r < 0.0)
		r = 0.0;
	if(v < 0.0)
		v = 0.0;
	if(r > DMS_RSUN_KM)
		return 0.0;
	const double vrel = thermal_relative_speed(solar_temperature(o, r), o->target_mass_gev[t], v);
	return solar_density(&o->targets[t], r) * channel_sigma(o, t, v) * vrel;
}

/* Total_DM_Scattering_Rate_Computed, src/Solar_Model.cpp:324-342 */
static double rate_computed(const dms_oracle* o, double r, double v)
{
	if(!isfinite(r) || !isfinite(v))
		return NAN;
	if(r < 0.0)
		r = 0.0;
	if(v < 0.0)
		v = 0.0;
	if(r > DMS_RSUN_KM)
		return 0.0;
	double total = rate_electron(o, r, v);
	for(int t = 0; t < DMS_NUM_TARGETS; t++) total += rate_nucleus(o, r, v, t);
	return total;
}

/* Total_DM_Scattering_Rate_Interpolated, src/Solar_Model.cpp:344-393 */
static double rate_interpolated(const dms_oracle* o, double r, double v)
{
	if(!isfinite(r) || !isfinite(v))
		return NAN;
	if(r > DMS_RSUN_KM || r < 0.0)
		return 0.0;
	if(v < 0.0)
		return 0.0;
	if(v > o->grid_vmax)
		return rate_computed(o, r, v);
	const double rc = r * o->grid_inv_r;
	const double vc = v * o->grid_inv_v;
	if(!isfinite(rc) || !isfinite(vc) || rc < 0.0 || vc < 0.0)
		return rate_computed(o, r, v);
	const unsigned int N = (unsigned int)o->grid_n;
	unsigned int ri = (unsigned int)rc;
	unsigned int vi = (unsigned int)vc;
	if(ri > N - 2) ri = N - 2;
	if(vi > N - 2) vi = N - 2;
	const double rf = rc - ri;
	const double vf = vc - vi;
	const size_t lower = (size_t)ri * N + vi;
	const size_t upper = lower + N;
	const double lower_rate = o->grid[lower] + vf * (o->grid[lower + 1] - o->grid[lower]);
	const double upper_rate = o->grid[upper] + vf * (o->grid[upper + 1] - o->grid[upper]);
	const double rate = lower_rate + rf * (upper_rate - lower_rate);
	return isfinite(rate) ? (rate > 0.0 ? rate : 0.0) : NAN;
}

/* Total_DM_Scattering_Rate, src/Solar_Model.cpp:305-322 */
static double rate_total(const dms_oracle* o, double r, double v)
{
	if(!isfinite(r) || !isfinite(v))
		return NAN;
	if(r < 0.0)
		r = 0.0;
	if(v < 0.0)
		v = 0.0;
	if(v <= o->grid_vmax)
		return rate_interpolated(o, r, v);
	return rate_computed(o, r, v);
}

/* ------------------------------------------------------------------------------------------
 * Standard Halo Model restated (oracle/shim/obscura/DM_Halo_Models.hpp), km/s units
 */
static double halo_pdf_speed(const dms_oracle* o, double v)
{
	if(v < 0.0 || v > o->vesc_halo + o->vobs)
		return 0.0;
	const double dm = v - o->vobs;
	const double dp = v + o->vobs;
	const double a = exp(-dm * dm / (o->v0 * o->v0));
	const double b = (dp <= o->vesc_halo) ? exp(-dp * dp / (o->v0 * o->v0)) : exp(-o->vesc_halo * o->vesc_halo / (o->v0 * o->v0));
	return v / (o->n_esc * SQRT_PI * o->v0 * o->vobs) * (a - b);
}

static double halo_pdf_velocity(const dms_oracle* o, vec3 vel)
{
	const vec3 w = v_add(vel, o->vel_obs);
	const double w2 = v_dot(w, w);
	if(w2 > o->vesc_halo * o->vesc_halo)
		return 0.0;
	return exp(-w2 / (o->v0 * o->v0)) / (o->n_esc * PI_1_5 * o->v0 * o->v0 * o->v0);
}

static const double GL7_X[7] = {0.0, -0.4058451513773971669066064, 0.4058451513773971669066064, -0.7415311855993944398638648, 0.7415311855993944398638648, -0.9491079123427585245261897, 0.9491079123427585245261897};
static const double GL7_W[7] = {0.4179591836734693877551020, 0.3818300505051189449503698, 0.3818300505051189449503698, 0.2797053914892766679014678, 0.2797053914892766679014678, 0.1294849661688696932706114, 0.1294849661688696932706114};

static double halo_moment(const dms_oracle* o, int power, double a, double b)
{
	const int panels = 256;
	const double h = (b - a) / panels;
	double sum = 0.0;
	for(int p = 0; p < panels; p++)
	{
		const double lo = a + p * h;
		const double mid = lo + 0.5 * h;
		double panel = 0.0;
		for(int k = 0; k < 7; k++)
		{
			const double v = mid + 0.5 * h * GL7_X[k];
			const double f = (power > 0) ? v * halo_pdf_speed(o, v) : ((v > 0.0) ? halo_pdf_speed(o, v) / v : 0.0);
			panel += GL7_W[k] * f;
		}
		sum += 0.5 * h * panel;
	}
	return sum;
}

/* libphysica::Spherical_Coordinates restated (oracle/shim/libphysica/Linear_Algebra.hpp) */
static vec3 spherical_coordinates(double r, double theta, double phi, vec3 axis)
{
	const vec3 e3 = v_div(axis, v_norm(axis));
	const vec3 ref = (fabs(e3.x[2]) < 0.9) ? v3(0.0, 0.0, 1.0) : v3(1.0, 0.0, 0.0);
	const vec3 e1 = v_normalized(v_cross(ref, e3));
	const vec3 e2 = v_normalized(v_cross(e3, e1));
	double st, ct, sp, cp;
	dms_sincos(theta, &st, &ct);
	dms_sincos(phi, &sp, &cp);
	vec3 out;
	for(int i = 0; i < 3; i++) out.x[i] = r * (st * cp * e1.x[i] + st * sp * e2.x[i] + ct * e3.x[i]);
	return out;
}

/* PDF_Initial_Speed, src/Simulation_Utilities.cpp:123-143 */
static double pdf_initial_speed(const dms_oracle* o, double v)
{
	if(v == 0.0)
		return 0.0;
	const double v_esc = solar_vesc(o, DMS_RSUN_KM);
	const double normalization = o->halo_avg_speed + v_esc * v_esc * o->halo_eta0;
	const double speed_pdf = halo_pdf_speed(o, v);
	return (speed_pdf * v + (speed_pdf / v) * v_esc * v_esc) / normalization;
}

/* PDF_Cos_Theta, src/Simulation_Utilities.cpp:146-174 */
static double pdf_cos_theta(const dms_oracle* o, double cos_theta, double v)
{
	const double speed_pdf = halo_pdf_speed(o, v);
	const double normalization = 2.0 * PI * v * v / speed_pdf;
	const vec3 axis = (v_norm(o->vel_obs) > 0.0) ? o->vel_obs : v3(0.0, 0.0, 1.0);
	const vec3 vel = spherical_coordinates(v, dms_acos(cos_theta), 0.0, axis);
	return normalization * halo_pdf_velocity(o, vel);
}

static double clamp_cosine(double c) { return c < -1.0 ? -1.0 : (c > 1.0 ? 1.0 : c); }
static double clamp_unit(double c) { return c < 0.0 ? 0.0 : (c > 1.0 ? 1.0 : c); }

/* Initial_Conditions, src/Simulation_Utilities.cpp:176-249; libphysica::Rejection_Sampling
 * restated in oracle/shim/libphysica/Statistics.hpp (x draw, then y draw, accept y <= pdf(x)) */
static event_t initial_conditions(dms_oracle* o)
{
	const double y_max_speed = DMS_IC_SPEED_YMAX_NATURAL / DMS_C_KMS; /* 1200 (natural) in s/km */
	const double v_max = o->vesc_halo + o->vobs;
	double u;
	for(;;)
	{
		const double x = sample_uniform(o, 0.0, v_max);
		const double y = sample_uniform(o, 0.0, y_max_speed);
		if(y <= pdf_initial_speed(o, x))
		{
			u = x;
			break;
		}
	}
	const double v_sun = v_norm(o->vel_obs);
	const double v_gal = v_max - v_sun;
	double cos_theta_max = (v_sun == 0.0) ? 1.0 : (v_gal * v_gal - v_sun * v_sun - u * u) / (2.0 * u * v_sun);
	if(cos_theta_max > 1.0)
		cos_theta_max = 1.0;
	const double y_max = pdf_cos_theta(o, -1.0, u);
	double cos_theta;
	for(;;)
	{
		const double x = sample_uniform(o, -1.0, cos_theta_max);
		const double y = sample_uniform(o, 0.0, y_max);
		if(y <= pdf_cos_theta(o, x, u))
		{
			cos_theta = x;
			break;
		}
	}
	const double phi = sample_uniform(o, 0.0, 2.0 * PI);
	const vec3 axis = (v_sun > 0.0) ? o->vel_obs : v3(0.0, 0.0, 1.0);
	vec3 velocity = spherical_coordinates(u, dms_acos(clamp_cosine(cos_theta)), phi, axis);
	const double asymptotic_distance = DMS_IC_ASYMPTOTIC_DISTANCE_AU * DMS_AU_KM;
	const double vesc_asymptotic = solar_vesc(o, asymptotic_distance);
	const double v = sqrt(u * u + vesc_asymptotic * vesc_asymptotic);
	velocity = v_scale(v, v_normalized(velocity));
	const double v_esc = solar_vesc(o, DMS_RSUN_KM);
	const double b_max = sqrt(u * u + v_esc * v_esc) / v * DMS_RSUN_KM;
	const vec3 e_z = v_scale(-1.0, v_normalized(velocity));
	const vec3 ref = (fabs(e_z.x[2]) < 0.9) ? v3(0.0, 0.0, 1.0) : v3(1.0, 0.0, 0.0);
	const vec3 e_x = v_normalized(v_cross(ref, e_z));
	const vec3 e_y = v_normalized(v_cross(e_z, e_x));
	const double phi_disk = sample_uniform(o, 0.0, 2.0 * PI);
	const double xi = sample_uniform(o, 0.0, 1.0);
	const double b = sqrt(xi) * b_max;
	event_t e;
	e.time = 0.0;
	double s, c;
	dms_sincos(phi_disk, &s, &c);
	for(int i = 0; i < 3; i++) e.position.x[i] = asymptotic_distance * e_z.x[i] + b * (c * e_x.x[i] + s * e_y.x[i]);
	e.velocity = velocity;
	return e;
}

static int finite_positive(double x) { return isfinite(x) && x > 0.0; }

/* Hyperbolic_Kepler_Shift, src/Simulation_Utilities.cpp:252-321 */
static int hyperbolic_kepler_shift(event_t* e, double R_final)
{
	const double mu = DMS_GMSUN_KM3S2;
	const double R_initial = ev_radius(e);
	const double speed = ev_speed(e);
	if(R_final < DMS_RSUN_KM || R_initial < DMS_RSUN_KM)
		return 0;
	if(!finite_positive(R_final) || !finite_positive(R_initial) || !finite_positive(speed))
		return 0;
	if(fabs(R_final - R_initial) <= DMS_KEPLER_DOMAIN_TOLERANCE * (R_initial > R_final ? R_initial : R_final))
		return 1;
	const double radial_velocity = v_dot(e->position, e->velocity) / R_initial;
	if(!isfinite(radial_velocity) || radial_velocity == 0.0)
		return 0;
	const double radial_direction = (radial_velocity < 0.0) ? -1.0 : 1.0;
	if(radial_direction < 0.0 && R_final > R_initial)
		return 0;
	if(radial_direction > 0.0 && R_final < R_initial)
		return 0;
	const double energy = 0.5 * speed * speed - mu / R_initial;
	if(!finite_positive(energy))
		return 0;
	const vec3 r_hat = v_div(e->position, R_initial);
	const vec3 h_vec = v_cross(e->position, e->velocity);
	const double h = v_norm(h_vec);
	const double h_scale = R_initial * speed;
	if(!isfinite(h) || h <= DMS_KEPLER_DOMAIN_TOLERANCE * h_scale)
	{
		const double final_speed_sqr = 2.0 * (energy + mu / R_final);
		if(!finite_positive(final_speed_sqr))
			return 0;
		e->position = v_scale(R_final, r_hat);
		e->velocity = v_scale(radial_direction * sqrt(final_speed_sqr), r_hat);
		return 1;
	}
	const double p = h * h / mu;
	const vec3 ecc_vec = v_sub(v_div(v_cross(e->velocity, h_vec), mu), r_hat);
	const double ecc = v_norm(ecc_vec);
	if(!finite_positive(p) || !isfinite(ecc) || ecc <= 1.0)
		return 0;
	const double cos_final = (p / R_final - 1.0) / ecc;
	if(!isfinite(cos_final) || cos_final > 1.0 + DMS_KEPLER_DOMAIN_TOLERANCE || cos_final < -1.0 - DMS_KEPLER_DOMAIN_TOLERANCE)
		return 0;
	vec3 axis_x = v_div(ecc_vec, ecc);
	const vec3 axis_z = v_div(h_vec, h);
	vec3 axis_y = v_cross(axis_z, axis_x);
	const double axis_y_norm = v_norm(axis_y);
	if(!finite_positive(axis_y_norm))
		return 0;
	axis_y = v_div(axis_y, axis_y_norm);
	axis_x = v_normalized(v_cross(axis_y, axis_z));
	const double theta_abs = dms_acos(clamp_cosine(cos_final));
	const double theta = radial_direction * theta_abs;
	double st, ct;
	dms_sincos(theta, &st, &ct);
	const double sq = sqrt(mu / p);
	for(int i = 0; i < 3; i++)
	{
		e->position.x[i] = R_final * (ct * axis_x.x[i] + st * axis_y.x[i]);
		e->velocity.x[i] = sq * (-st * axis_x.x[i] + (ecc + ct) * axis_y.x[i]);
	}
	return 1;
}

/* ------------------------------------------------------------------------------------------
 * Free_Particle_Propagator, src/Simulation_Trajectory.cpp:1403-1742
 */
typedef struct
{
	double time, radius, phi, v_radial, angular_momentum;
	vec3 axis_x, axis_y, axis_z;
	int radial_mode;
	double time_step;
} propagator_t;

/* Build_Stable_Orthonormal_Basis, src/Simulation_Trajectory.cpp:130-142 */
static void stable_basis(vec3 axis, vec3* e1, vec3* e2, vec3* e3)
{
	const double n = v_norm(axis);
	*e1 = v_div(axis, n);
	const vec3 ref = (fabs(e1->x[2]) < 0.9) ? v3(0.0, 0.0, 1.0) : v3(1.0, 0.0, 0.0);
	*e2 = v_normalized(v_cross(ref, *e1));
	*e3 = v_normalized(v_cross(*e1, *e2));
}

static void propagator_init(propagator_t* p, const event_t* e)
{
	p->time = e->time;
	p->radius = ev_radius(e);
	p->phi = 0.0;
	p->radial_mode = 0;
	p->time_step = DMS_RK45_DEFAULT_STEP_S;
	const double speed = ev_speed(e);
	const double radius_eps = 1.0e-12;
	const double angular_scale = (p->radius * speed > 1.0) ? p->radius * speed : 1.0;
	const double angular_eps = 1.0e-12 * angular_scale;
	const vec3 L = v_cross(e->position, e->velocity);
	const double L_norm = v_norm(L);
	if(isfinite(p->radius) && p->radius > radius_eps)
	{
		p->axis_x = v_div(e->position, p->radius);
		p->v_radial = v_dot(e->position, e->velocity) / p->radius;
	}
	else if(isfinite(speed) && speed > 0.0)
	{
		p->axis_x = v_div(e->velocity, speed);
		p->v_radial = speed;
		p->radius = 0.0;
		p->radial_mode = 1;
	}
	else
	{
		p->axis_x = v3(1.0, 0.0, 0.0);
		p->v_radial = 0.0;
		p->radius = 0.0;
		p->radial_mode = 1;
	}
	if(!p->radial_mode && isfinite(L_norm) && L_norm > angular_eps)
	{
		p->axis_z = v_div(L, L_norm);
		p->axis_y = v_cross(p->axis_z, p->axis_x);
		const double ny = v_norm(p->axis_y);
		if(isfinite(ny) && ny > 0.0)
		{
			p->axis_y = v_div(p->axis_y, ny);
			p->axis_x = v_normalized(v_cross(p->axis_y, p->axis_z));
			p->angular_momentum = L_norm;
		}
		else
			p->radial_mode = 1;
	}
	else
		p->radial_mode = 1;
	if(p->radial_mode)
	{
		vec3 a = p->axis_x;
		stable_basis(a, &p->axis_x, &p->axis_y, &p->axis_z);
		p->angular_momentum = 0.0;
	}
}

/* dv_dt / dphi_dt, src/Simulation_Trajectory.cpp:1471-1485 */
static double dv_dt(const propagator_t* p, double r, double gm)
{
	if(r < 1.0)
		r = 1.0;
	return p->angular_momentum * p->angular_momentum / r / r / r - gm / r / r;
}

static double dphi_dt(const propagator_t* p, double r)
{
	if(p->radial_mode || p->angular_momentum == 0.0 || r <= 0.0)
		return 0.0;
	return p->angular_momentum / r / r;
}

/* RK45_Sanitized_Time_Step, src/Simulation_Trajectory.cpp:58-63 */
static double sanitized_step(double step)
{
	if(!isfinite(step) || step <= 0.0)
		return DMS_RK45_DEFAULT_STEP_S;
	return step < DMS_RK45_ABS_MAX_STEP_S ? step : DMS_RK45_ABS_MAX_STEP_S;
}

static const double TOL[3] = {DMS_RK45_TOL_R_KM, DMS_RK45_TOL_V_KMS, DMS_RK45_TOL_PHI};

/* RK45_Next_Step_Size, src/Simulation_Trajectory.cpp:477-502 */
static double next_step_size(double current, const double err[3])
{
	for(int i = 0; i < 3; i++)
		if(!isfinite(err[i]))
			return DMS_RK45_MIN_STEP_FACTOR * current;
	double factor = DMS_RK45_MAX_STEP_FACTOR;
	for(int i = 0; i < 3; i++)
	{
		if(err[i] <= 0.0)
			continue;
		const double candidate = 0.84 * dms_pow_quarter(TOL[i] / err[i]);
		if(isfinite(candidate) && candidate < factor)
			factor = candidate;
	}
	if(factor > DMS_RK45_MAX_STEP_FACTOR) factor = DMS_RK45_MAX_STEP_FACTOR;
	if(factor < DMS_RK45_MIN_STEP_FACTOR) factor = DMS_RK45_MIN_STEP_FACTOR;
	return sanitized_step(factor * current);
}

/* Runge_Kutta_45_Step(Solar_Model&), src/Simulation_Trajectory.cpp:1487-1602 */
static int rk45_step(const dms_oracle* o, propagator_t* p)
{
	p->time_step = sanitized_step(p->time_step);
	int inner = 0;
	for(;;)
	{
		inner++;
		DMS_OPS_MARK(0);
		DMS_OPS_PHASE(0);
		const double dt = p->time_step;
		double kr[6], kv[6], kp[6], ri;
		kr[0] = dt * p->v_radial;
		kv[0] = dt * dv_dt(p, p->radius, solar_gm(o, p->radius));
		kp[0] = dt * dphi_dt(p, p->radius);
		ri = p->radius + kr[0] / 4.0;
		kr[1] = dt * (p->v_radial + kv[0] / 4.0);
		kv[1] = dt * dv_dt(p, ri, solar_gm(o, ri));
		ri = p->radius + 3.0 / 32.0 * kr[0] + 9.0 / 32.0 * kr[1];
		kr[2] = dt * (p->v_radial + 3.0 / 32.0 * kv[0] + 9.0 / 32.0 * kv[1]);
		kv[2] = dt * dv_dt(p, ri, solar_gm(o, ri));
		kp[2] = dt * dphi_dt(p, ri);
		ri = p->radius + 1932.0 / 2197.0 * kr[0] - 7200.0 / 2197.0 * kr[1] + 7296.0 / 2197.0 * kr[2];
		kr[3] = dt * (p->v_radial + 1932.0 / 2197.0 * kv[0] - 7200.0 / 2197.0 * kv[1] + 7296.0 / 2197.0 * kv[2]);
		kv[3] = dt * dv_dt(p, ri, solar_gm(o, ri));
		kp[3] = dt * dphi_dt(p, ri);
		ri = p->radius + 439.0 / 216.0 * kr[0] - 8.0 * kr[1] + 3680.0 / 513.0 * kr[2] - 845.0 / 4104.0 * kr[3];
		kr[4] = dt * (p->v_radial + 439.0 / 216.0 * kv[0] - 8.0 * kv[1] + 3680.0 / 513.0 * kv[2] - 845.0 / 4104.0 * kv[3]);
		kv[4] = dt * dv_dt(p, ri, solar_gm(o, ri));
		kp[4] = dt * dphi_dt(p, ri);
		ri = p->radius - 8.0 / 27.0 * kr[0] + 2.0 * kr[1] - 3544.0 / 2565.0 * kr[2] + 1859.0 / 4104.0 * kr[3] - 11.0 / 40.0 * kr[4];
		kr[5] = dt * (p->v_radial - 8.0 / 27.0 * kv[0] + 2.0 * kv[1] - 3544.0 / 2565.0 * kv[2] + 1859.0 / 4104.0 * kv[3] - 11.0 / 40.0 * kv[4]);
		kv[5] = dt * dv_dt(p, ri, solar_gm(o, ri));
		kp[5] = dt * dphi_dt(p, ri);
		const double r4 = p->radius + 25.0 / 216.0 * kr[0] + 1408.0 / 2565.0 * kr[2] + 2197.0 / 4104.0 * kr[3] - 1.0 / 5.0 * kr[4];
		const double v4 = p->v_radial + 25.0 / 216.0 * kv[0] + 1408.0 / 2565.0 * kv[2] + 2197.0 / 4104.0 * kv[3] - 1.0 / 5.0 * kv[4];
		const double p4 = p->phi + 25.0 / 216.0 * kp[0] + 1408.0 / 2565.0 * kp[2] + 2197.0 / 4104.0 * kp[3] - 1.0 / 5.0 * kp[4];
		const double r5 = p->radius + 16.0 / 135.0 * kr[0] + 6656.0 / 12825.0 * kr[2] + 28561.0 / 56430.0 * kr[3] - 9.0 / 50.0 * kr[4] + 2.0 / 55.0 * kr[5];
		const double v5 = p->v_radial + 16.0 / 135.0 * kv[0] + 6656.0 / 12825.0 * kv[2] + 28561.0 / 56430.0 * kv[3] - 9.0 / 50.0 * kv[4] + 2.0 / 55.0 * kv[5];
		const double p5 = p->phi + 16.0 / 135.0 * kp[0] + 6656.0 / 12825.0 * kp[2] + 28561.0 / 56430.0 * kp[3] - 9.0 / 50.0 * kp[4] + 2.0 / 55.0 * kp[5];
		const double err[3] = {fabs(r5 - r4), fabs(v5 - v4), fabs(p5 - p4)};
		const double new_step = next_step_size(dt, err);
		int within = 1;
		for(int i = 0; i < 3; i++)
			if(!isfinite(err[i]) || err[i] > TOL[i])
				within = 0;
		if(within)
		{
			p->time = p->time + dt;
			p->radius = r4 < 0.0 ? 0.0 : r4;
			p->v_radial = v4;
			p->phi = p4;
			p->time_step = new_step;
			return 1;
		}
		if(new_step < DMS_RK45_ABS_MIN_STEP_S || inner >= DMS_RK45_MAX_INNER_RETRIES)
		{
			const int ok = isfinite(r4) && isfinite(v4) && isfinite(p4);
			p->time = p->time + DMS_RK45_ABS_MIN_STEP_S;
			if(ok)
			{
				p->radius = r4 < 0.0 ? 0.0 : r4;
				p->v_radial = v4;
				p->phi = p4;
			}
			p->time_step = DMS_RK45_ABS_MIN_STEP_S;
			return 0;
		}
		p->time_step = new_step;
	}
}

static double prop_radius(const propagator_t* p) { return p->radius < 0.0 ? 0.0 : p->radius; }

static double prop_speed(const propagator_t* p)
{
	const double r = p->radius < 0.0 ? 0.0 : p->radius;
	if(r == 0 || p->angular_momentum == 0)
		return fabs(p->v_radial);
	return sqrt(p->v_radial * p->v_radial + p->angular_momentum * p->angular_momentum / r / r);
}

/* Event_In_3D, src/Simulation_Trajectory.cpp:1715-1742 */
static event_t prop_event(const propagator_t* p)
{
	const double safe = (isfinite(p->radius) && p->radius > 0.0) ? p->radius : 0.0;
	event_t e;
	e.time = p->time;
	if(p->radial_mode || p->angular_momentum == 0.0 || safe == 0.0)
	{
		for(int i = 0; i < 3; i++)
		{
			e.position.x[i] = safe * p->axis_x.x[i];
			e.velocity.x[i] = p->v_radial * p->axis_x.x[i];
		}
		return e;
	}
	double sp, cp;
	dms_sincos(p->phi, &sp, &cp);
	const double vt = p->angular_momentum / safe;
	const double vx = p->v_radial * cp - vt * sp;
	const double vy = p->v_radial * sp + vt * cp;
	for(int i = 0; i < 3; i++)
	{
		e.position.x[i] = safe * (cp * p->axis_x.x[i] + sp * p->axis_y.x[i]);
		e.velocity.x[i] = vx * p->axis_x.x[i] + vy * p->axis_y.x[i];
	}
	return e;
}

/* ------------------------------------------------------------------------------------------
 * Geometry helpers, src/Simulation_Trajectory.cpp:65-325
 */
static double step_cap(double radius, double speed, double max_distance)
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

static int outward_escaping(const dms_oracle* o, const event_t* e, double boundary)
{
	const double r = ev_radius(e);
	if(r < boundary)
		return 0;
	const double vr = (r > 0.0) ? v_dot(e->position, e->velocity) / r : 0.0;
	return vr > 0.0 && ev_speed(e) > solar_vesc(o, r);
}

static double radial_velocity(const event_t* e)
{
	const double r = ev_radius(e);
	if(r <= 0.0)
		return 0.0;
	return v_dot(e->position, e->velocity) / r;
}

/* Bound_Kepler_Return_At_Same_Radius, src/Simulation_Trajectory.cpp:152-201 */
static int bound_kepler_return(const event_t* out, event_t* in)
{
	const double radius = ev_radius(out);
	const double speed = ev_speed(out);
	const double vr = radial_velocity(out);
	if(!isfinite(radius) || !isfinite(speed) || !isfinite(vr) || radius <= DMS_RSUN_KM || speed <= 0.0 || vr <= 0.0)
		return 0;
	const double mu = DMS_GMSUN_KM3S2;
	const double E = 0.5 * speed * speed - mu / radius;
	if(!isfinite(E) || E >= 0.0)
		return 0;
	const double J = v_norm(v_cross(out->position, out->velocity));
	if(!isfinite(J))
		return 0;
	const double a = -mu / (2.0 * E);
	if(!isfinite(a) || a <= 0.0)
		return 0;
	double e2 = 1.0 + 2.0 * E * J * J / (mu * mu);
	if(!isfinite(e2) || e2 < 0.0)
		return 0;
	e2 = e2 > 0.0 ? e2 : 0.0;
	const double ecc = sqrt(e2);
	if(ecc <= 1.0e-14 || ecc >= 1.0)
		return 0;
	const double cosE = clamp_cosine((1.0 - radius / a) / ecc);
	const double Eanom = dms_acos(cosE);
	const double one_minus = 1.0 - cosE * cosE;
	const double sinE = sqrt(one_minus > 0.0 ? one_minus : 0.0);
	const double n = sqrt(mu / (a * a * a));
	if(!isfinite(n) || n <= 0.0)
		return 0;
	const double T = (2.0 * PI - 2.0 * Eanom + 2.0 * ecc * sinE) / n;
	if(!isfinite(T) || T <= 0.0)
		return 0;
	const vec3 rhat = v_div(out->position, radius);
	*in = *out;
	in->time += T;
	in->velocity = v_sub(out->velocity, v_scale(2.0 * vr, rhat));
	return in->time > out->time && isfinite(ev_speed(in));
}

/* Interpolate_Event, src/Simulation_Trajectory.cpp:203-216 */
static event_t interpolate_event(const event_t* a, const event_t* b, double f)
{
	f = clamp_unit(f);
	event_t e;
	for(int i = 0; i < 3; i++)
	{
		e.position.x[i] = a->position.x[i] + f * (b->position.x[i] - a->position.x[i]);
		e.velocity.x[i] = a->velocity.x[i] + f * (b->velocity.x[i] - a->velocity.x[i]);
	}
	e.time = a->time + f * (b->time - a->time);
	return e;
}

static double radius_at_fraction(const event_t* a, const event_t* b, double f)
{
	f = clamp_unit(f);
	double r2 = 0.0;
	for(int i = 0; i < 3; i++)
	{
		const double x = a->position.x[i] + f * (b->position.x[i] - a->position.x[i]);
		r2 += x * x;
	}
	return sqrt(r2 > 0.0 ? r2 : 0.0);
}

static int surface_crossings(const event_t* a, const event_t* b, double* first, double* second)
{
	double qa = 0.0, qb = 0.0, qc = -DMS_RSUN_KM * DMS_RSUN_KM;
	for(int i = 0; i < 3; i++)
	{
		const double d = b->position.x[i] - a->position.x[i];
		qa += d * d;
		qb += 2.0 * a->position.x[i] * d;
		qc += a->position.x[i] * a->position.x[i];
	}
	if(qa <= 0.0)
		return 0;
	const double disc = qb * qb - 4.0 * qa * qc;
	if(!isfinite(disc) || disc < 0.0)
		return 0;
	const double sq = sqrt(disc > 0.0 ? disc : 0.0);
	*first = (-qb - sq) / (2.0 * qa);
	*second = (-qb + sq) / (2.0 * qa);
	if(*first > *second)
	{
		const double t = *first;
		*first = *second;
		*second = t;
	}
	return 1;
}

static int in_unit(double f) { return f >= -1.0e-12 && f <= 1.0 + 1.0e-12; }

static double find_crossing(const event_t* a, const event_t* b, double lower, double upper)
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

/* Solar_Interior_Fraction_Interval, src/Simulation_Trajectory.cpp:282-325 */
static int interior_interval(const event_t* a, const event_t* b, double ra, double rb, double* start, double* end)
{
	const int a_in = ra < DMS_RSUN_KM, b_in = rb < DMS_RSUN_KM;
	double c1 = 0.0, c2 = 0.0;
	const int has = surface_crossings(a, b, &c1, &c2);
	if(a_in && b_in)
	{
		*start = 0.0;
		*end = 1.0;
		return 1;
	}
	if(!a_in && b_in)
	{
		if(has && in_unit(c1))
			*start = clamp_unit(c1);
		else if(has && in_unit(c2))
			*start = clamp_unit(c2);
		else
			*start = find_crossing(a, b, 0.0, 1.0);
		*end = 1.0;
		return *end > *start;
	}
	if(a_in && !b_in)
	{
		*start = 0.0;
		if(has && in_unit(c2))
			*end = clamp_unit(c2);
		else if(has && in_unit(c1))
			*end = clamp_unit(c1);
		else
			*end = find_crossing(a, b, 0.0, 1.0);
		return *end > *start;
	}
	if(has && in_unit(c1) && in_unit(c2))
	{
		*start = clamp_unit(c1);
		*end = clamp_unit(c2);
		return *end > *start;
	}
	return 0;
}

/* Scattering_Rate_At_Fraction, src/Simulation_Trajectory.cpp:327-345 */
static double rate_at_fraction(const dms_oracle* o, const event_t* a, const event_t* b, double f)
{
	f = clamp_unit(f);
	double r2 = 0.0, v2 = 0.0;
	for(int i = 0; i < 3; i++)
	{
		const double x = a->position.x[i] + f * (b->position.x[i] - a->position.x[i]);
		const double v = a->velocity.x[i] + f * (b->velocity.x[i] - a->velocity.x[i]);
		r2 += x * x;
		v2 += v * v;
	}
	const double r = sqrt(r2 > 0.0 ? r2 : 0.0);
	if(r >= DMS_RSUN_KM)
		return 0.0;
	return rate_total(o, r, sqrt(v2 > 0.0 ? v2 : 0.0));
}

typedef struct
{
	double start, end, rate_start, rate_end;
} od_piece;

/* Build_Optical_Depth_Pieces, src/Simulation_Trajectory.cpp:347-414 */
static int optical_depth_pieces(const dms_oracle* o, const event_t* a, const event_t* b, double s0, double s1, double dt,
                                int use_cached, double cached, int requested, od_piece* pieces, int* count, double* tau2,
                                double* tau4, int* invalid)
{
	*count = 0;
	*tau2 = 0.0;
	*tau4 = 0.0;
	*invalid = 0;
	if(!(s1 > s0) || dt <= 0.0)
		return 0;
	if(requested > DMS_MAX_OPTICAL_DEPTH_PIECES) requested = DMS_MAX_OPTICAL_DEPTH_PIECES;
	if(requested < 1) requested = 1;
	const double span = s1 - s0;
	double fr[DMS_MAX_OPTICAL_DEPTH_PIECES + 1], rt[DMS_MAX_OPTICAL_DEPTH_PIECES + 1];
	for(int i = 0; i <= requested; i++) fr[i] = s0 + (double)i / (double)requested * span;
	for(int i = 0; i <= requested; i++)
	{
		rt[i] = (i == 0 && use_cached) ? cached : rate_at_fraction(o, a, b, fr[i]);
		if(!isfinite(rt[i]) || rt[i] < 0.0)
		{
			*invalid = 1;
			return 1;
		}
	}
#define TRAP(i0, i1) (0.5 * (rt[i0] + rt[i1]) * (dt * (fr[i1] - fr[i0])))
	if(requested >= 4)
		*tau2 = TRAP(0, 2) + TRAP(2, 4);
	else
		for(int i = 0; i < requested; i++) *tau2 += TRAP(i, i + 1);
	for(int i = 0; i < requested; i++)
		if(fr[i + 1] > fr[i])
		{
			pieces[*count].start = fr[i];
			pieces[*count].end = fr[i + 1];
			pieces[*count].rate_start = rt[i];
			pieces[*count].rate_end = rt[i + 1];
			(*count)++;
			*tau4 += TRAP(i, i + 1);
		}
#undef TRAP
	return *count > 0;
}

/* Solve_Linear_Rate_Optical_Depth_Fraction, src/Simulation_Trajectory.cpp:416-464 */
static double solve_linear_rate(double r0, double r1, double dt, double target)
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
		const double roots[2] = {(-b + sq) / (2.0 * a), (-b - sq) / (2.0 * a)};
		for(int k = 0; k < 2; k++)
			if(isfinite(roots[k]) && roots[k] >= 0.0 && roots[k] <= 1.0)
				return clamp_unit(roots[k]);
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

/* ------------------------------------------------------------------------------------------
 * Trajectory simulator state, include/Simulation_Trajectory.hpp:53-180
 */
typedef struct
{
	int capture_mode;
	uint64_t max_free_steps, max_scatterings;
	double max_distance;
	/* TrajectoryBincount */
	double* dt_hist;
	double* v2dt_hist;
	int is_captured;
	double t_capture, t_last_bound, t_final_unbinding, t_boundary_escape, t_termination;
	int event_observed, boundary_escape_observed, survival_valid, invalid_escape;
	double max_drift_eV, max_drift_rel;
	/* simulator members */
	double prev_time, prev_r, prev_v2, prev_dt;
	double previous_capture_energy, free_flight_reference_energy;
	int bound_state;
} sim_t;

/* Capture_Energy_eV, src/Simulation_Trajectory.cpp:682-687 */
static double capture_energy_eV(const dms_oracle* o, double r, double v)
{
	const double vesc = solar_vesc(o, r);
	const double E = 0.5 * o->m_dm * ((v * v - vesc * vesc) / (DMS_C_KMS * DMS_C_KMS));
	return E / 1.0e-9;
}

/* Accumulate_Bincount_Step, src/Simulation_Trajectory.cpp:640-669 */
static void accumulate_bincount(sim_t* s, double r, double v2, double dt)
{
	if(!isfinite(dt) || dt <= 0.0)
		return;
	int bin = -1;
	if(isfinite(r) && r >= 0.0 && r < DMS_BIN_MAX_KM)
	{
		bin = (int)(r / DMS_BIN_WIDTH_KM);
		if(bin < 0) bin = 0;
		if(bin >= DMS_NUM_BINS) bin = -1;
	}
	if(bin >= 0)
	{
		s->dt_hist[bin] += dt;
		s->v2dt_hist[bin] += v2 * dt;
	}
}

/* Reset_Bincount_Anchor, src/Simulation_Trajectory.cpp:671-680 */
static void reset_anchor(sim_t* s, const event_t* e)
{
	if(s->capture_mode)
		return;
	s->prev_time = e->time;
	s->prev_r = ev_radius(e);
	const double v = ev_speed(e);
	s->prev_v2 = v * v;
}

/* Update_Capture_State, src/Simulation_Trajectory.cpp:689-760 */
static int update_capture_state(const dms_oracle* o, sim_t* s, double r, double v, double t, int allow_new)
{
	if(s->capture_mode && !allow_new && !s->is_captured)
		return 0;
	const double E = capture_energy_eV(o, r, v);
	s->previous_capture_energy = E;
	const int negative = E < 0.0;
	if(!allow_new)
	{
		if(s->is_captured && isfinite(s->free_flight_reference_energy))
		{
			const double drift = fabs(E - s->free_flight_reference_energy);
			if(isfinite(drift) && drift > s->max_drift_eV)
				s->max_drift_eV = drift;
			const double ref = fabs(s->free_flight_reference_energy);
			const double scale = ref > DMS_FREE_ENERGY_DRIFT_REL_E_SCALE_EV ? ref : DMS_FREE_ENERGY_DRIFT_REL_E_SCALE_EV;
			const double rel = drift / scale;
			if(isfinite(rel) && rel > s->max_drift_rel)
				s->max_drift_rel = rel;
		}
		if(s->bound_state && s->is_captured)
			s->t_last_bound = t;
		return 0;
	}
	const int was_bound = s->bound_state;
	s->bound_state = negative;
	s->free_flight_reference_energy = E;
	if(negative)
	{
		if(!s->is_captured)
		{
			s->is_captured = 1;
			s->t_capture = t;
			s->t_last_bound = t;
		}
		else if(!was_bound)
			s->t_final_unbinding = NAN;
		s->t_last_bound = t;
		return 1;
	}
	if(was_bound && s->is_captured)
		s->t_final_unbinding = t;
	return 0;
}

static int uncaptured_bound(const dms_oracle* o, const sim_t* s, const event_t* e)
{
	if(s->is_captured)
		return 0;
	const double E = capture_energy_eV(o, ev_radius(e), ev_speed(e));
	if(isfinite(E) && E >= 0.0)
		return 0;
	return 1;
}

/* commit_accepted_event, src/Simulation_Trajectory.cpp:842-874 */
static int commit_event(const dms_oracle* o, sim_t* s, const event_t* local, double origin)
{
	event_t abs_e = *local;
	abs_e.time += origin;
	const double t_now = local->time;
	if(!s->capture_mode)
	{
		const double r_now = ev_radius(local);
		const double v_now = ev_speed(local);
		const double v2 = v_now * v_now;
		if(s->prev_time >= 0.0)
		{
			const double dt = t_now - s->prev_time;
			accumulate_bincount(s, s->prev_r, s->prev_v2, dt);
			s->prev_dt = dt;
		}
		s->prev_time = t_now;
		s->prev_r = r_now;
		s->prev_v2 = v2;
	}
	return update_capture_state(o, s, ev_radius(&abs_e), ev_speed(&abs_e), abs_e.time, 0);
}

/* Propagate_Freely, src/Simulation_Trajectory.cpp:762-1119 */
static int propagate_freely(dms_oracle* o, sim_t* s, event_t* current)
{
	DMS_OPS_PHASE(2);
	if(outward_escaping(o, current, s->max_distance))
		return DMS_REASON_OUTWARD_ESCAPE;
	if(uncaptured_bound(o, s, current))
		return DMS_REASON_NUMERICAL_FAILURE;
	double origin = current->time;
	event_t local0 = *current;
	local0.time = 0.0;
	propagator_t prop;
	propagator_init(&prop, &local0);
	double minus_log_xi = -dms_log(positive_unit_uniform(o));
	int outcome = DMS_REASON_MAX_FREE_STEPS;
	uint64_t steps = 0;
	unsigned int retries = 0;
	const int fast = s->capture_mode;
	const double tau_limit = fast ? DMS_CAPTURE_MAX_OPTICAL_DEPTH_STEP : DMS_MAX_OPTICAL_DEPTH_STEP;
	const int pieces_target = fast ? DMS_CAPTURE_OPTICAL_DEPTH_PIECES : DMS_MAX_OPTICAL_DEPTH_PIECES;
	if(!s->capture_mode && s->prev_time >= 0.0)
		s->prev_time = 0.0;

	DMS_OPS_PHASE(1);
	while(steps < s->max_free_steps && outcome == DMS_REASON_MAX_FREE_STEPS)
	{
		const event_t before = prop_event(&prop);
		const double r_before = prop_radius(&prop);
		const double v_before = prop_speed(&prop);
		double rate_before = 0.0;
		if(r_before >= DMS_RSUN_KM)
		{
			const double cap = step_cap(r_before, v_before, s->max_distance);
			const double ts = sanitized_step(prop.time_step);
			prop.time_step = ts < cap ? ts : cap;
			const double vr = (r_before > 0.0) ? v_dot(before.position, before.velocity) / r_before : 0.0;
			if(r_before > DMS_RSUN_KM && vr < 0.0)
			{
				const double est = (r_before - DMS_RSUN_KM) / (-vr);
				if(isfinite(est) && est > 0.0)
				{
					const double lim = est > DMS_RK45_ABS_MIN_STEP_S ? est : DMS_RK45_ABS_MIN_STEP_S;
					if(lim < prop.time_step) prop.time_step = lim;
				}
			}
		}
		else
		{
			prop.time_step = sanitized_step(prop.time_step);
			rate_before = rate_total(o, r_before, v_before);
			if(!isfinite(rate_before) || rate_before < 0.0)
			{
				*current = prop_event(&prop);
				current->time += origin;
				return DMS_REASON_NUMERICAL_FAILURE;
			}
			if(rate_before > 0.0 && tau_limit / rate_before < prop.time_step)
				prop.time_step = tau_limit / rate_before;
		}
		const propagator_t prop_before = prop;
		const double t_before = prop.time;
		const int ok = rk45_step(o, &prop);
		DMS_OPS_PHASE(1);
		const double actual_dt = prop.time - t_before;
		const double r_after = prop_radius(&prop);
		const double v_after = prop_speed(&prop);
		const event_t after = prop_event(&prop);
		if(!ok)
		{
			*current = after;
			current->time += origin;
			return DMS_REASON_NUMERICAL_FAILURE;
		}
		if(!isfinite(r_after) || !isfinite(v_after) || !isfinite(actual_dt) || actual_dt <= 0.0)
		{
			*current = after;
			current->time += origin;
			return DMS_REASON_NON_FINITE_STATE;
		}
		if(v_after > DMS_V_MAX_C * DMS_C_KMS)
		{
			*current = after;
			current->time += origin;
			return DMS_REASON_SPEED_LIMIT;
		}
		int scattering = 0, reflection = 0;
		event_t accepted = after;
		double s0 = 0.0, s1 = 0.0;
		if(interior_interval(&before, &after, r_before, r_after, &s0, &s1))
		{
			if(r_after < DMS_RSUN_KM && v_after < 0.0)
				break;
			od_piece pieces[DMS_MAX_OPTICAL_DEPTH_PIECES];
			int count = 0, invalid = 0;
			double tau2 = 0.0, dtau = 0.0;
			const int use_cached = r_before < DMS_RSUN_KM && s0 <= 1.0e-12;
			optical_depth_pieces(o, &before, &after, s0, s1, actual_dt, use_cached, rate_before, pieces_target, pieces, &count, &tau2, &dtau, &invalid);
			if(invalid || !isfinite(dtau) || dtau < 0.0)
			{
				*current = after;
				current->time += origin;
				return DMS_REASON_NUMERICAL_FAILURE;
			}
			const double scale = dtau > DMS_OPTICAL_DEPTH_ABS_TOL ? dtau : DMS_OPTICAL_DEPTH_ABS_TOL;
			const double rel = fabs(dtau - tau2) / scale;
			const int reject_depth = dtau > tau_limit;
			const int reject_acc = !fast && rel > DMS_OPTICAL_DEPTH_REL_TOL;
			if(reject_depth || reject_acc)
			{
				retries++;
				if(retries > DMS_MAX_OPTICAL_DEPTH_RETRIES)
				{
					*current = before;
					current->time += origin;
					return DMS_REASON_NUMERICAL_FAILURE;
				}
				prop = prop_before;
				double factor = DMS_RK45_MAX_STEP_FACTOR;
				if(dtau > tau_limit && dtau > 0.0 && 0.8 * tau_limit / dtau < factor)
					factor = 0.8 * tau_limit / dtau;
				if(reject_acc && rel > 0.0 && 0.8 * sqrt(DMS_OPTICAL_DEPTH_REL_TOL / rel) < factor)
					factor = 0.8 * sqrt(DMS_OPTICAL_DEPTH_REL_TOL / rel);
				if(factor > 1.0) factor = 1.0;
				if(factor < DMS_RK45_MIN_STEP_FACTOR) factor = DMS_RK45_MIN_STEP_FACTOR;
				prop.time_step = sanitized_step(factor * actual_dt);
				continue;
			}
			if(dtau >= minus_log_xi)
			{
				double remaining = minus_log_xi;
				for(int k = 0; k < count; k++)
				{
					const double pdt = actual_dt * (pieces[k].end - pieces[k].start);
					const double ptau = 0.5 * (pieces[k].rate_start + pieces[k].rate_end) * pdt;
					if(ptau >= remaining)
					{
						const double lf = solve_linear_rate(pieces[k].rate_start, pieces[k].rate_end, pdt, remaining);
						const double f = pieces[k].start + lf * (pieces[k].end - pieces[k].start);
						accepted = interpolate_event(&before, &after, f);
						scattering = 1;
						outcome = DMS_REASON_SCATTER;
						break;
					}
					remaining -= ptau;
				}
				if(!scattering)
				{
					accepted = interpolate_event(&before, &after, s1);
					scattering = 1;
					outcome = DMS_REASON_SCATTER;
				}
			}
			else
				minus_log_xi -= dtau;
		}
		if(!scattering)
		{
			event_t boundary_ev = after;
			double r_b = r_after, v_b = v_after;
			if(r_before < s->max_distance && r_after >= s->max_distance && r_after > r_before)
			{
				const double f = (s->max_distance - r_before) / (r_after - r_before);
				boundary_ev = interpolate_event(&before, &after, f);
				r_b = ev_radius(&boundary_ev);
				v_b = ev_speed(&boundary_ev);
			}
			if(r_b >= s->max_distance && r_b >= r_before && v_b > solar_vesc(o, r_b))
			{
				accepted = boundary_ev;
				reflection = 1;
				outcome = DMS_REASON_OUTWARD_ESCAPE;
			}
			else if(r_b >= s->max_distance && r_b >= r_before)
			{
				event_t abs_b = boundary_ev;
				abs_b.time += origin;
				if(uncaptured_bound(o, s, &abs_b))
				{
					*current = abs_b;
					return DMS_REASON_NUMERICAL_FAILURE;
				}
				event_t inbound;
				if(bound_kepler_return(&boundary_ev, &inbound))
				{
					steps++;
					retries = 0;
					DMS_OPS_MARK(1);
					commit_event(o, s, &boundary_ev, origin);
					*current = inbound;
					current->time += origin;
					/* reset_propagator_at_absolute_event, :814-822 */
					origin = current->time;
					event_t loc = *current;
					loc.time = 0.0;
					propagator_init(&prop, &loc);
					if(!s->capture_mode && s->prev_time >= 0.0)
						s->prev_time = 0.0;
					continue;
				}
			}
		}
		steps++;
		retries = 0;
		DMS_OPS_MARK(1);
		const int captured_now = commit_event(o, s, &accepted, origin);
		*current = accepted;
		current->time += origin;
		if(uncaptured_bound(o, s, current))
			return DMS_REASON_NUMERICAL_FAILURE;
		if(s->capture_mode && captured_now)
			return DMS_REASON_CAPTURE_MODE;
		if(reflection || scattering)
			break;
	}
	return outcome;
}

/* Unit_Vector_At_Angle_From_Axis, src/Simulation_Trajectory.cpp:109-128; returns 0 on the
 * reference's runtime_error conditions */
static int unit_vector_at_angle(double cos_theta, double phi, vec3 axis, vec3* out)
{
	if(!isfinite(cos_theta) || cos_theta < -1.0 - 1.0e-12 || cos_theta > 1.0 + 1.0e-12 || !isfinite(phi))
		return 0;
	const double n = v_norm(axis);
	if(!isfinite(n) || n <= 0.0)
		return 0;
	const vec3 e3 = v_div(axis, n);
	const vec3 ref = (fabs(e3.x[2]) < 0.9) ? v3(0.0, 0.0, 1.0) : v3(1.0, 0.0, 0.0);
	const vec3 e1 = v_normalized(v_cross(ref, e3));
	const vec3 e2 = v_normalized(v_cross(e3, e1));
	cos_theta = clamp_cosine(cos_theta);
	const double st2 = 1.0 - cos_theta * cos_theta;
	const double st = sqrt(st2 > 0.0 ? st2 : 0.0);
	double sp, cp;
	dms_sincos(phi, &sp, &cp);
	for(int i = 0; i < 3; i++) out->x[i] = cos_theta * e3.x[i] + st * cp * e1.x[i] + st * sp * e2.x[i];
	return 1;
}

/* Scatter = Sample_Target + Sample_Target_Velocity + angle + New_DM_Velocity,
 * src/Simulation_Trajectory.cpp:1122-1269.  Returns 0 where the reference throws. */
static int scatter(dms_oracle* o, event_t* e)
{
	const double r = ev_radius(e);
	const double v = ev_speed(e);
	/* Sample_Target :1122-1158 */
	if(r > DMS_RSUN_KM)
		return 0;
	double rates[DMS_NUM_TARGETS];
	for(int t = 0; t < DMS_NUM_TARGETS; t++)
	{
		rates[t] = rate_nucleus(o, r, v, t);
		if(!isfinite(rates[t]) || rates[t] < 0.0)
			return 0;
	}
	const double re = rate_electron(o, r, v);
	if(!isfinite(re) || re < 0.0)
		return 0;
	double total = re;
	for(int t = 0; t < DMS_NUM_TARGETS; t++) total += rates[t];
	if(!isfinite(total) || total <= 0.0)
		return 0;
	const double xi = sample_uniform(o, 0.0, 1.0);
	int target = -2;
	double sum = re / total;
	if(sum > xi)
		target = -1;
	else
		for(int t = 0; t < DMS_NUM_TARGETS; t++)
		{
			sum += rates[t] / total;
			if(sum > xi || t == DMS_NUM_TARGETS - 1)
			{
				target = t;
				break;
			}
		}
	const double m_target = (target == -1) ? DMS_MELECTRON_GEV : o->target_mass_gev[target];
	/* Sample_Target_Velocity :1160-1226 (Romano & Walsh free-gas rejection) */
	const double T = solar_temperature(o, r);
	if(!isfinite(T) || T <= 0.0 || !isfinite(m_target) || m_target <= 0.0)
		return 0;
	const double kappa = sqrt(m_target / 2.0 / T) / DMS_C_KMS;
	const double vdm = v_norm(e->velocity);
	if(!isfinite(kappa) || kappa <= 0.0 || !isfinite(vdm) || vdm <= 0.0)
		return 0;
	const double y = kappa * vdm;
	double x = y, mu = 1.0;
	unsigned long attempts = 0;
	for(;;)
	{
		const double x2 = x * x, y2 = y * y;
		const double raw = x2 + y2 - 2.0 * x * y * mu;
		const double den = x + y;
		const double ax = fabs(x * y);
		const double rs = (1.0 > x2 + y2 + 2.0 * ax) ? 1.0 : x2 + y2 + 2.0 * ax;
		if(!isfinite(x) || x < 0.0 || !isfinite(y) || y <= 0.0 || !isfinite(mu) || mu < -1.0 || mu > 1.0 || !isfinite(raw) ||
		   raw < -1.0e-12 * rs || !isfinite(den) || den <= 0.0)
			return 0;
		const double rel2 = raw > 0.0 ? raw : 0.0;
		const double ratio = sqrt(rel2) / den;
		if(!isfinite(ratio) || ratio < 0.0 || ratio > 1.0 + 1.0e-12)
			return 0;
		const double accept = ratio < 1.0 ? ratio : 1.0;
		if(!(accept < sample_uniform(o, 0.0, 1.0)))
			break;
		attempts++;
		if(attempts > DMS_TARGET_VELOCITY_MAX_REJECTIONS)
			return 0;
		mu = sample_uniform(o, -1.0, 1.0);
		const double xi1 = sample_uniform(o, 0.0, 1.0);
		if(xi1 < 2.0 / (SQRT_PI * y + 2.0))
		{
			const double xi2 = positive_unit_uniform(o);
			const double xi3 = positive_unit_uniform(o);
			const double z = -dms_log(xi2) - dms_log(xi3);
			x = sqrt(z);
		}
		else
		{
			const double xi2 = positive_unit_uniform(o);
			const double xi3 = sample_uniform(o, 0.0, 1.0);
			const double xi4 = positive_unit_uniform(o);
			const double c = dms_cos(PI / 2.0 * xi3);
			const double z = -dms_log(xi2) - (c * c) * dms_log(xi4);
			x = sqrt(z);
		}
	}
	const double vT = x / kappa;
	const double phi_t = sample_uniform(o, 0.0, 2.0 * PI);
	vec3 unit_t;
	if(!unit_vector_at_angle(mu, phi_t, e->velocity, &unit_t))
		return 0;
	const vec3 vel_t = v_scale(vT, unit_t);
	if(!isfinite(v_norm(vel_t)))
		return 0;
	/* scattering angle, one draw: isotropic for the contact interactions (SI,
	 * oracle/shim/obscura/DM_Particle.hpp; dark photon "Contact", 2 xi - 1), or the General
	 * form factor's closed form (Sample_Scattering_Angle_*, src/Dark_Photon.cpp:286-325) */
	if(o->trace != NULL && o->trace_length < o->trace_capacity)
	{
		o->trace[3 * o->trace_length + 0] = r;
		o->trace[3 * o->trace_length + 1] = v;
		o->trace[3 * o->trace_length + 2] = (double)o->draw_index;
	}
	if(o->trace != NULL)
		o->trace_length++;
	double cos_alpha;
	if(o->interaction == DMS_INTERACTION_DARK_PHOTON_GENERAL)
	{
		const double xi = sample_uniform(o, 0.0, 1.0);
		const double q2 = o->q2c[target == -1 ? DMS_NUM_TARGETS : target] * (vdm * vdm);
		cos_alpha = (o->ff_m2 * (2.0 * xi - 1.0) + q2 * xi) / (o->ff_m2 + q2 * xi);
	}
	else
		cos_alpha = sample_uniform(o, -1.0, 1.0);
	/* New_DM_Velocity :1228-1247 */
	if(!isfinite(cos_alpha) || cos_alpha < -1.0 - 1.0e-12 || cos_alpha > 1.0 + 1.0e-12 || !isfinite(o->m_dm) || o->m_dm <= 0.0 ||
	   !isfinite(v_norm(e->velocity)) || !isfinite(v_norm(vel_t)))
		return 0;
	const double ca = clamp_cosine(cos_alpha);
	const double phi_n = sample_uniform(o, 0.0, 2.0 * PI);
	vec3 n;
	if(!unit_vector_at_angle(ca, phi_n, e->velocity, &n))
		return 0;
	const double rel_speed = v_norm(v_sub(vel_t, e->velocity));
	const double mt = m_target, md = o->m_dm;
	const double sc = mt * rel_speed / (mt + md);
	vec3 out;
	for(int i = 0; i < 3; i++) out.x[i] = sc * n.x[i] + (md * e->velocity.x[i] + mt * vel_t.x[i]) / (mt + md);
	if(!isfinite(v_norm(out)))
		return 0;
	e->velocity = out;
	return 1;
}

/* Simulate, src/Simulation_Trajectory.cpp:1276-1400 */
static void simulate(dms_oracle* o, sim_t* s, const event_t* ic, dms_traj_record* rec)
{
	event_t cur = *ic;
	uint64_t nscat = 0;
	memset(s->dt_hist, 0, DMS_NUM_BINS * sizeof(double));
	memset(s->v2dt_hist, 0, DMS_NUM_BINS * sizeof(double));
	s->is_captured = 0;
	s->t_capture = -1.0;
	s->t_last_bound = -1.0;
	s->t_final_unbinding = NAN;
	s->t_boundary_escape = NAN;
	s->t_termination = -1.0;
	s->event_observed = 0;
	s->boundary_escape_observed = 0;
	s->survival_valid = 1;
	s->invalid_escape = 0;
	s->max_drift_eV = 0.0;
	s->max_drift_rel = 0.0;
	s->prev_time = -1.0;
	s->prev_r = 0.0;
	s->prev_v2 = 0.0;
	s->prev_dt = 0.0;
	s->previous_capture_energy = capture_energy_eV(o, ev_radius(&cur), ev_speed(&cur));
	s->free_flight_reference_energy = NAN;
	s->bound_state = 0;
	int reason = DMS_REASON_UNKNOWN;
	while(nscat < s->max_scatterings)
	{
		const int pr = propagate_freely(o, s, &cur);
		if(pr == DMS_REASON_SCATTER && ev_radius(&cur) < DMS_RSUN_KM)
		{
			DMS_OPS_PHASE(2);
			if(!scatter(o, &cur))
			{
				reason = DMS_REASON_NUMERICAL_FAILURE;
				break;
			}
			nscat++;
			DMS_OPS_MARK(2);
			const int cap = update_capture_state(o, s, ev_radius(&cur), ev_speed(&cur), cur.time, 1);
			reset_anchor(s, &cur);
			if(s->capture_mode && cap)
			{
				reason = DMS_REASON_CAPTURE_MODE;
				break;
			}
		}
		else
		{
			reason = pr;
			break;
		}
	}
	DMS_OPS_PHASE(3);
	if(reason == DMS_REASON_UNKNOWN && nscat >= s->max_scatterings)
		reason = DMS_REASON_MAX_SCATTERINGS;
	s->t_termination = cur.time;
	if(s->is_captured)
	{
		const double r_f = ev_radius(&cur), v_f = ev_speed(&cur);
		const double vesc_f = solar_vesc(o, r_f);
		const double E_f = 0.5 * o->m_dm * ((v_f * v_f - vesc_f * vesc_f) / (DMS_C_KMS * DMS_C_KMS)) / 1.0e-9;
		if(reason == DMS_REASON_OUTWARD_ESCAPE && E_f >= 0.0)
		{
			if(isfinite(s->t_final_unbinding))
			{
				s->boundary_escape_observed = 1;
				s->t_boundary_escape = s->t_termination;
				s->event_observed = 1;
			}
			else
			{
				reason = DMS_REASON_ENERGY_DRIFT_ESCAPE;
				s->survival_valid = 0;
				s->invalid_escape = 1;
				s->boundary_escape_observed = 0;
				s->event_observed = 0;
			}
		}
	}
	/* TrajectoryTerminationInvalidatesSurvival, :506-522 */
	switch(reason)
	{
		case DMS_REASON_ENERGY_DRIFT_ESCAPE:
		case DMS_REASON_NUMERICAL_FAILURE:
		case DMS_REASON_NON_FINITE_STATE:
		case DMS_REASON_SPEED_LIMIT:
		case DMS_REASON_WALL_TIME_LIMIT:
		case DMS_REASON_MAX_FREE_STEPS:
		case DMS_REASON_MAX_SCATTERINGS:
		case DMS_REASON_UNKNOWN: s->survival_valid = 0; break;
		default: break;
	}
	if(s->is_captured)
	{
		if(!s->event_observed)
		{
			s->t_final_unbinding = NAN;
			if(reason != DMS_REASON_CAPTURE_MODE)
				s->survival_valid = 0;
		}
	}
	rec->number_of_scatterings = nscat;
	rec->termination_reason = (uint32_t)reason;
	rec->final_time = cur.time;
	memcpy(rec->final_position, cur.position.x, sizeof cur.position.x);
	memcpy(rec->final_velocity, cur.velocity.x, sizeof cur.velocity.x);
	rec->t_capture = s->t_capture;
	rec->t_last_bound = s->t_last_bound;
	rec->t_final_unbinding_scatter = s->t_final_unbinding;
	rec->t_boundary_escape = s->t_boundary_escape;
	rec->t_termination = s->t_termination;
	rec->max_free_energy_drift_eV = s->max_drift_eV;
	rec->max_free_energy_drift_rel = s->max_drift_rel;
	uint32_t flags = DMS_REC_SHIFT_OK;
	if(s->is_captured) flags |= DMS_REC_CAPTURED;
	if(s->event_observed) flags |= DMS_REC_EVENT_OBSERVED;
	if(s->survival_valid) flags |= DMS_REC_SURVIVAL_VALID;
	if(s->boundary_escape_observed) flags |= DMS_REC_BOUNDARY_ESCAPE;
	if(s->invalid_escape) flags |= DMS_REC_INVALID_ESCAPE;
	/* Particle_Free / Particle_Reflected, :529-542, and the reflection shift, src/Data_Generation.cpp:824-846 */
	if(!s->is_captured && reason == DMS_REASON_OUTWARD_ESCAPE)
	{
		if(nscat == 0)
			flags |= DMS_REC_FREE;
		else
		{
			const double rf = ev_radius(&cur);
			const double vesc = sqrt(2 * DMS_GMSUN_KM3S2 / rf);
			if(rf > DMS_RSUN_KM && ev_speed(&cur) > vesc)
			{
				flags |= DMS_REC_REFLECTED;
				event_t fin = cur;
				if(hyperbolic_kepler_shift(&fin, DMS_AU_KM))
				{
					flags |= DMS_REC_REFLECT_SHIFT_OK;
					if(o->reflection != NULL)
					{
						/* src/Data_Generation.cpp:829-840: the speed at 1 AU and the angle of the
						 * position to the Sun's velocity that Isoreflection_Ring bins */
						const double* vs = o->vel_obs.x;
						const double sun = sqrt(vs[0] * vs[0] + vs[1] * vs[1] + vs[2] * vs[2]);
						o->reflection[0] = ev_speed(&fin);
						o->reflection[1] = (fin.position.x[0] * vs[0] + fin.position.x[1] * vs[1] + fin.position.x[2] * vs[2]) /
						                   ev_radius(&fin) / sun;
					}
				}
			}
		}
	}
	rec->flags = flags;
	/* Build_Evaporation_Record lifetime, src/Data_Generation.cpp:118-164 */
	const int invalid_escape = s->invalid_escape || reason == DMS_REASON_ENERGY_DRIFT_ESCAPE;
	const int valid = s->survival_valid && !invalid_escape;
	const int observed = valid && s->event_observed;
	const double lifetime = observed ? s->t_final_unbinding - s->t_capture : -1.0;
	rec->lifetime_unbinding = (s->is_captured && isfinite(lifetime) && lifetime >= 0.0) ? lifetime : -1.0;
}

/* ------------------------------------------------------------------------------------------
 * Public API
 */
dms_oracle* dms_oracle_create(const char* path)
{
	dms_oracle* o = (dms_oracle*)calloc(1, sizeof(dms_oracle));
	if(!o)
		return NULL;
	if(load_solar(o, path) != 0)
	{
		fprintf(stderr, "dms_oracle_create: %s\n", o->error);
		dms_oracle_destroy(o);
		return NULL;
	}
	return o;
}

void dms_oracle_destroy(dms_oracle* o)
{
	if(!o)
		return;
	table1d* tabs[4] = {&o->gm, &o->temp, &o->vesc2, &o->n_e};
	for(int k = 0; k < 4; k++)
	{
		free(tabs[k]->y);
		free(tabs[k]->s);
	}
	for(int t = 0; t < DMS_NUM_TARGETS; t++)
	{
		free(o->targets[t].y);
		free(o->targets[t].s);
	}
	free(o->r);
	free(o->grid);
	free(o);
}

const char* dms_oracle_last_error(const dms_oracle* o) { return o ? o->error : "null oracle"; }

int dms_oracle_set_point(dms_oracle* o, const dms_point_params* p)
{
	if(!o || !p || !(p->mass_gev > 0.0))
		return DMS_ERR_INVALID_ARGUMENT;
	if(p->interaction > DMS_INTERACTION_DARK_PHOTON_GENERAL ||
	   (p->interaction == DMS_INTERACTION_DARK_PHOTON_GENERAL && !(p->mediator_mass_mev > 0.0 && isfinite(p->mediator_mass_mev))))
		return DMS_ERR_INVALID_ARGUMENT;
	o->m_dm = p->mass_gev;
	o->interaction = p->interaction;
	const int dark_photon = p->interaction != DMS_INTERACTION_SI;
	const double mu_p = o->m_dm * DMS_MPROTON_GEV / (o->m_dm + DMS_MPROTON_GEV);
	const double mu_e = o->m_dm * DMS_MELECTRON_GEV / (o->m_dm + DMS_MELECTRON_GEV);
	o->sigma_e = p->sigma_e_cm2 * 1.0e-10;
	/* the dark photon's proton cross section follows from the electron one through the kinetic
	 * mixing (Set_Sigma_Electron then Sigma_Proton, src/Dark_Photon.cpp:130-133, 157-161) */
	const double ratio_pe = mu_p / mu_e;
	const double sigma_p = dark_photon ? o->sigma_e * ratio_pe * ratio_pe : p->sigma_p_cm2 * 1.0e-10;
	for(int t = 0; t < DMS_NUM_TARGETS; t++)
	{
		/* DM_Particle_SI::Sigma_Total_Nucleus restated (oracle/shim/obscura/DM_Particle.hpp), or the
		 * dark photon's low-mass Sigma_Total_Nucleus, sigma_p (mu_N/mu_p)^2 Z^2 (src/Dark_Photon.cpp:167-184) */
		const dms_target_isotope* iso = &DMS_TARGET_ISOTOPES[t];
		const double mN = o->target_mass_gev[t];
		const double mu_N = o->m_dm * mN / (o->m_dm + mN);
		const double coupling = dark_photon ? (double)iso->Z : iso->Z + p->fn_over_fp * (iso->A - iso->Z);
		const double ratio = mu_N / mu_p;
		o->sigma_target[t] = sigma_p * ratio * ratio * coupling * coupling;
		const double mc = mu_N / DMS_C_KMS;
		o->q2c[t] = 4.0 * mc * mc;
	}
	{
		const double mc = mu_e / DMS_C_KMS;
		o->q2c[DMS_NUM_TARGETS] = 4.0 * mc * mc;
	}
	if(p->interaction == DMS_INTERACTION_DARK_PHOTON_GENERAL)
	{
		const double m = p->mediator_mass_mev * 1.0e-3;
		const double q_ref = DMS_ALPHA_EM * DMS_MELECTRON_GEV;
		const double a = q_ref * q_ref + m * m;
		o->ff_m2 = m * m;
		o->ff_num = a * a / m / m;
	}
	else
	{
		o->ff_m2 = 0.0;
		o->ff_num = 0.0;
	}
	o->v0 = p->halo_v0_kms;
	o->vesc_halo = p->halo_vesc_kms;
	o->vel_obs = v3(p->halo_vobs_kms[0], p->halo_vobs_kms[1], p->halo_vobs_kms[2]);
	o->vobs = v_norm(o->vel_obs);
	const double z = o->vesc_halo / o->v0;
	o->n_esc = erf(z) - 2.0 * z * exp(-z * z) / SQRT_PI;
	o->halo_avg_speed = halo_moment(o, 1, 0.0, o->vesc_halo - o->vobs) + halo_moment(o, 1, o->vesc_halo - o->vobs, o->vesc_halo + o->vobs);
	o->halo_eta0 = halo_moment(o, -1, 0.0, o->vesc_halo - o->vobs) + halo_moment(o, -1, o->vesc_halo - o->vobs, o->vesc_halo + o->vobs);
	/* rate grid, Interpolate_Total_DM_Scattering_Rate src/Solar_Model.cpp:395-465 */
	const unsigned int N = p->interpolation_points;
	free(o->grid);
	o->grid = NULL;
	if(N < 2)
	{
		/* N < 2: no grid, every lookup is computed (src/Solar_Model.cpp:397-405) */
		o->grid_n = 0;
		o->grid_inv_r = 0.0;
		o->grid_inv_v = 0.0;
		o->grid_vmax = -1.0;
		o->has_point = 1;
		return DMS_OK;
	}
	o->grid = (double*)malloc((size_t)N * N * sizeof(double));
	if(!o->grid)
		return DMS_ERR_CAPACITY;
	o->grid_n = (int)N;
	const double vmax_c = DMS_V_MAX_C;
	const double vstep_c = (vmax_c - 0.0) / (N - 1);
	for(unsigned int i = 0; i < N; i++)
	{
		const double radius = DMS_RSUN_KM * (double)i / (double)(N - 1);
		for(unsigned int j = 0; j < N; j++)
		{
			const double speed = (0.0 + j * vstep_c) * DMS_C_KMS;
			o->grid[(size_t)i * N + j] = rate_computed(o, radius, speed);
		}
	}
	o->grid_inv_r = (double)(N - 1) / DMS_RSUN_KM;
	o->grid_vmax = vmax_c * DMS_C_KMS;
	o->grid_inv_v = (double)(N - 1) / o->grid_vmax;
	o->has_point = 1;
	return DMS_OK;
}

double dms_oracle_query(dms_oracle* o, int what, double a, double b, double c)
{
	if(!o)
		return NAN;
	switch(what)
	{
		case 0: return solar_gm(o, a);
		case 1: return solar_temperature(o, a) / DMS_KB_GEV_PER_K;
		case 2: return solar_vesc(o, a);
		case 3: return solar_density(&o->n_e, a);
		case 4: return solar_density(&o->targets[(int)b], a);
		case 5: return o->has_point ? rate_total(o, a, b) : NAN;
		case 6: return o->has_point ? rate_computed(o, a, b) : NAN;
		case 7: return thermal_relative_speed(a * DMS_KB_GEV_PER_K, b, c);
		case 8: return o->has_point ? halo_pdf_speed(o, a) : NAN;
		case 9: return o->has_point ? o->halo_avg_speed : NAN;
		case 10: return o->has_point ? o->halo_eta0 : NAN;
		case 11: return o->target_mass_gev[(int)a];
		case 12:
			if(!o->has_point)
				return NAN;
			return (b < 0.0) ? rate_electron(o, a, c) : rate_nucleus(o, a, c, (int)b);
		default: return NAN;
	}
}

int dms_oracle_num_nodes(const dms_oracle* o) { return o ? o->n : 0; }

int dms_oracle_tables(const dms_oracle* o, double* r, double* gm, double* temperature_gev, double* vesc2, double* n_e, double* n_targets)
{
	if(!o)
		return DMS_ERR_INVALID_ARGUMENT;
	for(int i = 0; i < o->n; i++)
	{
		if(r) r[i] = o->r[i];
		if(gm) gm[i] = o->gm.y[i];
		if(temperature_gev) temperature_gev[i] = o->temp.y[i];
		if(vesc2) vesc2[i] = o->vesc2.y[i];
		if(n_e) n_e[i] = o->n_e.y[i];
		if(n_targets)
			for(int t = 0; t < DMS_NUM_TARGETS; t++) n_targets[(size_t)i * DMS_NUM_TARGETS + t] = o->targets[t].y[i];
	}
	return DMS_OK;
}

int dms_oracle_rate_grid(const dms_oracle* o, double* grid)
{
	if(!o || !o->has_point)
		return DMS_ERR_NO_POINT;
	memcpy(grid, o->grid, (size_t)o->grid_n * o->grid_n * sizeof(double));
	return DMS_OK;
}

/* dms_oracle_run_records in Parameter-point mode that also returns, per trajectory, the
 * reflection-spectrum sample: reflection[2k] = speed at 1 AU [km/s], reflection[2k+1] = cosine
 * of the angle between the position at 1 AU and the Sun's velocity; NaN unless trajectory k is a
 * reflected particle whose final Kepler shift succeeded (src/Data_Generation.cpp:824-846). */
int dms_oracle_run_reflections(dms_oracle* o, uint32_t seed, uint32_t point, uint64_t max_scatterings, double boundary_rsun,
                               uint64_t first, uint64_t count, dms_traj_record* records, double* reflection)
{
	if(!o)
		return DMS_ERR_INVALID_ARGUMENT;
	o->reflection_base = reflection;
	const int rc = dms_oracle_run_records(o, seed, point, 0, max_scatterings, boundary_rsun, first, count, records, NULL, NULL,
	                                      NULL, 0, NULL);
	o->reflection_base = NULL;
	o->reflection = NULL;
	return rc;
}

/* dms_oracle_run_records with the event after the initial Kepler shift of every trajectory
 * given by the caller (starts: 7 doubles t [s], x [km], v [km/s] per trajectory): the initial
 * conditions still run, so the draws after them are the usual ones.  Replays the reference's own
 * shifted initial states (whose computation from 1000 AU amplifies last-bit differences about
 * 1e7-fold) to compare the rest of the path. */
int dms_oracle_run_from_starts(dms_oracle* o, uint32_t seed, uint32_t point, int capture_mode, uint64_t max_scatterings,
                               double boundary_rsun, uint64_t first, uint64_t count, const double* starts,
                               dms_traj_record* records, double* trace, size_t trace_capacity, size_t* trace_length)
{
	if(!o || !starts)
		return DMS_ERR_INVALID_ARGUMENT;
	o->start_base = starts;
	const int rc = dms_oracle_run_records(o, seed, point, capture_mode, max_scatterings, boundary_rsun, first, count, records, NULL,
	                                      NULL, trace, trace_capacity, trace_length);
	o->start_base = NULL;
	return rc;
}

/* Replaces the current point's N x N grid (the rate_grid member of Solar_Model,
 * include/Solar_Model.hpp:309) by one built elsewhere: the test of the engine's own device-built
 * grid replays the oracle on that grid, the same role dms_set_rate_grid plays for the engine. */
int dms_oracle_set_rate_grid(dms_oracle* o, const double* grid, uint32_t n)
{
	if(!o || !o->has_point)
		return DMS_ERR_NO_POINT;
	if(!grid || n < 2 || (int)n != o->grid_n)
		return DMS_ERR_INVALID_ARGUMENT;
	memcpy(o->grid, grid, (size_t)n * n * sizeof(double));
	return DMS_OK;
}

int dms_oracle_run_records(dms_oracle* o, uint32_t seed, uint32_t point, int capture_mode, uint64_t max_scatterings,
                           double boundary_rsun, uint64_t first, uint64_t count, dms_traj_record* records, double* hist_dt,
                           double* hist_v2dt, double* trace, size_t trace_capacity, size_t* trace_length)
{
	if(!o || !o->has_point || !records)
		return DMS_ERR_INVALID_ARGUMENT;
	sim_t s;
	memset(&s, 0, sizeof s);
	s.capture_mode = capture_mode;
	s.max_free_steps = 1000000000000ULL;  /* DEFAULT_MAXIMUM_FREE_TIME_STEPS */
	s.max_scatterings = max_scatterings;
	s.max_distance = boundary_rsun * DMS_RSUN_KM;
	double* dt_buf = (double*)malloc(DMS_NUM_BINS * sizeof(double));
	double* v2_buf = (double*)malloc(DMS_NUM_BINS * sizeof(double));
	s.dt_hist = dt_buf;
	s.v2dt_hist = v2_buf;
	for(uint64_t k = 0; k < count; k++)
	{
		dms_traj_record* rec = &records[k];
		memset(rec, 0, sizeof *rec);
		rec->trajectory_id = first + k;
		rec->point = point;
		o->seed = seed;
		o->point = point;
		o->traj = first + k;
		o->draw_index = 0;
		o->trace = (trace != NULL && k == 0) ? trace : NULL;
		o->reflection = o->reflection_base != NULL ? o->reflection_base + 2 * k : NULL;
		if(o->reflection != NULL)
			o->reflection[0] = o->reflection[1] = NAN;
		o->trace_capacity = trace_capacity;
		o->trace_length = 0;
		DMS_OPS_MARK(3);
		DMS_OPS_PHASE(3);
		event_t ic = initial_conditions(o);
		const int shift_ok = hyperbolic_kepler_shift(&ic, s.max_distance);
		if(o->start_base != NULL)
		{
			const double* st = o->start_base + 7 * k;
			ic.time = st[0];
			for(int i = 0; i < 3; i++)
			{
				ic.position.x[i] = st[1 + i];
				ic.velocity.x[i] = st[4 + i];
			}
		}
		rec->initial_time = ic.time;
		memcpy(rec->initial_position, ic.position.x, sizeof ic.position.x);
		memcpy(rec->initial_velocity, ic.velocity.x, sizeof ic.velocity.x);
		if(!shift_ok)
		{
			rec->termination_reason = DMS_REASON_NUMERICAL_FAILURE;
			rec->flags = 0;
			rec->final_time = ic.time;
			memcpy(rec->final_position, ic.position.x, sizeof ic.position.x);
			memcpy(rec->final_velocity, ic.velocity.x, sizeof ic.velocity.x);
			rec->t_capture = -1.0;
			rec->t_last_bound = -1.0;
			rec->t_final_unbinding_scatter = NAN;
			rec->t_boundary_escape = NAN;
			rec->t_termination = -1.0;
			rec->lifetime_unbinding = -1.0;
			memset(dt_buf, 0, DMS_NUM_BINS * sizeof(double));
			memset(v2_buf, 0, DMS_NUM_BINS * sizeof(double));
		}
		else
			simulate(o, &s, &ic, rec);
		rec->number_of_draws = o->draw_index;
		if(hist_dt) memcpy(hist_dt + k * DMS_NUM_BINS, dt_buf, DMS_NUM_BINS * sizeof(double));
		if(hist_v2dt) memcpy(hist_v2dt + k * DMS_NUM_BINS, v2_buf, DMS_NUM_BINS * sizeof(double));
		if(o->trace != NULL && trace_length)
			*trace_length = o->trace_length;
	}
	o->trace = NULL;
	free(dt_buf);
	free(v2_buf);
	return DMS_OK;
}
