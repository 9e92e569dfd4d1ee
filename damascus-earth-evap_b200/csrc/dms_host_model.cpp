// Host-side model construction; see dms_host_model.h.
#include "dms_host_model.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace dms
{

namespace
{
void Slopes(const std::vector<double>& x, const std::vector<double>& y, std::vector<double>& s)
{
	s.assign(x.size(), 0.0);
	for(size_t i = 0; i + 1 < x.size(); i++)
		s[i] = (y[i + 1] - y[i]) / (x[i + 1] - x[i]);
}

int Knot_Search(const std::vector<double>& x, double v)
{
	int lo = 0, hi = static_cast<int>(x.size()) - 1;
	if(v >= x[hi - 1])
		return hi - 1;
	while(hi - lo > 1)
	{
		const int mid = (lo + hi) / 2;
		if(x[mid] <= v)
			lo = mid;
		else
			hi = mid;
	}
	return lo;
}

const double GL7_X[7] = {0.0, -0.4058451513773971669066064, 0.4058451513773971669066064, -0.7415311855993944398638648, 0.7415311855993944398638648, -0.9491079123427585245261897, 0.9491079123427585245261897};
const double GL7_W[7] = {0.4179591836734693877551020, 0.3818300505051189449503698, 0.3818300505051189449503698, 0.2797053914892766679014678, 0.2797053914892766679014678, 0.1294849661688696932706114, 0.1294849661688696932706114};
const double SQRT_PI = std::sqrt(3.14159265358979323846);

// Standard Halo Model speed distribution f(v) in the observer frame (see
// Halo_Pdf_Speed in dms_device.cuh for the formula).
double Halo_Pdf_Speed(const PointConstants& c, double v)
{
	if(v < 0.0 || v > c.vesc_halo + c.vobs)
		return 0.0;
	const double dm = v - c.vobs;
	const double dp = v + c.vobs;
	const double a = std::exp(-dm * dm / (c.v0 * c.v0));
	const double b = (dp <= c.vesc_halo) ? std::exp(-dp * dp / (c.v0 * c.v0)) : std::exp(-c.vesc_halo * c.vesc_halo / (c.v0 * c.v0));
	return v / (c.n_esc * SQRT_PI * c.v0 * c.vobs) * (a - b);
}

// 256-panel composite 7-point Gauss-Legendre of v^power f(v) on [a, b] (power = +1 or -1).
double Halo_Moment(const PointConstants& c, int power, double a, double b)
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
			const double f = (power > 0) ? v * Halo_Pdf_Speed(c, v) : ((v > 0.0) ? Halo_Pdf_Speed(c, v) / v : 0.0);
			panel += GL7_W[k] * f;
		}
		sum += 0.5 * h * panel;
	}
	return sum;
}
}	// namespace

double Table_Eval(const SolarTables& t, const std::vector<double>& y, const std::vector<double>& s, double x)
{
	const int i = Knot_Search(t.r, x);
	return y[i] + (x - t.r[i]) * s[i];
}

std::string Load_Solar_Tables(const std::string& path, SolarTables& t)
{
	FILE* f = std::fopen(path.c_str(), "r");
	if(!f)
		return "cannot open solar model file " + path;
	char line[4096];
	for(int i = 0; i < DMS_SOLAR_DATA_SKIP_LINES; i++)
		if(!std::fgets(line, sizeof line, f))
			break;
	// raw rows in file units, with room for the two padding rows
	std::vector<double> raw(DMS_SOLAR_COLUMNS, 0.0);
	size_t rows = 0;
	while(std::fgets(line, sizeof line, f))
	{
		double vals[DMS_SOLAR_COLUMNS];
		int k = 0;
		char* p = line;
		char* end;
		while(k < DMS_SOLAR_COLUMNS)
		{
			const double v = std::strtod(p, &end);
			if(end == p)
				break;
			vals[k++] = v;
			p = end;
		}
		if(k == 0)
			continue;
		if(k != DMS_SOLAR_COLUMNS)
		{
			std::fclose(f);
			return "malformed solar model row " + std::to_string(rows + 1) + " (" + std::to_string(k) + " columns)";
		}
		raw.insert(raw.end(), vals, vals + DMS_SOLAR_COLUMNS);
		rows++;
	}
	std::fclose(f);
	if(rows < 2)
		return "solar model file has fewer than two data rows";
	raw.insert(raw.end(), DMS_SOLAR_COLUMNS, 0.0);
	const int n = static_cast<int>(rows) + 2;
	// padding rows, src/Solar_Model.cpp:47-65
	double* first = &raw[0];
	double* last = &raw[(n - 1) * DMS_SOLAR_COLUMNS];
	const double* front = &raw[DMS_SOLAR_COLUMNS];
	const double* back = &raw[(n - 2) * DMS_SOLAR_COLUMNS];
	for(int i = 0; i < DMS_SOLAR_COLUMNS; i++)
	{
		first[i] = (i == 0 || i == 1) ? 0.0 : front[i];
		last[i] = back[i];
	}
	last[0] = 1.0;
	last[1] = 1.0;
	last[2] = DMS_PHOTOSPHERE_T_K;
	last[3] = DMS_PHOTOSPHERE_RHO_GCM3;
	for(int i = 1; i < n; i++)
		if(!(raw[i * DMS_SOLAR_COLUMNS + 1] > raw[(i - 1) * DMS_SOLAR_COLUMNS + 1]))
			return "solar model radii are not strictly increasing at row " + std::to_string(i);

	t.n = n;
	t.r.resize(n);
	t.gm.resize(n);
	t.temp.resize(n);
	t.vesc2.resize(n);
	t.ne.assign(n, 0.0);
	for(int i = 0; i < n; i++)
	{
		const double* row = &raw[i * DMS_SOLAR_COLUMNS];
		t.r[i] = row[1] * DMS_RSUN_KM;
		t.gm[i] = row[0] * DMS_GMSUN_KM3S2;
		t.temp[i] = row[2] * DMS_KB_GEV_PER_K;
		for(int c = 0; c < DMS_SOLAR_COLUMNS; c++)
			if(!std::isfinite(row[c]))
				return "non-finite value in solar model row " + std::to_string(i);
	}
	Slopes(t.r, t.gm, t.gm_s);
	Slopes(t.r, t.temp, t.temp_s);

	// escape speed: Create_Escape_Speed_Table (src/Solar_Model.cpp:79-96), integrand G M(x)/x^2 with
	// integrand(0) = 0; exact integral of the piecewise-linear profile on each knot interval,
	// trapezoid on an interval that starts at x = 0
	for(int k = 0; k < n; k++)
	{
		const double rk = t.r[k];
		double integral;
		if(rk < DMS_RSUN_KM)
		{
			integral = 0.0;
			for(int j = k; j + 1 < n; j++)
			{
				const double lo = t.r[j], hi = t.r[j + 1];
				const double f_lo = (lo == 0.0) ? 0.0 : Table_Eval(t, t.gm, t.gm_s, lo) / lo / lo;
				const double f_hi = (hi == 0.0) ? 0.0 : Table_Eval(t, t.gm, t.gm_s, hi) / hi / hi;
				if(lo == 0.0)
				{
					integral += 0.5 * (hi - lo) * (f_lo + f_hi);
					continue;
				}
				const double g_lo = f_lo * lo * lo, g_hi = f_hi * hi * hi;
				const double h = hi - lo;
				const double s = (g_hi - g_lo) / h;
				integral += g_lo * h / (lo * hi) + s * (std::log1p(h / lo) - h / hi);
			}
		}
		else
			integral = DMS_GMSUN_KM3S2 * (1.0 / rk - 1.0 / DMS_RSUN_KM);
		t.vesc2[k] = 2.0 * DMS_GMSUN_KM3S2 / DMS_RSUN_KM * (1.0 + DMS_RSUN_KM / DMS_GMSUN_KM3S2 * integral);
	}
	Slopes(t.r, t.vesc2, t.vesc2_s);

	// isotope number densities n = f rho / m, times the natural abundance (src/Solar_Model.cpp:98-110, 143-163)
	t.nt.assign(static_cast<size_t>(n) * DMS_NUM_TARGETS, 0.0);
	t.nt_s.assign(static_cast<size_t>(n) * DMS_NUM_TARGETS, 0.0);
	std::vector<double> col(n), col_s;
	for(int k = 0; k < DMS_NUM_TARGETS; k++)
	{
		const dms_target_isotope& iso = DMS_TARGET_ISOTOPES[k];
		const double m_gev = (iso.A == 1) ? DMS_MPROTON_GEV : iso.A * DMS_MNUCLEON_GEV;
		const double m_kg = m_gev / DMS_GEV_PER_KG;
		t.target_mass_gev[k] = m_gev;
		for(int i = 0; i < n; i++)
		{
			const double* row = &raw[i * DMS_SOLAR_COLUMNS];
			const double rho = row[3] * 1.0e12;  // g/cm^3 -> kg/km^3
			col[i] = row[6 + iso.element_index] * rho / m_kg;
		}
		if(iso.element_index >= 10)
			for(int i = 0; i < n; i++) col[i] *= iso.abundance;
		Slopes(t.r, col, col_s);
		for(int i = 0; i < n; i++)
		{
			t.nt[static_cast<size_t>(i) * DMS_NUM_TARGETS + k] = col[i];
			t.nt_s[static_cast<size_t>(i) * DMS_NUM_TARGETS + k] = col_s[i];
		}
	}
	// electron density, src/Solar_Model.cpp:112-126: sum over targets of Z n_i at the knots
	for(int k = 0; k < DMS_NUM_TARGETS; k++)
	{
		std::vector<double> y(n), s(n);
		for(int i = 0; i < n; i++)
		{
			y[i] = t.nt[static_cast<size_t>(i) * DMS_NUM_TARGETS + k];
			s[i] = t.nt_s[static_cast<size_t>(i) * DMS_NUM_TARGETS + k];
		}
		for(int i = 0; i < n; i++)
		{
			const double ri = t.r[i];
			const double nk = (ri > DMS_RSUN_KM) ? 0.0 : Table_Eval(t, y, s, ri < 0.0 ? 0.0 : ri);
			t.ne[i] += static_cast<double>(DMS_TARGET_ISOTOPES[k].Z) * nk;
		}
	}
	Slopes(t.r, t.ne, t.ne_s);

	// bucket acceleration for the device knot search.  The device maps x in [0, R_sun] to bucket
	// b = (int)(x * scale) with scale = nbuckets / R_sun (one IEEE multiply, truncation).  The
	// base of bucket b is the knot interval of the smallest x that the device maps to b, so every
	// x of the bucket lies in that interval or a later one; when no bucket holds more than one
	// knot, the interval is the base or the base + 1 and the device search is one select.
	if(n > 65535)
		return "solar model has too many rows";
	t.nbuckets = 8192;
	const double scale = static_cast<double>(t.nbuckets) / DMS_RSUN_KM;
	std::vector<double> lowest(t.nbuckets + 2, DMS_RSUN_KM);
	t.bucket_index.resize(t.nbuckets + 1);
	for(int b = 0; b <= t.nbuckets; b++)
	{
		// smallest double x >= 0 with (int)(x * scale) >= b
		double x = static_cast<double>(b) / scale;
		while(x > 0.0 && static_cast<int>(x * scale) >= b) x = std::nextafter(x, -1.0);
		while(static_cast<int>(x * scale) < b) x = std::nextafter(x, 2.0 * DMS_RSUN_KM);
		lowest[b] = x;
		t.bucket_index[b] = static_cast<uint16_t>(Knot_Search(t.r, x));
	}
	t.bucket_single_step = 1;
	for(int b = 0; b < t.nbuckets; b++)
	{
		// the last x of bucket b is just below lowest[b + 1]: its interval must be base or base + 1
		const double top = std::nextafter(lowest[b + 1], -1.0);
		if(Knot_Search(t.r, top) > t.bucket_index[b] + 1)
			t.bucket_single_step = 0;
	}
	if(Knot_Search(t.r, DMS_RSUN_KM) > t.bucket_index[t.nbuckets] + 1)
		t.bucket_single_step = 0;
	return "";
}

std::string Make_Point_Constants(const SolarTables& t, const dms_point_params& p, PointConstants& c)
{
	if(!(p.mass_gev > 0.0) || !std::isfinite(p.mass_gev))
		return "DM mass must be finite and positive";
	if(!(p.sigma_p_cm2 >= 0.0) || !std::isfinite(p.sigma_p_cm2) || !(p.sigma_e_cm2 >= 0.0) || !std::isfinite(p.sigma_e_cm2))
		return "DM cross sections must be finite and non-negative";
	if(static_cast<uint64_t>(p.interpolation_points) * p.interpolation_points > (1ULL << 28))
		return "interpolation grid too large";
	if(!(p.halo_v0_kms > 0.0) || !(p.halo_vesc_kms > 0.0))
		return "halo v0 and v_esc must be positive";
	if(p.interaction > DMS_INTERACTION_DARK_PHOTON_GENERAL)
		return "unknown DM interaction model";
	if(p.interaction == DMS_INTERACTION_DARK_PHOTON_GENERAL && !(p.mediator_mass_mev > 0.0 && std::isfinite(p.mediator_mass_mev)))
		return "'DM_mediator_mass' must be finite and positive for the General form factor";
	c.m_dm = p.mass_gev;
	c.interaction = p.interaction;
	const bool dark_photon = p.interaction != DMS_INTERACTION_SI;
	const double mu_p = c.m_dm * DMS_MPROTON_GEV / (c.m_dm + DMS_MPROTON_GEV);
	const double mu_e = c.m_dm * DMS_MELECTRON_GEV / (c.m_dm + DMS_MELECTRON_GEV);
	c.sigma_e = p.sigma_e_cm2 * 1.0e-10;
	// the dark photon's kinetic mixing ties its proton cross section to the electron one:
	// sigma_p = sigma_e (mu_p/mu_e)^2 (Set_Sigma_Electron, Sigma_Proton, src/Dark_Photon.cpp:130-133, 157-161)
	const double ratio_pe = mu_p / mu_e;
	const double sigma_p = dark_photon ? c.sigma_e * ratio_pe * ratio_pe : p.sigma_p_cm2 * 1.0e-10;
	for(int k = 0; k < DMS_NUM_TARGETS; k++)
	{
		// contact cross section in low-mass mode: sigma_p (mu_N/mu_p)^2 [Z + (f_n/f_p)(A - Z)]^2 for
		// SI, sigma_p (mu_N/mu_p)^2 Z^2 for the dark photon (src/Dark_Photon.cpp:167-184)
		const dms_target_isotope& iso = DMS_TARGET_ISOTOPES[k];
		const double mN = t.target_mass_gev[k];
		const double mu_N = c.m_dm * mN / (c.m_dm + mN);
		const double coupling = dark_photon ? static_cast<double>(iso.Z) : iso.Z + p.fn_over_fp * (iso.A - iso.Z);
		const double ratio = mu_N / mu_p;
		c.sigma_target[k] = sigma_p * ratio * ratio * coupling * coupling;
		const double mc = mu_N / DMS_C_KMS;
		c.q2c[k] = 4.0 * mc * mc;
	}
	{
		const double mc = mu_e / DMS_C_KMS;
		c.q2c[DMS_NUM_TARGETS] = 4.0 * mc * mc;
	}
	if(p.interaction == DMS_INTERACTION_DARK_PHOTON_GENERAL)
	{
		// (q_ref^2 + m^2)^2 / m^2 with q_ref = alpha m_e (src/Dark_Photon.cpp:15-16, 194-198)
		const double m = p.mediator_mass_mev * 1.0e-3;
		const double q_ref = DMS_ALPHA_EM * DMS_MELECTRON_GEV;
		const double a = q_ref * q_ref + m * m;
		c.ff_m2 = m * m;
		c.ff_num = a * a / m / m;
	}
	else
	{
		c.ff_m2 = 0.0;
		c.ff_num = 0.0;
	}
	c.v0 = p.halo_v0_kms;
	c.vesc_halo = p.halo_vesc_kms;
	for(int i = 0; i < 3; i++) c.vel_obs[i] = p.halo_vobs_kms[i];
	double s = 0.0;
	for(int i = 0; i < 3; i++) s += c.vel_obs[i] * c.vel_obs[i];
	c.vobs = std::sqrt(s);
	if(!(c.vobs > 0.0))
		return "the observer velocity must be non-zero";
	const double z = c.vesc_halo / c.v0;
	c.n_esc = std::erf(z) - 2.0 * z * std::exp(-z * z) / SQRT_PI;
	c.avg_speed = Halo_Moment(c, 1, 0.0, c.vesc_halo - c.vobs) + Halo_Moment(c, 1, c.vesc_halo - c.vobs, c.vesc_halo + c.vobs);
	c.eta0 = Halo_Moment(c, -1, 0.0, c.vesc_halo - c.vobs) + Halo_Moment(c, -1, c.vesc_halo - c.vobs, c.vesc_halo + c.vobs);
	const unsigned int N = p.interpolation_points;
	if(N < 2)
	{
		// no grid (Interpolate_Total_DM_Scattering_Rate with N < 2, src/Solar_Model.cpp:397-405):
		// every lookup is Total_DM_Scattering_Rate_Computed; a negative limit speed sends every
		// speed to that branch
		c.grid_n = 0;
		c.grid_inv_r = 0.0;
		c.grid_inv_v = 0.0;
		c.grid_vmax = -1.0;
		return "";
	}
	c.grid_n = static_cast<int>(N);
	c.grid_inv_r = static_cast<double>(N - 1) / DMS_RSUN_KM;
	c.grid_vmax = DMS_V_MAX_C * DMS_C_KMS;
	c.grid_inv_v = static_cast<double>(N - 1) / c.grid_vmax;
	return "";
}

}	// namespace dms
