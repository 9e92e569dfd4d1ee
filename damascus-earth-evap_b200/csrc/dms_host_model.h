// Host-side model construction for the engine: the AGSS09 radial tables
// (Solar_Model::Solar_Model, src/Solar_Model.cpp:43-166), the parameter-point constants
// (DM particle cross sections, Standard Halo Model moments) and the packed device images
// of both.  Everything here runs once per context / per point; the trajectory work is on
// the device.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/dms.h"
#include "../../include/dms_constants.h"
#include "../../include/dms_nuclear_data.h"

namespace dms
{

// Radial tables in engine units, knots r [km]; y and per-interval slope for every table.
struct SolarTables
{
	int n = 0;                       // knots (1970 for AGSS09)
	std::vector<double> r;
	std::vector<double> gm, gm_s;    // G*M(r) [km^3/s^2]
	std::vector<double> temp, temp_s;// T(r) [GeV]
	std::vector<double> vesc2, vesc2_s; // v_esc^2 [km^2/s^2]
	std::vector<double> ne, ne_s;    // n_e [1/km^3]
	std::vector<double> nt, nt_s;    // n_i [1/km^3], node-major n x DMS_NUM_TARGETS
	double target_mass_gev[DMS_NUM_TARGETS];
	// bucket acceleration of the knot search: bucket b covers [b, b+1) * rsun / nbuckets,
	// bucket_index[b] = knot interval containing the smallest radius the device maps to b;
	// bucket_single_step = 1 when the interval of every radius of a bucket is its base or the
	// base + 1 (no bucket holds two knots)
	int nbuckets = 0;
	int bucket_single_step = 0;
	std::vector<uint16_t> bucket_index;
};

// Loads the solar model file; returns an empty string on success, else the error.
std::string Load_Solar_Tables(const std::string& path, SolarTables& t);

// Piecewise-linear evaluation with the knot search of the tables (largest i with r_i <= x,
// clamped to [0, n-2]).
double Table_Eval(const SolarTables& t, const std::vector<double>& y, const std::vector<double>& s, double x);

// Per-point constants (SI contact, low-mass mode; Standard Halo Model).
struct PointConstants
{
	double m_dm;                     // GeV
	double sigma_target[DMS_NUM_TARGETS]; // km^2
	double sigma_e;                  // km^2
	unsigned int interaction;        // DMS_INTERACTION_*
	double ff_num, ff_m2;            // General form factor: (q_ref^2 + m^2)^2 / m^2, m^2 [GeV^2]
	double q2c[DMS_NUM_TARGETS + 1]; // 4 mu_k^2 / c^2 [GeV^2 s^2 / km^2]; [63] the electron
	double v0, vesc_halo, vobs;      // km/s
	double vel_obs[3];
	double n_esc;
	double avg_speed, eta0;          // halo <v> [km/s], <1/v> [s/km]
	int grid_n;
	double grid_inv_r, grid_inv_v, grid_vmax;
};

std::string Make_Point_Constants(const SolarTables& t, const dms_point_params& p, PointConstants& c);

}	// namespace dms
