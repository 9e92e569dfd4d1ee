// Run configuration: a libconfig-subset parser and the run keys of the reference's
// Configuration class (src/Parameter_Scan.cpp:63-471) for the "Capture" and
// "Parameter point" run modes.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace dms
{

// A parsed value: number (integer or float), string, boolean or list.
struct ConfigValue
{
	enum Kind
	{
		Number,
		String,
		Boolean,
		List
	} kind = Number;
	double number = 0.0;
	bool is_integer = false;
	std::string text;
	bool boolean = false;
	std::vector<ConfigValue> items;
};

// Parses `name = value;` settings with numbers (1, 1.0e-3, 10L), strings, true/false,
// lists "( ... )" and lists of lists, and //, /* */ and # comments.  Returns an empty
// string on success, else a message naming the line.
std::string Parse_Config(const std::string& text, std::map<std::string, ConfigValue>& out);

struct RunConfig
{
	std::string id;
	std::string run_mode;          // "Parameter point" or "Capture"
	bool capture_mode = false;
	uint32_t sample_size = 0;
	uint32_t fixed_seed = 0;
	uint32_t max_trajectories = 0; // 0 = unlimited
	uint32_t interpolation_points = 0;
	uint32_t isoreflection_rings = 1;
	uint64_t maximum_number_of_scatterings = 100000000000000ULL;
	double max_trajectory_wall_time_sec = 0.0;
	bool snapshot_enabled = false;
	double snapshot_interval = 60.0;  // seconds; the reference's default when snapshots are on
	std::string output_dir = "./";
	// DM particle (low-mass mode: SI contact or dark photon)
	double DM_mass_gev = 0.0;
	double DM_spin = 0.5;
	double DM_fraction = 1.0;
	bool DM_light = true;
	std::string DM_interaction;
	bool DM_isospin_conserved = true;
	double fn_over_fp = 1.0;
	double sigma_nucleon_cm2 = 0.0;
	double sigma_electron_cm2 = 0.0;
	std::string DM_form_factor = "Contact";
	unsigned int interaction = 0;       // DMS_INTERACTION_*
	double mediator_mass_mev = 0.0;     // DM_mediator_mass (dark photon, General form factor)
	// halo
	double rho_local = 0.4;
	double v0 = 220.0, vesc = 544.0;
	double vobs[3] = {11.1, 232.2, 7.3};
};

// Reads and validates a configuration file; returns an empty string on success, else the
// reference's error text for the first invalid or missing key.
std::string Load_Run_Config(const std::string& path, RunConfig& cfg);

}	// namespace dms
