// Reference build of the oracle: a C-callable driver around the reference's OWN hot-path
// classes (compiled unmodified from the reference sources against the shims in oracle/shim).
// Test infrastructure: used by tests/ to pin the C oracle, and as the timed reference arm
// of bench.py.  Never linked into the engine.
//
// Per trajectory it performs exactly what simulate_one_trajectory does
// (src/Data_Generation.cpp:745-861): Initial_Conditions, Hyperbolic_Kepler_Shift to the
// boundary radius, Trajectory_Simulator::Simulate, then the free / reflected / captured
// classification, with every uniform draw taken from the engine's Philox stream keyed by
// (seed, point, trajectory id).
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <limits>
#include <memory>
#include <string>

#include "Dark_Photon.hpp"
#include "Data_Generation.hpp"
#include "Simulation_Trajectory.hpp"
#include "Simulation_Utilities.hpp"
#include "Solar_Model.hpp"
#include "obscura/Astronomy.hpp"
#include "obscura/DM_Halo_Models.hpp"
#include "obscura/DM_Particle_Standard.hpp"

#include "../include/dms.h"
#include "shim/shim_control.h"

std::string g_top_level_dir = "./";

using namespace DaMaSCUS_SUN;
using namespace libphysica::natural_units;

namespace
{
std::unique_ptr<Solar_Model> g_ssm;
std::unique_ptr<obscura::DM_Particle> g_dm;
std::unique_ptr<obscura::Standard_Halo_Model> g_halo;
std::string g_error;

void To_Engine(const Event& e, double& t, double x[3], double v[3])
{
	t = In_Units(e.time, sec);
	for(int i = 0; i < 3; i++)
	{
		x[i] = In_Units(e.position[i], km);
		v[i] = In_Units(e.velocity[i], km / sec);
	}
}

double Seconds_Or_Nan(double t) { return t; }
}	// namespace

extern "C" {

const char* dms_ref_last_error(void) { return g_error.c_str(); }

int dms_ref_init(void)
{
	try
	{
		g_ssm.reset(new Solar_Model());
		return 0;
	}
	catch(const std::exception& e)
	{
		g_error = e.what();
		return -1;
	}
}

int dms_ref_num_targets(void) { return g_ssm ? static_cast<int>(g_ssm->target_isotopes.size()) : -1; }

int dms_ref_set_point(const dms_point_params* p)
{
	if(!g_ssm)
		return -1;
	try
	{
		if(p->interaction == DMS_INTERACTION_SI)
		{
			auto* si = new obscura::DM_Particle_SI(p->mass_gev * GeV);
			g_dm.reset(si);
			si->Set_Low_Mass_Mode(true);
			si->Set_Sigma_Proton(p->sigma_p_cm2 * cm * cm);
			si->Set_Sigma_Electron(p->sigma_e_cm2 * cm * cm);
			si->Fix_Coupling_Ratio(1.0, p->fn_over_fp);
		}
		else
		{
			// the steps of Configuration::Construct_DM_Particle for "Dark photon"
			// (src/Parameter_Scan.cpp:386-471, 473-520)
			auto* dp = new DM_Particle_Dark_Photon();
			g_dm.reset(dp);
			const bool general = p->interaction == DMS_INTERACTION_DARK_PHOTON_GENERAL;
			dp->Set_FormFactor_DM(general ? "General" : "Contact", general ? p->mediator_mass_mev * MeV : -1.0);
			dp->Set_Interaction_Parameter(p->sigma_e_cm2 * cm * cm, "Electrons");
			dp->Set_Mass(p->mass_gev * GeV);
			dp->Set_Low_Mass_Mode(true);
		}
		libphysica::Vector vobs({p->halo_vobs_kms[0] * km / sec, p->halo_vobs_kms[1] * km / sec, p->halo_vobs_kms[2] * km / sec});
		g_halo.reset(new obscura::Standard_Halo_Model(p->halo_v0_kms * km / sec, p->halo_vesc_kms * km / sec, vobs));
		g_ssm->Interpolate_Total_DM_Scattering_Rate(*g_dm, p->interpolation_points, p->interpolation_points);
		return 0;
	}
	catch(const std::exception& e)
	{
		g_error = e.what();
		return -1;
	}
}

// Table and rate queries in engine units (r in km, v in km/s, T in K, densities in 1/km^3,
// rates in 1/s, speeds in km/s).
//   what: 0 G*M(r) [km^3/s^2]  1 T(r) [K]  2 v_esc(r) [km/s]  3 n_e(r)  4 n_i(r) (b = i)
//         5 total rate (interpolated path)  6 total rate computed  7 <v_rel>(T=a [K], m=b [GeV], v) -> uses c
//         8 halo PDF_Speed(v=a) [s/km]  9 halo Average_Speed [km/s]  10 halo Eta(0) [s/km]
//         11 target mass [GeV] (a = i)  12 rate of target i (b = i, -1 = electron) at r = a, v = c
double dms_ref_query(int what, double a, double b, double c)
{
	if(!g_ssm)
		return std::numeric_limits<double>::quiet_NaN();
	Solar_Model& s = *g_ssm;
	switch(what)
	{
		case 0: return In_Units(G_Newton * s.Mass(a * km), km * km * km / sec / sec);
		case 1: return In_Units(s.Temperature(a * km), Kelvin);
		case 2: return In_Units(s.Local_Escape_Speed(a * km), km / sec);
		case 3: return In_Units(s.Number_Density_Electron(a * km), 1.0 / km / km / km);
		case 4: return In_Units(s.Number_Density_Nucleus(a * km, static_cast<unsigned int>(b)), 1.0 / km / km / km);
		case 5: return In_Units(s.Total_DM_Scattering_Rate(*g_dm, a * km, b * km / sec), 1.0 / sec);
		case 6: return In_Units(s.Total_DM_Scattering_Rate_Computed(*g_dm, a * km, b * km / sec), 1.0 / sec);
		case 7: return In_Units(Thermal_Averaged_Relative_Speed(a * Kelvin, b * GeV, c * km / sec), km / sec);
		case 8: return g_halo->PDF_Speed(a * km / sec) * (km / sec);
		case 9: return In_Units(g_halo->Average_Speed(), km / sec);
		case 10: return g_halo->Eta_Function(0.0) * (km / sec);
		case 11: return In_Units(s.target_isotopes[static_cast<unsigned int>(a)].mass, GeV);
		case 12:
			if(b < 0.0)
				return In_Units(s.DM_Scattering_Rate_Electron(*g_dm, a * km, c * km / sec), 1.0 / sec);
			return In_Units(s.DM_Scattering_Rate_Nucleus(*g_dm, a * km, c * km / sec, static_cast<unsigned int>(b)), 1.0 / sec);
		default: return std::numeric_limits<double>::quiet_NaN();
	}
}

}	// extern "C"

namespace
{
int Run_Records(uint32_t seed, uint32_t point, int capture_mode, uint64_t max_scatterings, double boundary_rsun, uint64_t first,
                uint64_t count, dms_traj_record* records, double* hist_dt, double* hist_v2dt, double* trace,
                size_t trace_capacity, size_t* trace_length, double* reflection);
}

extern "C" {

// One record per trajectory id in [first, first + count).  Optional per-trajectory histograms
// (count * NUM_BINS each) and a scatter trace of the FIRST trajectory: (r_km, v_kms, draw index)
// per scattering, up to trace_capacity triples.
int dms_ref_run_records(uint32_t seed, uint32_t point, int capture_mode, uint64_t max_scatterings, double boundary_rsun,
                        uint64_t first, uint64_t count, dms_traj_record* records, double* hist_dt, double* hist_v2dt,
                        double* trace, size_t trace_capacity, size_t* trace_length)
{
	return Run_Records(seed, point, capture_mode, max_scatterings, boundary_rsun, first, count, records, hist_dt, hist_v2dt,
	                   trace, trace_capacity, trace_length, nullptr);
}

// The records, and for every reflected particle whose final Kepler shift to 1 AU succeeded the
// reflection-spectrum sample of src/Data_Generation.cpp:824-840: reflection[2k] = its speed at
// 1 AU [km/s], reflection[2k+1] = the cosine of the angle between its position at 1 AU and the
// Sun's velocity (the quantity Isoreflection_Ring bins, src/Simulation_Utilities.cpp:82-92);
// NaN for every other trajectory.
int dms_ref_run_reflections(uint32_t seed, uint32_t point, uint64_t max_scatterings, double boundary_rsun, uint64_t first,
                            uint64_t count, dms_traj_record* records, double* reflection)
{
	return Run_Records(seed, point, 0, max_scatterings, boundary_rsun, first, count, records, nullptr, nullptr, nullptr, 0,
	                   nullptr, reflection);
}

}	// extern "C"

namespace
{
int Run_Records(uint32_t seed, uint32_t point, int capture_mode, uint64_t max_scatterings, double boundary_rsun, uint64_t first,
                uint64_t count, dms_traj_record* records, double* hist_dt, double* hist_v2dt, double* trace,
                size_t trace_capacity, size_t* trace_length, double* reflection)
{
	if(!g_ssm || !g_dm || !g_halo)
		return -1;
	try
	{
		const double R = boundary_rsun * rSun;
		Trajectory_Simulator simulator(*g_ssm, DEFAULT_MAXIMUM_FREE_TIME_STEPS, max_scatterings, R);
		simulator.Enable_Capture_Mode(capture_mode != 0);
		dms_shim_set_tracing(trace != nullptr ? 1 : 0);
		for(uint64_t k = 0; k < count; k++)
		{
			const uint64_t id = first + k;
			dms_shim_set_stream(seed, point, id);
			dms_traj_record& rec = records[k];
			std::memset(&rec, 0, sizeof(rec));
			rec.trajectory_id = id;
			rec.point = point;
			if(reflection)
				reflection[2 * k] = reflection[2 * k + 1] = std::numeric_limits<double>::quiet_NaN();
			Event IC = Initial_Conditions(*g_halo, *g_ssm, simulator.PRNG);
			const bool shift_ok = Hyperbolic_Kepler_Shift(IC, R);
			To_Engine(IC, rec.initial_time, rec.initial_position, rec.initial_velocity);
			if(!shift_ok)
			{
				rec.termination_reason = DMS_REASON_NUMERICAL_FAILURE;
				rec.flags = 0;
				rec.number_of_draws = dms_shim_draw_count();
				To_Engine(IC, rec.final_time, rec.final_position, rec.final_velocity);
				rec.t_capture = -1.0;
				rec.t_last_bound = -1.0;
				rec.t_final_unbinding_scatter = std::numeric_limits<double>::quiet_NaN();
				rec.t_boundary_escape = std::numeric_limits<double>::quiet_NaN();
				rec.t_termination = -1.0;
				rec.lifetime_unbinding = -1.0;
				if(hist_dt) std::memset(hist_dt + k * NUM_BINS, 0, NUM_BINS * sizeof(double));
				if(hist_v2dt) std::memset(hist_v2dt + k * NUM_BINS, 0, NUM_BINS * sizeof(double));
				continue;
			}
			Trajectory_Result result = simulator.Simulate(IC, *g_dm, 0);
			const TrajectoryBincount& bc = result.bincount;
			rec.number_of_scatterings = result.number_of_scatterings;
			rec.termination_reason = static_cast<uint32_t>(bc.termination_reason);
			uint32_t flags = DMS_REC_SHIFT_OK;
			if(bc.is_captured) flags |= DMS_REC_CAPTURED;
			if(bc.event_observed) flags |= DMS_REC_EVENT_OBSERVED;
			if(bc.survival_valid) flags |= DMS_REC_SURVIVAL_VALID;
			if(bc.boundary_escape_observed) flags |= DMS_REC_BOUNDARY_ESCAPE;
			if(bc.numerically_invalid_escape) flags |= DMS_REC_INVALID_ESCAPE;
			if(!bc.is_captured && bc.termination_reason == TrajectoryTerminationReason::OutwardEscape)
			{
				if(result.Particle_Free())
					flags |= DMS_REC_FREE;
				else if(result.Particle_Reflected())
				{
					flags |= DMS_REC_REFLECTED;
					Event final_event = result.final_event;
					if(Hyperbolic_Kepler_Shift(final_event, 1.0 * AU))
					{
						flags |= DMS_REC_REFLECT_SHIFT_OK;
						if(reflection)
						{
							const libphysica::Vector vs = obscura::Sun_Velocity();
							reflection[2 * k] = In_Units(final_event.Speed(), km / sec);
							reflection[2 * k + 1] = final_event.position.Dot(vs) / final_event.position.Norm() / vs.Norm();
						}
					}
				}
			}
			rec.flags = flags;
			rec.number_of_draws = dms_shim_draw_count();
			To_Engine(result.final_event, rec.final_time, rec.final_position, rec.final_velocity);
			rec.t_capture = bc.t_capture;
			rec.t_last_bound = bc.t_last_bound;
			rec.t_final_unbinding_scatter = Seconds_Or_Nan(bc.t_final_unbinding_scatter);
			rec.t_boundary_escape = Seconds_Or_Nan(bc.t_boundary_escape);
			rec.t_termination = bc.t_termination;
			rec.max_free_energy_drift_eV = bc.max_free_energy_drift_eV;
			rec.max_free_energy_drift_rel = bc.max_free_energy_drift_rel;
			const bool invalid_escape = bc.numerically_invalid_escape || bc.termination_reason == TrajectoryTerminationReason::EnergyDriftEscape;
			const bool survival_valid = bc.survival_valid && !invalid_escape;
			const bool observed = survival_valid && bc.event_observed;
			const double lifetime = observed ? bc.t_final_unbinding_scatter - bc.t_capture : -1.0;
			rec.lifetime_unbinding = (bc.is_captured && std::isfinite(lifetime) && lifetime >= 0.0) ? lifetime : -1.0;
			if(hist_dt) std::memcpy(hist_dt + k * NUM_BINS, bc.dt_hist.data(), NUM_BINS * sizeof(double));
			if(hist_v2dt) std::memcpy(hist_v2dt + k * NUM_BINS, bc.v2dt_hist.data(), NUM_BINS * sizeof(double));
			if(trace != nullptr && k == 0)
			{
				const size_t n = dms_shim_trace_size() / 3;
				const double* t = dms_shim_trace_data();
				const size_t m = (n < trace_capacity) ? n : trace_capacity;
				for(size_t i = 0; i < m; i++)
				{
					trace[3 * i + 0] = In_Units(t[3 * i + 0], km);
					trace[3 * i + 1] = In_Units(t[3 * i + 1], km / sec);
					trace[3 * i + 2] = t[3 * i + 2];
				}
				if(trace_length) *trace_length = n;
			}
		}
		dms_shim_set_tracing(0);
		return 0;
	}
	catch(const std::exception& e)
	{
		g_error = e.what();
		return -1;
	}
}
}	// namespace

extern "C" {

// The reference's own ensemble driver, Simulation_Data::Generate_Data + output writers, on one
// process (single-rank MPI shim).  Draws come from one sequential stream keyed by (seed, point).
// Writes bincount.txt / evaporation_times.txt into out_dir in Parameter-point mode and prints the
// reference summary to stdout.
int dms_ref_generate_data(uint32_t seed, uint32_t point, int capture_mode, uint32_t sample_size, uint32_t max_trajectories,
                          uint64_t max_scatterings, const char* out_dir)
{
	if(!g_ssm || !g_dm || !g_halo)
		return -1;
	try
	{
		dms_shim_set_stream(seed, point, ~0ULL);
		Simulation_Data data(sample_size, max_trajectories, 0.0, 1);
		data.Configure(2.0 * rSun, 1, max_scatterings);
		data.Generate_Data(*g_dm, *g_ssm, *g_halo, SnapshotConfig(), seed, capture_mode != 0);
		if(capture_mode)
			data.Print_Capture_Mode_Summary(0);
		else
		{
			data.Print_Summary(0);
			if(out_dir != nullptr)
				data.Write_Output_Files(out_dir, *g_dm);
		}
		return 0;
	}
	catch(const std::exception& e)
	{
		g_error = e.what();
		return -1;
	}
}

}	// extern "C"
