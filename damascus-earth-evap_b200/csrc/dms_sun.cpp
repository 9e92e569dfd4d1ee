// dms_sun <config.cfg> — drop-in for the reference executable's "Capture" and
// "Parameter point" run modes (src/main.cpp:20-140) on one GPU: reads the libconfig run file,
// builds the solar model and the point's rate grid on the device, runs the trajectory Monte
// Carlo until the captured sample is complete, prints the reference summary and (Parameter
// point) writes results_<log10 m>_<log10 sigma>/bincount.txt and evaporation_times.txt.
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <iostream>
#include <string>

#include "../../include/dms.h"
#include "../../include/dms_driver.h"
#include "dms_config.h"

int main(int argc, char* argv[])
{
	if(argc < 2)
	{
		std::cerr << "Usage: " << argv[0] << " <config.cfg> [--device N] [--solar-model path]" << std::endl;
		return 1;
	}
	int device = 0;
	std::string solar = "";
	for(int i = 2; i + 1 < argc; i++)
	{
		if(std::strcmp(argv[i], "--device") == 0)
			device = std::atoi(argv[++i]);
		else if(std::strcmp(argv[i], "--solar-model") == 0)
			solar = argv[++i];
	}
	if(solar.empty())
	{
		// data/model_agss09.dat beside the library (the reference reads it from its project dir)
		std::string self = argv[0];
		const size_t slash = self.find_last_of('/');
		const std::string dir = (slash == std::string::npos) ? "." : self.substr(0, slash);
		solar = dir + "/data/model_agss09.dat";
	}
	const auto start = std::chrono::system_clock::now();
	const std::time_t start_t = std::chrono::system_clock::to_time_t(start);
	std::string when = std::ctime(&start_t);
	if(!when.empty() && when.back() == '\n')
		when.pop_back();
	std::cout << "[Started on " << when << "]" << std::endl << "DaMaSCUS-SUN (B200 engine)" << std::endl << "GPU device:\t" << device << std::endl;

	dms::RunConfig cfg;
	const std::string err = dms::Load_Run_Config(argv[1], cfg);
	if(!err.empty())
	{
		std::cerr << err << std::endl;
		return EXIT_FAILURE;
	}
	dms_ctx* ctx = nullptr;
	if(dms_create(&ctx, device) != DMS_OK)
	{
		std::cerr << "Error: no usable CUDA device " << device << "." << std::endl;
		return EXIT_FAILURE;
	}
	auto fail = [&](const char* what) {
		std::cerr << "Error in " << what << ": " << dms_last_error(ctx) << std::endl;
		dms_destroy(ctx);
		return EXIT_FAILURE;
	};
	if(dms_load_solar_model(ctx, solar.c_str()) != DMS_OK)
		return fail("dms_load_solar_model");
	dms_point_params p;
	std::memset(&p, 0, sizeof p);
	p.mass_gev = cfg.DM_mass_gev;
	p.sigma_p_cm2 = cfg.sigma_nucleon_cm2;
	p.sigma_e_cm2 = cfg.sigma_electron_cm2;
	p.fn_over_fp = cfg.fn_over_fp;
	p.halo_v0_kms = cfg.v0;
	p.halo_vesc_kms = cfg.vesc;
	for(int i = 0; i < 3; i++) p.halo_vobs_kms[i] = cfg.vobs[i];
	p.interpolation_points = cfg.interpolation_points;
	p.interaction = cfg.interaction;
	p.mediator_mass_mev = cfg.mediator_mass_mev;
	int pid = -1;
	std::cout << (cfg.capture_mode ? "Generate data in CAPTURE MODE..." : "Generate data...") << std::endl
	          << "\tm_DM [MeV]:\t" << cfg.DM_mass_gev * 1000.0 << "\t\tsigma_p [cm2]:\t" << cfg.sigma_nucleon_cm2 << std::endl
	          << "\tu_min [km/sec]:\t0\t\tsigma_e [cm2]:\t" << cfg.sigma_electron_cm2 << std::endl
	          << std::endl;
	if(dms_add_point(ctx, &p, &pid) != DMS_OK)
		return fail("dms_add_point");
	dms_generate_opts g;
	dms_default_generate_opts(&g);
	g.sample_size = cfg.sample_size;
	g.max_trajectories = cfg.max_trajectories;
	g.seed = cfg.fixed_seed;
	g.capture_mode = cfg.capture_mode ? 1 : 0;
	g.max_scatterings = cfg.maximum_number_of_scatterings;
	g.sigma_p_cm2 = cfg.sigma_nucleon_cm2;
	g.max_trajectory_wall_time_s = cfg.max_trajectory_wall_time_sec;
	g.print_progress = 1;
	// output path, src/main.cpp:89-92 (std::to_string of log10 values); snapshots go to its
	// snapshot/ folder (src/Data_Generation.cpp:522-529)
	const std::string out = cfg.output_dir + "results_" + std::to_string(std::log10(cfg.DM_mass_gev)) + "_" +
	                        std::to_string(std::log10(cfg.sigma_nucleon_cm2)) + "/";
	const std::string snapshot_dir = out + "snapshot/";
	if(cfg.snapshot_enabled && !cfg.capture_mode)
	{
		g.snapshot_dir = snapshot_dir.c_str();
		g.snapshot_interval_s = cfg.snapshot_interval;
		g.snapshot_mass_gev = cfg.DM_mass_gev;
		g.snapshot_sigma_cm2 = cfg.sigma_nucleon_cm2;
	}
	dms_generate_summary s;
	if(dms_generate_data(ctx, pid, &g, &s) != DMS_OK)
		return fail("dms_generate_data");
	dms_print_summary(ctx, pid, &s, g.capture_mode);
	if(!cfg.capture_mode)
	{
		if(dms_write_outputs(ctx, pid, &s, cfg.DM_mass_gev, cfg.sigma_nucleon_cm2, out.c_str()) != DMS_OK)
			std::cerr << "Warning: failed to write the output files into " << out << std::endl;
		// reflection spectrum, src/main.cpp:95-99
		dms_reflection_spectrum spectrum;
		if(cfg.isoreflection_rings == 1 && dms_get_reflection_spectrum(ctx, pid, 1, 0, cfg.rho_local, &spectrum) == DMS_OK &&
		   spectrum.reflections > 0)
			dms_print_reflection_summary(&spectrum);
	}
	dms_destroy(ctx);
	const double total = std::chrono::duration<double>(std::chrono::system_clock::now() - start).count();
	std::cout << "\n[Finished in " << total << " s]" << std::endl;
	return 0;
}
