// Oracle test shim: the spin-independent contact DM particle in low-mass mode.
//   sigma_N  = sigma_p * (mu_N / mu_p)^2 * [Z + (f_n/f_p)(A - Z)]^2   (no form factor)
//   sigma_e  = constant
//   scattering angle: isotropic, cos(alpha) = Sample_Uniform(PRNG, -1, 1) (one draw)
// These are the standard SI contact formulas; the reference delegates them to obscura
// (call sites src/Solar_Model.cpp:277, 301 and src/Simulation_Trajectory.cpp:1265).
#ifndef DMS_SHIM_DM_PARTICLE_HPP
#define DMS_SHIM_DM_PARTICLE_HPP
#include <random>
#include <string>
#include "../libphysica/Natural_Units.hpp"
#include "Target_Nucleus.hpp"
namespace obscura
{
class DM_Particle
{
  public:
	double mass = 10.0 * libphysica::natural_units::GeV;
	double spin = 0.5;
	double fractional_density = 1.0;
	bool low_mass = true;
	virtual ~DM_Particle() {}
	void Set_Mass(double m) { mass = m; }
	void Set_Spin(double s) { spin = s; }
	void Set_Fractional_Density(double f) { fractional_density = f; }
	void Set_Low_Mass_Mode(bool l) { low_mass = l; }
	virtual double Sigma_Proton() const { return 0.0; }
	virtual double Sigma_Electron() const { return 0.0; }
	virtual double Get_Interaction_Parameter(const std::string& target) const { return target == "Electrons" ? Sigma_Electron() : Sigma_Proton(); }
	virtual double Sigma_Total_Nucleus(const Isotope& target, double vDM, double param = -1.0) = 0;
	virtual double Sigma_Total_Electron(double vDM, double param = -1.0) = 0;
	virtual double Sample_Scattering_Angle_Nucleus(std::mt19937& PRNG, const Isotope& target, double vDM, double param = -1.0) = 0;
	virtual double Sample_Scattering_Angle_Electron(std::mt19937& PRNG, double vDM, double param = -1.0) = 0;
};
}	// namespace obscura
#endif
