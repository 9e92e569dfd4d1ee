// Oracle test shim: obscura's DM particle interface (the base class of the reference's dark
// photon, include/Dark_Photon.hpp) and the spin-independent contact DM particle in low-mass mode.
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
// Electron-target types of obscura's interface: only their names are needed here (the
// ionization and crystal cross sections are not on the trajectory path).
struct Atomic_Electron
{
	double Ionization_Form_Factor(double, double) const { return 0.0; }
};
struct Crystal
{
	double Crystal_Form_Factor(double, double) const { return 0.0; }
};

class DM_Particle
{
  public:
	double mass = 10.0 * libphysica::natural_units::GeV;
	double spin = 0.5;
	double fractional_density = 1.0;
	bool low_mass = true;
	bool using_cross_section = false;
	bool DD_use_eta_function = false;
	DM_Particle() {}
	explicit DM_Particle(double m) : mass(m) {}
	virtual ~DM_Particle() {}
	virtual void Set_Mass(double m) { mass = m; }
	void Set_Spin(double s) { spin = s; }
	void Set_Fractional_Density(double f) { fractional_density = f; }
	void Set_Low_Mass_Mode(bool l) { low_mass = l; }
	virtual double Sigma_Proton() const { return 0.0; }
	virtual double Sigma_Neutron() const { return Sigma_Proton(); }
	virtual double Sigma_Electron() const { return 0.0; }
	virtual double Get_Interaction_Parameter(std::string target) const { return target == "Electrons" ? Sigma_Electron() : Sigma_Proton(); }
	virtual void Set_Interaction_Parameter(double par, std::string target)
	{
		if(target == "Electrons")
			Set_Sigma_Electron(par);
		else
			Set_Sigma_Proton(par);
	}
	virtual void Set_Sigma_Proton(double) {}
	virtual void Set_Sigma_Electron(double) {}
	virtual double dSigma_dq2_Nucleus(double, const Isotope&, double, double = -1.0) const { return 0.0; }
	virtual double dSigma_dq2_Electron(double, double, double = -1.0) const { return 0.0; }
	virtual double d2Sigma_dq2_dEe_Ionization(double, double, double, Atomic_Electron&) const { return 0.0; }
	virtual double d2Sigma_dq2_dEe_Crystal(double, double, double, Crystal&) const { return 0.0; }
	virtual double Sigma_Total_Nucleus(const Isotope& target, double vDM, double param = -1.0) = 0;
	virtual double Sigma_Total_Electron(double vDM, double param = -1.0) = 0;
	virtual double PDF_Scattering_Angle_Nucleus(double, const Isotope&, double, double = -1.0) { return 0.5; }
	virtual double PDF_Scattering_Angle_Electron(double, double, double = -1.0) { return 0.5; }
	virtual double CDF_Scattering_Angle_Nucleus(double cos_alpha, const Isotope&, double, double = -1.0) { return (1.0 + cos_alpha) / 2.0; }
	virtual double CDF_Scattering_Angle_Electron(double cos_alpha, double, double = -1.0) { return (1.0 + cos_alpha) / 2.0; }
	virtual double Sample_Scattering_Angle_Nucleus(std::mt19937& PRNG, const Isotope& target, double vDM, double param = -1.0) = 0;
	virtual double Sample_Scattering_Angle_Electron(std::mt19937& PRNG, double vDM, double param = -1.0) = 0;
	virtual void Print_Summary(int = 0) const {}

  protected:
	// The nuclear-form-factor ("high mass") forms: not shimmed, the engine runs in low-mass mode.
	void Print_Summary_Base(int = 0) const {}
	double Sigma_Total_Nucleus_Base(const Isotope&, double, double = -1.0) { return High_Mass_Not_Shimmed(); }
	double PDF_Scattering_Angle_Nucleus_Base(double, const Isotope&, double, double = -1.0) { return High_Mass_Not_Shimmed(); }
	double CDF_Scattering_Angle_Nucleus_Base(double, const Isotope&, double, double = -1.0) { return High_Mass_Not_Shimmed(); }
	double Sample_Scattering_Angle_Nucleus_Base(std::mt19937&, const Isotope&, double, double = -1.0) { return High_Mass_Not_Shimmed(); }
	static double High_Mass_Not_Shimmed();
};
}	// namespace obscura
#endif
