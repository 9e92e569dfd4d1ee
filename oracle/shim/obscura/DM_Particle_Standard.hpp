#ifndef DMS_SHIM_DM_PARTICLE_STANDARD_HPP
#define DMS_SHIM_DM_PARTICLE_STANDARD_HPP
#include "DM_Particle.hpp"
namespace obscura
{
class DM_Particle_SI : public DM_Particle
{
	double sigma_proton = 0.0;
	double sigma_electron = 0.0;
	double fn_over_fp = 1.0;

  public:
	DM_Particle_SI() {}
	explicit DM_Particle_SI(double m) { mass = m; }
	void Set_Sigma_Proton(double s) { sigma_proton = s; }
	void Set_Sigma_Electron(double s) { sigma_electron = s; }
	void Set_Sigma_Neutron(double) {}
	void Fix_Coupling_Ratio(double fp, double fn) { fn_over_fp = fn / fp; }
	void Unfix_Coupling_Ratios() {}
	double Sigma_Proton() const override { return sigma_proton; }
	double Sigma_Electron() const override { return sigma_electron; }
	double Sigma_Total_Nucleus(const Isotope& target, double vDM, double param = -1.0) override;
	double Sigma_Total_Electron(double vDM, double param = -1.0) override;
	double Sample_Scattering_Angle_Nucleus(std::mt19937& PRNG, const Isotope& target, double vDM, double param = -1.0) override;
	double Sample_Scattering_Angle_Electron(std::mt19937& PRNG, double vDM, double param = -1.0) override;
};
}	// namespace obscura
#endif
