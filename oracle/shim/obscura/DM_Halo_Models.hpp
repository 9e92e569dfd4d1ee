// Oracle test shim: Standard Halo Model -- a Maxwell-Boltzmann velocity distribution of
// dispersion v0, truncated at the galactic escape speed v_esc, seen from an observer moving
// with velocity v_obs (DM velocity v in the observer frame <-> v + v_obs in the galactic frame):
//   f(v_vec) = exp(-|v + v_obs|^2 / v0^2) / (N_esc pi^(3/2) v0^3)  for |v + v_obs| <= v_esc
//   N_esc    = erf(z) - 2 z exp(-z^2)/sqrt(pi),  z = v_esc / v0
//   f(v)     = v/(N_esc sqrt(pi) v0 |v_obs|) * [exp(-(v-|v_obs|)^2/v0^2) - exp(-min((v+|v_obs|)^2, v_esc^2)/v0^2)]
//              for 0 <= v <= v_esc + |v_obs|.
// Average_Speed() = int v f(v) dv and Eta_Function(0) = int f(v)/v dv are evaluated with
// 256-panel composite 7-point Gauss-Legendre on [0, v_esc-|v_obs|] and [v_esc-|v_obs|, v_esc+|v_obs|].
#ifndef DMS_SHIM_DM_HALO_MODELS_HPP
#define DMS_SHIM_DM_HALO_MODELS_HPP
#include "DM_Distribution.hpp"
namespace obscura
{
class Standard_Halo_Model : public DM_Distribution
{
	double v_0, v_esc, v_obs;
	libphysica::Vector vel_observer;
	double N_esc;

  public:
	Standard_Halo_Model(double v0, double vesc, const libphysica::Vector& vobs);
	libphysica::Vector Get_Observer_Velocity() const { return vel_observer; }
	double PDF_Velocity(const libphysica::Vector& vel) override;
	double PDF_Speed(double v) override;
	double Minimum_DM_Speed() const override { return 0.0; }
	double Maximum_DM_Speed() const override { return v_esc + v_obs; }
	double Average_Speed(double vMin = -1.0) override;
	double Eta_Function(double vMin) override;
};
}	// namespace obscura
#endif
