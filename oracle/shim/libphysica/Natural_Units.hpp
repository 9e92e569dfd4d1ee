// Oracle test shim: natural units (hbar = c = k_B = 1, energies in GeV) for compiling the
// reference's own hot-path sources without libphysica.  Values come from the shared constants
// header so the shim, the C oracle and the CUDA engine start from identical numbers.
#ifndef DMS_SHIM_NATURAL_UNITS_HPP
#define DMS_SHIM_NATURAL_UNITS_HPP
#include <iomanip>
#include <iostream>
#include <vector>
#include "../../../include/dms_constants.h"
namespace libphysica
{
class Vector;
namespace natural_units
{
constexpr double GeV = 1.0;
constexpr double MeV = 1.0e-3 * GeV;
constexpr double keV = 1.0e-6 * GeV;
constexpr double eV = 1.0e-9 * GeV;
constexpr double meter = 1.0 / DMS_HBARC_GEV_M;
constexpr double km = 1.0e3 * meter;
constexpr double cm = 1.0e-2 * meter;
constexpr double sec = 1.0 / DMS_HBAR_GEV_S;
constexpr double day = 86400.0 * sec;
constexpr double kg = DMS_GEV_PER_KG * GeV;
constexpr double gram = 1.0e-3 * kg;
constexpr double Kelvin = DMS_KB_GEV_PER_K * GeV;
constexpr double dyne = 1.0e-5 * kg * meter / sec / sec;
constexpr double pb = 1.0e-36 * cm * cm;
constexpr double deg = 3.14159265358979323846 / 180.0;
constexpr double G_Newton = DMS_G_SI * meter * meter * meter / kg / sec / sec;
constexpr double mSun = DMS_MSUN_KG * kg;
constexpr double rSun = DMS_RSUN_KM * km;
constexpr double AU = DMS_AU_KM * km;
constexpr double mProton = DMS_MPROTON_GEV * GeV;
constexpr double mElectron = DMS_MELECTRON_GEV * GeV;
constexpr double mNucleon = DMS_MNUCLEON_GEV * GeV;
constexpr double aEM = 1.0 / 137.035999084;
inline double In_Units(double quantity, double unit) { return quantity / unit; }
std::vector<double> In_Units(const std::vector<double>& quantity, double unit);
Vector In_Units(const Vector& quantity, double unit);
}	// namespace natural_units
}	// namespace libphysica
#endif
