// Oracle test shim: of libphysica's special functions only the reduced mass is used.
#ifndef DMS_SHIM_SPECIAL_FUNCTIONS_HPP
#define DMS_SHIM_SPECIAL_FUNCTIONS_HPP
#include <cmath>
#include "Linear_Algebra.hpp"
#include "Utilities.hpp"
namespace libphysica
{
inline double Reduced_Mass(double m1, double m2) { return m1 * m2 / (m1 + m2); }
}	// namespace libphysica
#endif
