// Oracle test shim: definite integral used by the reference only for the escape-speed table
// (src/Solar_Model.cpp:79-96, integrand Mass(x)/x^2 with integrand(0) = 0).
// Rule: the interval is split at the knots of the most recently constructed Interpolation;
// on each piece [a,b] the integrand is written as g(x)/x^2 with g linear between the piece
// ends (g(a) = f(a) a^2, g(b) = f(b) b^2) and integrated exactly,
//   (g_a - s a)(1/a - 1/b) + s ln(b/a),   s = (g_b - g_a)/(b - a);
// a piece that starts at x = 0 uses the trapezoid rule with the integrand's own value at 0.
// This is exact for the piecewise-linear mass profile and reproduces the reference KAT
// v_esc(0) = 1384.13 +- 0.1 km/s (tests/test_Solar_Model.cpp:73-81).
#ifndef DMS_SHIM_INTEGRATION_HPP
#define DMS_SHIM_INTEGRATION_HPP
#include <functional>
#include <string>
namespace libphysica
{
double Integrate(std::function<double(double)> func, double a, double b, const std::string& method = "");
}	// namespace libphysica
#endif
