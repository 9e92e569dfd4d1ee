// Oracle test shim: one-dimensional tabulated function with piecewise-linear interpolation.
//   i = largest knot index with x_i <= x, clamped to [0, N-2];
//   y(x) = y_i + (x - x_i) * s_i,   s_i = (y_{i+1} - y_i) / (x_{i+1} - x_i).
// Piecewise-linear interpolation is what the reference's own tests pin: a density that is
// flat between the padded r=0 row and the first data row must be returned exactly at
// r = 0.001 R_sun (tests/test_Solar_Model.cpp:30-41), which a global spline would not do.
#ifndef DMS_SHIM_NUMERICS_HPP
#define DMS_SHIM_NUMERICS_HPP
#include <vector>
#include "Linear_Algebra.hpp"
namespace libphysica
{
class Interpolation
{
	std::vector<double> xs, ys, slopes;
	void Compute_Slopes();

  public:
	Interpolation() {}
	explicit Interpolation(const std::vector<std::vector<double>>& table, double dim1 = -1.0, double dim2 = -1.0);
	double operator()(double x) const;
	void Multiply(double factor);
	const std::vector<double>& Knots() const { return xs; }
};
}	// namespace libphysica
#endif
