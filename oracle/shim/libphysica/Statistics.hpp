// Oracle test shim: sampling helpers.  All uniform draws come from the engine's draw stream
// (include/dms_philox.h) selected by dms_shim_set_stream(); the std::mt19937 argument is
// accepted for source compatibility and ignored.
//   Sample_Uniform(PRNG, a, b) = a + u * (b - a),  u in [0,1)
//   Rejection_Sampling: repeat { x = Sample_Uniform(xMin, xMax); y = Sample_Uniform(0, yMax) }
//                       until y <= PDF(x); two draws per attempt, x first.
#ifndef DMS_SHIM_STATISTICS_HPP
#define DMS_SHIM_STATISTICS_HPP
#include <functional>
#include <random>
#include "Linear_Algebra.hpp"
#include "Utilities.hpp"
namespace libphysica
{
double Sample_Uniform(std::mt19937& PRNG, double x_min = 0.0, double x_max = 1.0);
double Rejection_Sampling(const std::function<double(double)>& PDF, double xMin, double xMax, double yMax, std::mt19937& PRNG);
struct DataPoint
{
	double value;
	double weight;
	DataPoint(double v = 0.0, double w = 1.0) : value(v), weight(w) {}
	bool operator<(const DataPoint& o) const { return value < o.value; }
};
}	// namespace libphysica
#endif
