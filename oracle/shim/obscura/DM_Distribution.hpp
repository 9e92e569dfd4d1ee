#ifndef DMS_SHIM_DM_DISTRIBUTION_HPP
#define DMS_SHIM_DM_DISTRIBUTION_HPP
#include "../libphysica/Linear_Algebra.hpp"
namespace obscura
{
class DM_Distribution
{
  public:
	virtual ~DM_Distribution() {}
	virtual double PDF_Velocity(const libphysica::Vector& vel) = 0;
	virtual double PDF_Speed(double v) = 0;
	virtual double Minimum_DM_Speed() const = 0;
	virtual double Maximum_DM_Speed() const = 0;
	virtual double Average_Speed(double vMin = -1.0) = 0;
	virtual double Eta_Function(double vMin) = 0;
};
}	// namespace obscura
#endif
