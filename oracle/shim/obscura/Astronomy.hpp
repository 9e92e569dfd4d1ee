#ifndef DMS_SHIM_ASTRONOMY_HPP
#define DMS_SHIM_ASTRONOMY_HPP
#include "../libphysica/Linear_Algebra.hpp"
namespace obscura
{
// Solar velocity in the galactic rest frame (only used for isoreflection rings).
libphysica::Vector Sun_Velocity();
}
#endif
