// Oracle test shim: nothing beyond <cmath> is used from libphysica's special functions.
#ifndef DMS_SHIM_SPECIAL_FUNCTIONS_HPP
#define DMS_SHIM_SPECIAL_FUNCTIONS_HPP
#include <cmath>
#include "Linear_Algebra.hpp"
#include "Utilities.hpp"
#endif
