#pragma once
// Oracle build shim: see boost/math/oracle_math_shim.hpp.
#include <boost/math/oracle_math_shim.hpp>
