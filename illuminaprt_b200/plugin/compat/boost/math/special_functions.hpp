#pragma once
#include <cmath>
namespace boost { namespace math { inline double erf(double x) { return std::erf(x); } inline double erfc(double x) { return std::erfc(x); } using std::isnan; } }
