// Test-infrastructure shim for the absent Boost.Multiprecision: the reference carries
// only its final extraction/sum in cpp_dec_float_100 (Twisty/CombinedWeightUtils.h:160-174,
// Twisty/FullExperimentRunnerOptimalPerturb.cpp:232-378). x87 long double (64-bit
// mantissa, range to 1e4932) stands in: enough range for weights of 1e951 and beyond.
#pragma once
#include <cmath>
namespace boost {
namespace multiprecision {
typedef long double cpp_dec_float_100;
typedef long double cpp_dec_float_50;
inline long double log10(long double x) { return std::log10(x); }
inline long double pow(long double b, long double e) { return std::pow(b, e); }
inline long double exp(long double x) { return std::exp(x); }
}  // namespace multiprecision
}  // namespace boost
