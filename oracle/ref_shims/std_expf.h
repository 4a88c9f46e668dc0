// Shim for building the reference's CPU code with g++ 13 (TEST INFRASTRUCTURE ONLY):
// libstdc++ 13 lacks std::expf / std::logf, which the reference's host spectral code names.
#pragma once
#include <cmath>
namespace std {
inline float expf(float x) { return ::expf(x); }
inline float logf(float x) { return ::logf(x); }
}  // namespace std
