// ytf_digits.cuh -- the fixed-point digit form of the int8x3 Bessel contraction's operands:
// a value v of a column whose largest |v| is m becomes Y = rint(v * BI_SCALE / m) (< 2^23),
// written as three signed base-256 digits d0 d1 d2 (Y = 65536 d0 + 256 d1 + d2, each digit in
// [-128, 127]); the MMA sums the six digit products exactly in INT32.
#pragma once
#include <cstdint>

namespace ytf {

constexpr double BI_SCALE = 8355000.0;
constexpr int BI_NODES = 64;  // nodes per pipeline stage: one byte each, 64-byte rows

__device__ __forceinline__ void digits3b(int Y, uint32_t& d0, uint32_t& d1, uint32_t& d2) {
  d2 = (uint32_t)Y & 255u;
  d1 = (uint32_t)((Y + 128) >> 8) & 255u;
  d0 = (uint32_t)((Y + 32896) >> 16) & 255u;
}

// the digit scale of a column from its maximum's IEEE bits (0 for an empty or non-finite column)
__device__ __forceinline__ double col_scale(unsigned long long bits) {
  const double m = __longlong_as_double((long long)bits);
  return (m > 0.0 && isfinite(m)) ? BI_SCALE / m : 0.0;
}

}  // namespace ytf
