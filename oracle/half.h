// half.h — IEEE 754 binary16 conversions for the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY (see pyro_oracle.cpp).  The renderer's textures
// are rgba16float; their stores convert binary32 to binary16 with round to
// nearest, ties to even (pinned against numpy's float16 in the tests).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

namespace oracle_half {

// binary32 -> binary16, round to nearest, ties to even; finite values that
// round past 65504 give infinity; NaN stays a (quiet) NaN.
inline uint16_t f32_to_f16(float f) {
  uint32_t x;
  std::memcpy(&x, &f, 4);
  const uint16_t sign = (uint16_t)((x >> 16) & 0x8000u);
  const uint32_t ax = x & 0x7fffffffu;
  if (ax > 0x7f800000u) return sign | 0x7e00u;   // NaN
  if (ax >= 0x477ff000u) return sign | 0x7c00u;  // >= 65520 (or inf): infinity
  const int e = (int)(ax >> 23) - 127;           // unbiased exponent
  const uint32_t mant = ax & 0x7fffffu;
  if (e >= -14) {  // normal binary16: keep 10 of the 23 fraction bits
    uint32_t h = ((uint32_t)(e + 15) << 10) | (mant >> 13);
    const uint32_t r = mant & 0x1fffu;
    if (r > 0x1000u || (r == 0x1000u && (h & 1u))) h++;  // a carry moves into the exponent
    return sign | (uint16_t)h;
  }
  // subnormal binary16 (units of 2^-24): significand 1.mant shifted right
  const int shift = -(e + 1);  // >= 14
  if (shift > 24) return sign;  // below 2^-25: rounds to zero
  const uint32_t m = 0x800000u | mant;
  uint32_t h = m >> shift;
  const uint32_t r = m & ((1u << shift) - 1u), half = 1u << (shift - 1);
  if (r > half || (r == half && (h & 1u))) h++;
  return sign | (uint16_t)h;
}

inline float f16_to_f32(uint16_t h) {
  const int e = (h >> 10) & 0x1f;
  const uint32_t m = h & 0x3ffu;
  float v;
  if (e == 0) v = std::ldexp((float)m, -24);
  else if (e == 31) v = m ? NAN : INFINITY;
  else v = std::ldexp((float)(m | 0x400u), e - 25);
  return (h & 0x8000u) ? -v : v;
}

}  // namespace oracle_half
