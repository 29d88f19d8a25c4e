// fixed128.cuh — reading the 128-bit fixed-point sums of the accumulator
// rows ([row][bin][kAccWords]: field f's low word at f, high word at 7 + f,
// the pair count at 14).
#pragma once

#include "xi_kernels.cuh"

namespace tos {

// Field f of one (row, bin) as a signed 128-bit integer.
__device__ __forceinline__ __int128 acc128(const unsigned long long* base, int f) {
  return (__int128)(((unsigned __int128)(unsigned long long)base[7 + f] << 64) | base[f]);
}

// Signed 128-bit value as a double with one relative rounding (by magnitude).
__device__ __forceinline__ double i128_double(__int128 v) {
  const bool neg = v < 0;
  const unsigned __int128 m = neg ? (unsigned __int128)(-v) : (unsigned __int128)v;
  const double d = __fma_rn((double)(unsigned long long)(m >> 64), 18446744073709551616.0 /* 2^64 */,
                            (double)(unsigned long long)m);
  return neg ? -d : d;
}

}  // namespace tos
