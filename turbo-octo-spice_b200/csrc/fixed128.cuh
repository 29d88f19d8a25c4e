// fixed128.cuh — reading the fixed-point sums of the accumulator rows
// ([row][bin][kAccWords], the carry-free format described at kAccWords:
// field f = hi * 2^32 + lo with lo at word f, hi at word 7 + f; the pair
// count at word 14).
#pragma once

#include "xi_kernels.cuh"

namespace tos {

// Field f of one (row, bin) as a signed 128-bit integer.
__device__ __forceinline__ __int128 acc128(const unsigned long long* base, int f) {
  return (__int128)(long long)base[7 + f] * (__int128)4294967296ll + (__int128)base[f];
}

// Store v (|v| < 2^95) as field f of a row kept in the same format.
__device__ __forceinline__ void store128(unsigned long long* base, int f, __int128 v) {
  base[f] = (unsigned long long)v & 0xFFFFFFFFull;
  base[7 + f] = (unsigned long long)(long long)(v >> 32);
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
