/*
 * philox.cuh - counter-based Philox4x32-10 (Salmon, Moraes, Dror, Shaw,
 * "Parallel random numbers: as easy as 1, 2, 3", SC'11) for the transport
 * kernels.  Counter layout (include/ptrans_gpu.h):
 *   c0 = flight_no, c1 = sub | stream << 8, c2 = lo32(sample), c3 = hi32(sample)
 *   key = (lo32(seed), hi32(seed)).
 */
#ifndef PTG_PHILOX_CUH
#define PTG_PHILOX_CUH

#include <stdint.h>

namespace ptg {

struct Key2 {
  uint32_t k0, k1;
};

__device__ __forceinline__ uint4 philox10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                          Key2 k) {
  uint32_t k0 = k.k0, k1 = k.k1;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    /* one 32x32 -> 64-bit product per multiplier gives both halves */
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    c0 = n0;
    c1 = (uint32_t)p1;
    c2 = n2;
    c3 = (uint32_t)p0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return make_uint4(c0, c1, c2, c3);
}

/* (k + 0.5) * 2^-52 from the top 52 bits of (a,b): open interval (0,1). */
__device__ __forceinline__ double u52d(uint32_t a, uint32_t b) {
  const uint64_t k = ((uint64_t)a << 20) | (uint64_t)(b >> 12);
  return ((double)k + 0.5) * (1.0 / 4503599627370496.0);
}

/* (k + 0.5) * 2^-23 from the low 23 bits k of a: open interval (0,1).
   Built from the bit pattern 1 + k 2^-23 minus (1 - 2^-24), which is exact
   and avoids the integer-to-float conversion pipe. */
__device__ __forceinline__ float u23f(uint32_t a) {
  return __uint_as_float((a & 0x007fffffu) | 0x3f800000u) - 0.99999994039535522f;
}

}  // namespace ptg

#endif
