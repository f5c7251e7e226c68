// Scrambled low-discrepancy sampling shared by the pool kernels and the host.
//
// Points are a 2D Sobol (0,2)-sequence with hash-based Owen scrambling and
// an Owen-scrambled index shuffle, after B. Burley, "Practical Hash-based
// Owen Scrambling", Journal of Computer Graphics Techniques 9(4), 2020.
// Independent 2D streams (sun shape, slope error) use different seeds, the
// "padded 2D" construction of that paper.  All of it is integer arithmetic
// and gives identical bits on host and device.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define QS_HD __host__ __device__ __forceinline__
#else
#define QS_HD inline
#endif

namespace qm {

QS_HD uint32_t reverse_bits32(uint32_t x) {
#if defined(__CUDA_ARCH__)
  return __brev(x);
#else
  x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
  x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
  x = ((x >> 4) & 0x0f0f0f0fu) | ((x & 0x0f0f0f0fu) << 4);
  x = ((x >> 8) & 0x00ff00ffu) | ((x & 0x00ff00ffu) << 8);
  return (x >> 16) | (x << 16);
#endif
}

// Integer finaliser (the "lowbias32" mix of C. Wellons' hash-prospector).
QS_HD uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

QS_HD uint32_t hash_combine(uint32_t seed, uint32_t v) { return seed ^ (v + (seed << 6) + (seed >> 2)); }

// Burley 2020, listing 3: the improved Laine-Karras permutation, applied to a
// bit-reversed value so that it is a nested uniform (Owen) scramble.
QS_HD uint32_t lk_permutation(uint32_t x, uint32_t seed) {
  x += seed;
  x ^= x * 0x6c50b47cu;
  x ^= x * 0xb82f1e52u;
  x ^= x * 0xc7afe638u;
  x ^= x * 0x8d22f6e6u;
  return x;
}

QS_HD uint32_t owen_scramble(uint32_t x, uint32_t seed) {
  return reverse_bits32(lk_permutation(reverse_bits32(x), seed));
}

// Second Sobol dimension: primitive polynomial x + 1, direction numbers
// v_1 = 2^31, v_k = v_{k-1} ^ (v_{k-1} >> 1).
QS_HD uint32_t sobol_dim1(uint32_t index) {
  uint32_t r = 0u, v = 0x80000000u;
  for (; index; index >>= 1, v ^= v >> 1)
    if (index & 1u) r ^= v;
  return r;
}

// Owen-scrambled 2D Sobol point `index` of stream `seed`, as two 32-bit
// fixed-point fractions.
QS_HD void sobol2_owen(uint32_t index, uint32_t seed, uint32_t& x, uint32_t& y) {
  const uint32_t shuffled = owen_scramble(index, mix32(seed));
  x = owen_scramble(reverse_bits32(shuffled), mix32(hash_combine(seed, 0u)));
  y = owen_scramble(sobol_dim1(shuffled), mix32(hash_combine(seed, 1u)));
}

// 32-bit fraction -> double in (0, 1): the cell midpoint, never 0 or 1.
QS_HD double unit_open(uint32_t x) { return ((double)x + 0.5) * (1.0 / 4294967296.0); }
// 32-bit fraction -> float in [0, 1) (24 significant bits kept).
QS_HD float unit_float(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

// Per-facet pool offset in [0, pool): an unbiased-enough multiply-shift of a
// hashed (seed, heliostat, facet) triple.
QS_HD int facet_offset(uint32_t seed, uint32_t heliostat, uint32_t facet, uint32_t pool) {
  uint32_t h = mix32(hash_combine(hash_combine(mix32(seed ^ 0x9e3779b9u), heliostat), facet));
  return (int)(((uint64_t)h * (uint64_t)pool) >> 32);
}

}  // namespace qm
