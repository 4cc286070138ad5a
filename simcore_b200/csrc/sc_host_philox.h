// Philox4x32-10 (Salmon et al., SC'11) for host and device code.
//
// Thermal-noise stream of filament f: key (system seed, f); the k-th uniform
// since dynamics started is word (k & 3) of philox(counter (k>>2, k>>34, 0,
// 0)), mapped to (word + 0.5) * 2^-32 in (0, 1), the range of
// gsl_rng_uniform_pos that the reference draws from (src/rng.cpp:20).
#ifndef SC_HOST_PHILOX_H
#define SC_HOST_PHILOX_H

#include <stdint.h>

#if defined(__CUDACC__)
#define SC_HD __host__ __device__ __forceinline__
#else
#define SC_HD static inline
#endif

SC_HD void sc_host_philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2,
                                 uint32_t c3, uint32_t k0, uint32_t k1,
                                 uint32_t out[4]) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
#if defined(__CUDA_ARCH__)
    uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
#else
    uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

SC_HD uint32_t sc_host_philox_word(uint32_t k0, uint32_t k1, uint64_t k) {
  uint32_t o[4];
  sc_host_philox4x32_10((uint32_t)(k >> 2), (uint32_t)(k >> 34), 0u, 0u, k0, k1, o);
  return o[k & 3u];
}

SC_HD double sc_host_philox_uniform(uint32_t k0, uint32_t k1, uint64_t k) {
  return ((double)sc_host_philox_word(k0, k1, k) + 0.5) * 2.3283064365386963e-10;
}

#endif
