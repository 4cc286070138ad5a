/* ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into the product library.
 *
 * Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
 * "Parallel random numbers: as easy as 1, 2, 3", SC'11), written from the
 * published round function.  It is the shared noise source of the CPU
 * oracle, the GSL shim used to build the reference's own code, and (in an
 * independent implementation) the CUDA kernels.
 *
 * Stream convention (identical in every code that draws thermal noise):
 *   key     = (k0, k1) = (system seed, filament index within the system)
 *   draw k  = k-th uniform of that filament since dynamics started
 *   word    = philox4x32_10(counter = (k >> 2 low32, k >> 34, 0, 0), key)[k & 3]
 *   uniform = (word + 0.5) * 2^-32, strictly inside (0, 1) like
 *             gsl_rng_uniform_pos (reference src/rng.cpp:20).
 * The reference draws, per midstep, one uniform per site and per dimension in
 * site-major order (reference src/filament.cpp:527-531), so site j, dim i of
 * midstep m uses k = (m * n_sites + j) * n_dim + i.
 */
#ifndef SC_ORACLE_PHILOX_H
#define SC_ORACLE_PHILOX_H

#include <stdint.h>

#define SC_PHILOX_M0 0xD2511F53u
#define SC_PHILOX_M1 0xCD9E8D57u
#define SC_PHILOX_W0 0x9E3779B9u
#define SC_PHILOX_W1 0xBB67AE85u

static inline void sc_philox4x32_10(const uint32_t ctr_in[4],
                                    const uint32_t key_in[2],
                                    uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  int r;
  for (r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)SC_PHILOX_M0 * (uint64_t)c0;
    uint64_t p1 = (uint64_t)SC_PHILOX_M1 * (uint64_t)c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += SC_PHILOX_W0;
    k1 += SC_PHILOX_W1;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

/* k-th 32-bit word of the stream keyed by (k0, k1). */
static inline uint32_t sc_philox_word(uint32_t k0, uint32_t k1, uint64_t k) {
  uint32_t ctr[4], key[2], out[4];
  ctr[0] = (uint32_t)(k >> 2);
  ctr[1] = (uint32_t)(k >> 34);
  ctr[2] = 0u;
  ctr[3] = 0u;
  key[0] = k0;
  key[1] = k1;
  sc_philox4x32_10(ctr, key, out);
  return out[k & 3u];
}

/* Uniform strictly inside (0, 1); exact in double. */
static inline double sc_philox_uniform(uint32_t k0, uint32_t k1, uint64_t k) {
  return ((double)sc_philox_word(k0, k1, k) + 0.5) * 2.3283064365386963e-10;
}

#endif
