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
 *   The reference draws, per midstep, one uniform per site and per dimension
 *   in site-major order (reference src/filament.cpp:527-531).  The draw for
 *   site j, dimension i (< 3) of the filament's m-th noisy midstep is
 *     word    = philox4x32_10(counter = (j, m low32, m >> 32, 0), key)[i]
 *     uniform = (word + 0.5) * 2^-32, strictly inside (0, 1) like
 *               gsl_rng_uniform_pos (reference src/rng.cpp:20).
 *   A filament's k-th draw since dynamics started maps to
 *   m = k / (n_sites n_dim), j = (k / n_dim) % n_sites, i = k % n_dim.
 * Any other draw of a stream (the reference's construction and insertion
 * calls, which happen before the stream is rewound) uses
 *   word = philox4x32_10(counter = (k >> 2, k >> 34, 0, 0xFFFFFFFF), key)[k & 3].
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

/* Thermal-noise uniform of site j, dimension i, midstep m of stream (k0, k1). */
static inline double sc_philox_noise(uint32_t k0, uint32_t k1, uint64_t m,
                                     uint32_t j, int i) {
  uint32_t ctr[4], key[2], out[4];
  ctr[0] = j;
  ctr[1] = (uint32_t)m;
  ctr[2] = (uint32_t)(m >> 32);
  ctr[3] = 0u;
  key[0] = k0;
  key[1] = k1;
  sc_philox4x32_10(ctr, key, out);
  return ((double)out[i] + 0.5) * 2.3283064365386963e-10;
}

/* Any other (non-noise) word k of stream (k0, k1). */
static inline uint32_t sc_philox_other_word(uint32_t k0, uint32_t k1, uint64_t k) {
  uint32_t ctr[4], key[2], out[4];
  ctr[0] = (uint32_t)(k >> 2);
  ctr[1] = (uint32_t)(k >> 34);
  ctr[2] = 0u;
  ctr[3] = 0xFFFFFFFFu;
  key[0] = k0;
  key[1] = k1;
  sc_philox4x32_10(ctr, key, out);
  return out[k & 3u];
}

#endif
