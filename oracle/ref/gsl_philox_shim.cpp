// ORACLE / TEST INFRASTRUCTURE ONLY -- linked only into oracle/_ref, the
// build of the reference's own hot-path sources that pins the CPU oracle.
//
// Implements the GSL random-number interface that the reference's
// src/rng.cpp calls (RNG::RNG, RandomUniform, GetSeed, ... at
// src/rng.cpp:3-20) on top of the Philox4x32-10 stream of ../sc_philox.h.
// Each gsl_rng is one stream keyed by (global seed, seed passed to
// gsl_rng_set); the harness constructs filament i with seed i, so filament i
// draws from key (global seed, i) exactly like the CPU oracle and the GPU.
//
// Every live generator is kept in a registry so the harness can rewind all
// streams to draw 0 once the initial configuration has been loaded
// (construction and insertion consume draws that the dynamics must not see).
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <mutex>
#include <set>

#include "gsl/gsl_randist.h"
#include "gsl/gsl_rng.h"
#include "../sc_philox.h"

struct sc_shim_rng {
  uint32_t key0;
  uint32_t key1;
  uint64_t k;       // next draw index
  int noise_sites;  // > 0 once the harness declared this a filament's noise stream
  int noise_dim;
};

namespace {
std::mutex g_mtx;
std::set<sc_shim_rng *> *g_live = nullptr;
uint32_t g_seed = 0;
const gsl_rng_type g_type = {"philox4x32_10"};

uint32_t next_word(const gsl_rng *r) {
  sc_shim_rng *s = const_cast<sc_shim_rng *>(r);
  return sc_philox_other_word(s->key0, s->key1, s->k++);
}
}  // namespace

extern "C" {

const gsl_rng_type *gsl_rng_default = &g_type;

const gsl_rng_type *gsl_rng_env_setup(void) { return &g_type; }

gsl_rng *gsl_rng_alloc(const gsl_rng_type *) {
  sc_shim_rng *r = new sc_shim_rng;
  r->key0 = g_seed;
  r->key1 = 0;
  r->k = 0;
  r->noise_sites = 0;
  r->noise_dim = 0;
  std::lock_guard<std::mutex> lk(g_mtx);
  if (!g_live) g_live = new std::set<sc_shim_rng *>();
  g_live->insert(r);
  return r;
}

void gsl_rng_set(const gsl_rng *r, unsigned long int seed) {
  sc_shim_rng *s = const_cast<sc_shim_rng *>(r);
  s->key0 = g_seed;
  s->key1 = (uint32_t)seed;
  s->k = 0;
}

void gsl_rng_free(gsl_rng *r) {
  {
    std::lock_guard<std::mutex> lk(g_mtx);
    if (g_live) g_live->erase(r);
  }
  delete r;
}

unsigned long int gsl_rng_get(const gsl_rng *r) { return next_word(r); }

double gsl_rng_uniform_pos(const gsl_rng *r) {
  sc_shim_rng *s = const_cast<sc_shim_rng *>(r);
  if (s->noise_sites > 0) {
    // A filament's noise draws: site-major, dimension-minor per midstep
    // (src/filament.cpp:527-531), mapped onto the shared noise counters.
    uint64_t k = s->k++;
    uint64_t per = (uint64_t)s->noise_sites * (uint64_t)s->noise_dim;
    uint64_t m = k / per;
    uint32_t j = (uint32_t)((k / s->noise_dim) % s->noise_sites);
    int i = (int)(k % s->noise_dim);
    return sc_philox_noise(s->key0, s->key1, m, j, i);
  }
  return ((double)next_word(r) + 0.5) * 2.3283064365386963e-10;
}

unsigned long int gsl_rng_uniform_int(const gsl_rng *r, unsigned long int n) {
  if (n == 0) return 0;
  return (unsigned long int)floor(gsl_rng_uniform_pos(r) * (double)n) % n;
}

void *gsl_rng_state(const gsl_rng *r) { return const_cast<gsl_rng *>(r); }

size_t gsl_rng_size(const gsl_rng *) { return sizeof(sc_shim_rng); }

unsigned int gsl_ran_poisson(const gsl_rng *r, double mu) {
  // Inversion by sequential search; adequate for the small means it could see.
  double L = exp(-mu), p = 1.0;
  unsigned int k = 0;
  do {
    ++k;
    p *= gsl_rng_uniform_pos(r);
  } while (p > L && k < 100000u);
  return k - 1;
}

double gsl_ran_gaussian_ziggurat(const gsl_rng *r, double sigma) {
  // Box-Muller (not a ziggurat): only the distribution matters off the path.
  double u1 = gsl_rng_uniform_pos(r), u2 = gsl_rng_uniform_pos(r);
  return sigma * sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

void gsl_ran_shuffle(const gsl_rng *r, void *base, size_t n, size_t size) {
  unsigned char *b = (unsigned char *)base;
  unsigned char tmp[256];
  if (size > sizeof(tmp)) return;
  for (size_t i = n; i > 1; --i) {
    size_t j = gsl_rng_uniform_int(r, i);
    memcpy(tmp, b + (i - 1) * size, size);
    memcpy(b + (i - 1) * size, b + j * size, size);
    memcpy(b + j * size, tmp, size);
  }
}

// Harness controls (not part of the GSL interface).
void scshim_set_global_seed(uint32_t seed) { g_seed = seed; }

void scshim_rewind_all(void) {
  std::lock_guard<std::mutex> lk(g_mtx);
  if (!g_live) return;
  for (sc_shim_rng *r : *g_live) r->k = 0;
}

// Declares the stream keyed (global seed, key1) a filament noise stream of a
// filament with n_sites sites in n_dim dimensions.
void scshim_set_noise_layout(uint32_t key1, int n_sites, int n_dim) {
  std::lock_guard<std::mutex> lk(g_mtx);
  if (!g_live) return;
  for (sc_shim_rng *r : *g_live)
    if (r->key0 == g_seed && r->key1 == key1) {
      r->noise_sites = n_sites;
      r->noise_dim = n_dim;
    }
}

}  // extern "C"
