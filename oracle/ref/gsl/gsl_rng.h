/* ORACLE / TEST INFRASTRUCTURE ONLY.
 * Declaration-compatible stand-in for the handful of GSL random-number calls
 * that the reference's src/rng.cpp makes.  GSL is not installed here, and the
 * oracle deliberately replaces the GSL Mersenne-Twister stream with the shared
 * Philox4x32-10 stream (see ../../sc_philox.h).  This header declares the
 * interface only; oracle/ref/gsl_philox_shim.cpp implements it from Philox,
 * not from GSL source. */
#ifndef SC_SHIM_GSL_RNG_H
#define SC_SHIM_GSL_RNG_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct sc_shim_rng_type { const char *name; } gsl_rng_type;
typedef struct sc_shim_rng gsl_rng;
extern const gsl_rng_type *gsl_rng_default;
const gsl_rng_type *gsl_rng_env_setup(void);
gsl_rng *gsl_rng_alloc(const gsl_rng_type *T);
void gsl_rng_set(const gsl_rng *r, unsigned long int seed);
void gsl_rng_free(gsl_rng *r);
unsigned long int gsl_rng_get(const gsl_rng *r);
double gsl_rng_uniform_pos(const gsl_rng *r);
unsigned long int gsl_rng_uniform_int(const gsl_rng *r, unsigned long int n);
void *gsl_rng_state(const gsl_rng *r);
size_t gsl_rng_size(const gsl_rng *r);
#ifdef __cplusplus
}
#endif
#endif
