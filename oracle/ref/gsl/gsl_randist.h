/* ORACLE / TEST INFRASTRUCTURE ONLY.  Declarations of the GSL distribution
 * calls named by the reference's src/rng.cpp; implemented from the Philox
 * stream in oracle/ref/gsl_philox_shim.cpp.  None of them is reached by the
 * Brownian-dynamics step (only gsl_rng_uniform_pos is). */
#ifndef SC_SHIM_GSL_RANDIST_H
#define SC_SHIM_GSL_RANDIST_H
#include "gsl_rng.h"
#ifdef __cplusplus
extern "C" {
#endif
unsigned int gsl_ran_poisson(const gsl_rng *r, double mu);
double gsl_ran_gaussian_ziggurat(const gsl_rng *r, double sigma);
void gsl_ran_shuffle(const gsl_rng *r, void *base, size_t n, size_t size);
#ifdef __cplusplus
}
#endif
#endif
