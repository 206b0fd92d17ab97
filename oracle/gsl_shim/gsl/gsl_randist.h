/* Project-written stand-in for GSL distribution functions used by the
 * reference (randomGen.pyx:18-19, specFun.pyx:28-29).  Test infrastructure. */
#ifndef OEC_GSL_SHIM_RANDIST_H
#define OEC_GSL_SHIM_RANDIST_H
#include "gsl_rng.h"
#ifdef __cplusplus
extern "C" {
#endif
double gsl_ran_gaussian_ziggurat(const gsl_rng *r, double sigma);
double gsl_ran_binomial_pdf(unsigned int k, double p, unsigned int n);
#ifdef __cplusplus
}
#endif
#endif
