/* Project-written stand-in for the subset of GSL's random-number API that the
 * openECLOUD reference binds (randomGen.pyx:9-16).  Test infrastructure only:
 * it exists so the reference Cython can be compiled as an oracle without GSL.
 * Generator: MT19937 (Matsumoto & Nishimura, ACM TOMACS 8(1), 1998). */
#ifndef OEC_GSL_SHIM_RNG_H
#define OEC_GSL_SHIM_RNG_H
#ifdef __cplusplus
extern "C" {
#endif
typedef struct gsl_rng_type gsl_rng_type;
typedef struct gsl_rng gsl_rng;
extern const gsl_rng_type *gsl_rng_mt19937;
gsl_rng *gsl_rng_alloc(const gsl_rng_type *T);
void gsl_rng_free(gsl_rng *r);
void gsl_rng_set(gsl_rng *r, unsigned long int seed);
unsigned long gsl_rng_get(const gsl_rng *r);
double gsl_rng_uniform(const gsl_rng *r);
unsigned long gsl_rng_uniform_int(const gsl_rng *r, unsigned long n);
#ifdef __cplusplus
}
#endif
#endif
