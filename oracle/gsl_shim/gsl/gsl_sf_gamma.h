/* Project-written stand-in for GSL gamma/beta special functions used by the
 * reference (specFun.pyx:17-22).  Test infrastructure. */
#ifndef OEC_GSL_SHIM_SF_GAMMA_H
#define OEC_GSL_SHIM_SF_GAMMA_H
#ifdef __cplusplus
extern "C" {
#endif
double gsl_sf_beta(double a, double b);
double gsl_sf_beta_inc(double a, double b, double x);
double gsl_sf_gamma_inc_P(double a, double x);
double gsl_sf_gamma(double a);
double gsl_sf_lngamma(double a);
#ifdef __cplusplus
}
#endif
#endif
