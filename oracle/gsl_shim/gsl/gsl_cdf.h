/* Project-written stand-in for GSL quantile functions used by the reference
 * (specFun.pyx:24-26).  Test infrastructure. */
#ifndef OEC_GSL_SHIM_CDF_H
#define OEC_GSL_SHIM_CDF_H
#ifdef __cplusplus
extern "C" {
#endif
double gsl_cdf_ugaussian_Pinv(double p);
double gsl_cdf_ugaussian_Qinv(double q);
double gsl_cdf_tdist_Pinv(double p, double nu);
#ifdef __cplusplus
}
#endif
#endif
