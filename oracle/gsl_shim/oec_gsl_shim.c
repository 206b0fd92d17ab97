/*
 * oec_gsl_shim.c -- project-written replacement for the small part of GSL 1.15
 * that the openECLOUD reference binds.  TEST INFRASTRUCTURE ONLY: it is linked
 * into (1) the reference Cython modules compiled as an oracle under
 * oracle/_ref and (2) the C restatement of the reference (oracle/oec_oracle.c),
 * so both consume an identical random stream and identical special functions.
 * Nothing in the product (openecloud_b200/) links against this file.
 *
 * GSL is not vendored with the reference and is not installed here, so the
 * exact GSL numbers are NOT reproduced ("parity unpinned" for GSL's own
 * streams).  Every function below is written from a published method:
 *
 *   MT19937 ........ Matsumoto & Nishimura, ACM TOMACS 8(1):3-30, 1998
 *                    (2002 "init_genrand" seeding recurrence)
 *   Gaussian ....... Marsaglia & Bray polar method (SIAM Review 6, 1964)
 *   ln Gamma ....... C99 lgamma()
 *   P(a,x) ......... power series / Legendre continued fraction
 *                    (Abramowitz & Stegun 6.5.29, 6.5.31), modified Lentz
 *   I_x(a,b) ....... continued fraction A&S 26.5.8, modified Lentz
 *   Phi^-1(p) ...... P. J. Acklam's rational start + Halley steps on erfc
 *   t quantile ..... bisection on the t CDF expressed through I_x(nu/2,1/2)
 *   binomial pdf ... exp of log-gamma combination
 *
 * Reference call sites: randomGen.pyx:9-35, specFun.pyx:17-50.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "gsl/gsl_cdf.h"
#include "gsl/gsl_randist.h"
#include "gsl/gsl_rng.h"
#include "gsl/gsl_sf_gamma.h"

/* ------------------------------------------------------------------ RNG */

enum { MT_N = 624, MT_M = 397 };

struct gsl_rng_type {
    const char *name;
};

struct gsl_rng {
    uint32_t state[MT_N];
    int pos;
};

static const gsl_rng_type mt_type = {"mt19937"};
const gsl_rng_type *gsl_rng_mt19937 = &mt_type;

gsl_rng *gsl_rng_alloc(const gsl_rng_type *T) {
    (void)T;
    gsl_rng *r = (gsl_rng *)calloc(1, sizeof(gsl_rng));
    if (r) gsl_rng_set(r, 0);
    return r;
}

void gsl_rng_free(gsl_rng *r) { free(r); }

void gsl_rng_set(gsl_rng *r, unsigned long int seed) {
    uint32_t s = (uint32_t)(seed & 0xffffffffUL);
    if (s == 0) s = 4357u; /* zero seed is mapped to a fixed non-zero value */
    r->state[0] = s;
    for (int i = 1; i < MT_N; ++i) {
        uint32_t prev = r->state[i - 1];
        r->state[i] = 1812433253u * (prev ^ (prev >> 30)) + (uint32_t)i;
    }
    r->pos = MT_N;
}

static void mt_refill(gsl_rng *r) {
    /* One "twist" of the whole 624-word state (TOMACS 1998, eq. 2.1). */
    uint32_t *s = r->state;
    for (int k = 0; k < MT_N; ++k) {
        uint32_t y = (s[k] & 0x80000000u) | (s[(k + 1) % MT_N] & 0x7fffffffu);
        uint32_t v = s[(k + MT_M) % MT_N] ^ (y >> 1);
        if (y & 1u) v ^= 0x9908b0dfu;
        s[k] = v;
    }
    r->pos = 0;
}

static uint32_t mt_next(gsl_rng *r) {
    if (r->pos >= MT_N) mt_refill(r);
    uint32_t y = r->state[r->pos++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

unsigned long gsl_rng_get(const gsl_rng *r) { return mt_next((gsl_rng *)r); }

double gsl_rng_uniform(const gsl_rng *r) {
    return (double)mt_next((gsl_rng *)r) * (1.0 / 4294967296.0);
}

unsigned long gsl_rng_uniform_int(const gsl_rng *r, unsigned long n) {
    /* Uniform integer in [0, n) by scaling with rejection of the tail. */
    if (n == 0) return 0;
    const unsigned long range = 0xffffffffUL;
    unsigned long bucket = range / n;
    unsigned long k;
    do {
        k = (unsigned long)mt_next((gsl_rng *)r) / bucket;
    } while (k >= n);
    return k;
}

double gsl_ran_gaussian_ziggurat(const gsl_rng *r, double sigma) {
    /* Polar method; one normal deviate per call (no caching of the pair). */
    double u, v, s;
    do {
        u = 2.0 * gsl_rng_uniform(r) - 1.0;
        v = 2.0 * gsl_rng_uniform(r) - 1.0;
        s = u * u + v * v;
    } while (s >= 1.0 || s == 0.0);
    return sigma * u * sqrt(-2.0 * log(s) / s);
}

/* --------------------------------------------------------- special funcs */

double gsl_sf_lngamma(double a) { return lgamma(a); }

double gsl_sf_gamma(double a) { return tgamma(a); }

double gsl_sf_beta(double a, double b) {
    return exp(lgamma(a) + lgamma(b) - lgamma(a + b));
}

static const double SF_TINY = 1e-300;
static const double SF_EPS = 1e-16;

/* Regularised lower incomplete gamma P(a, x), a > 0. */
double gsl_sf_gamma_inc_P(double a, double x) {
    if (!(x > 0.0)) return 0.0;
    if (isinf(x)) return 1.0;
    double lpref = -x + a * log(x) - lgamma(a);
    if (x < a + 1.0) {
        /* sum_{n>=0} x^n / (a (a+1) ... (a+n)) */
        double term = 1.0 / a, sum = term, an = a;
        for (int n = 0; n < 100000; ++n) {
            an += 1.0;
            term *= x / an;
            sum += term;
            if (fabs(term) <= fabs(sum) * SF_EPS) break;
        }
        double p = sum * exp(lpref);
        return p > 1.0 ? 1.0 : p;
    }
    /* Q(a,x) via the Legendre continued fraction, modified Lentz. */
    double b = x + 1.0 - a;
    double c = 1.0 / SF_TINY;
    double d = 1.0 / b;
    double f = d;
    for (int i = 1; i < 100000; ++i) {
        double an = -i * (i - a);
        b += 2.0;
        d = an * d + b;
        if (fabs(d) < SF_TINY) d = SF_TINY;
        c = b + an / c;
        if (fabs(c) < SF_TINY) c = SF_TINY;
        d = 1.0 / d;
        double delta = d * c;
        f *= delta;
        if (fabs(delta - 1.0) <= SF_EPS) break;
    }
    double q = exp(lpref) * f;
    double p = 1.0 - q;
    return p < 0.0 ? 0.0 : p;
}

/* Continued fraction for I_x(a,b) (A&S 26.5.8), modified Lentz. */
static double beta_cf(double a, double b, double x) {
    double qab = a + b, qap = a + 1.0, qam = a - 1.0;
    double c = 1.0, d = 1.0 - qab * x / qap;
    if (fabs(d) < SF_TINY) d = SF_TINY;
    d = 1.0 / d;
    double h = d;
    for (int m = 1; m < 100000; ++m) {
        int m2 = 2 * m;
        double aa = m * (b - m) * x / ((qam + m2) * (a + m2));
        d = 1.0 + aa * d;
        if (fabs(d) < SF_TINY) d = SF_TINY;
        c = 1.0 + aa / c;
        if (fabs(c) < SF_TINY) c = SF_TINY;
        d = 1.0 / d;
        h *= d * c;
        aa = -(a + m) * (qab + m) * x / ((a + m2) * (qap + m2));
        d = 1.0 + aa * d;
        if (fabs(d) < SF_TINY) d = SF_TINY;
        c = 1.0 + aa / c;
        if (fabs(c) < SF_TINY) c = SF_TINY;
        d = 1.0 / d;
        double del = d * c;
        h *= del;
        if (fabs(del - 1.0) <= SF_EPS) break;
    }
    return h;
}

/* Regularised incomplete beta I_x(a, b), a, b > 0. */
double gsl_sf_beta_inc(double a, double b, double x) {
    if (x <= 0.0) return 0.0;
    if (x >= 1.0) return 1.0;
    double lbt = lgamma(a + b) - lgamma(a) - lgamma(b) + a * log(x) + b * log1p(-x);
    double bt = exp(lbt);
    if (x < (a + 1.0) / (a + b + 2.0)) return bt * beta_cf(a, b, x) / a;
    return 1.0 - bt * beta_cf(b, a, 1.0 - x) / b;
}

double gsl_ran_binomial_pdf(unsigned int k, double p, unsigned int n) {
    if (k > n) return 0.0;
    if (p == 0.0) return k == 0 ? 1.0 : 0.0;
    if (p == 1.0) return k == n ? 1.0 : 0.0;
    double lc = lgamma((double)n + 1.0) - lgamma((double)k + 1.0) - lgamma((double)(n - k) + 1.0);
    return exp(lc + k * log(p) + (double)(n - k) * log1p(-p));
}

/* Standard normal quantile. */
double gsl_cdf_ugaussian_Pinv(double p) {
    if (p <= 0.0) return -INFINITY;
    if (p >= 1.0) return INFINITY;
    /* Acklam's rational approximation as a starting point. */
    static const double a[6] = {-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
                                1.383577518672690e+02, -3.066479806614716e+01, 2.506628277459239e+00};
    static const double b[5] = {-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
                                6.680131188771972e+01, -1.328068155288572e+01};
    static const double c[6] = {-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
                                -2.549732539343734e+00, 4.374664141464968e+00, 2.938163982698783e+00};
    static const double d[4] = {7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00,
                                3.754408661907416e+00};
    const double plow = 0.02425;
    double x;
    if (p < plow) {
        double q = sqrt(-2.0 * log(p));
        x = (((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
            ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1.0);
    } else if (p <= 1.0 - plow) {
        double q = p - 0.5, r = q * q;
        x = (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * q /
            (((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1.0);
    } else {
        double q = sqrt(-2.0 * log1p(-p));
        x = -(((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
            ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1.0);
    }
    /* Halley refinement on Phi(x) - p with Phi(x) = erfc(-x/sqrt2)/2. */
    for (int it = 0; it < 3; ++it) {
        double e = 0.5 * erfc(-x / M_SQRT2) - p;
        double u = e * sqrt(2.0 * M_PI) * exp(0.5 * x * x);
        x = x - u / (1.0 + 0.5 * x * u);
    }
    return x;
}

double gsl_cdf_ugaussian_Qinv(double q) { return -gsl_cdf_ugaussian_Pinv(q); }

/* Student-t CDF for t >= 0 through the incomplete beta function. */
static double t_cdf_upper_half(double t, double nu) {
    double x = nu / (nu + t * t);
    return 1.0 - 0.5 * gsl_sf_beta_inc(0.5 * nu, 0.5, x);
}

double gsl_cdf_tdist_Pinv(double p, double nu) {
    if (p <= 0.0) return -INFINITY;
    if (p >= 1.0) return INFINITY;
    if (p == 0.5) return 0.0;
    if (p < 0.5) return -gsl_cdf_tdist_Pinv(1.0 - p, nu);
    double lo = 0.0, hi = 1.0;
    for (int i = 0; i < 2000 && t_cdf_upper_half(hi, nu) < p; ++i) hi *= 2.0;
    for (int i = 0; i < 200; ++i) {
        double mid = 0.5 * (lo + hi);
        if (t_cdf_upper_half(mid, nu) < p)
            lo = mid;
        else
            hi = mid;
        if (hi - lo <= 1e-15 * hi) break;
    }
    return 0.5 * (lo + hi);
}
