/*
 * oec_oracle_emit.c -- CPU restatement of the Furman-Pivi secondary
 * emission (particleEmitter.pyx:154-308), the uniform loader
 * (particleEmitter.pyx:41-72) and the reference's own special-function
 * inverses (specFun.pyx:53-341).  TEST INFRASTRUCTURE ONLY (see oec_oracle.c).
 *
 * Two sources of random numbers:
 *  - mode 0: the global MT19937 stream of the GSL stand-in, consumed in the
 *    reference's order (rand / randn) -- with the same seed this replays the
 *    compiled reference exactly;
 *  - mode 1: injected uniforms, 32 per absorbed particle: draw 0 picks the
 *    secondary count, the following draws are consumed in order and a normal
 *    deviate is Box-Muller of two draws -- the layout of the GPU kernel.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "gsl/gsl_cdf.h"
#include "gsl/gsl_randist.h"
#include "gsl/gsl_rng.h"
#include "gsl/gsl_sf_gamma.h"

double orc_rand(void);
double orc_randn(void);

static const double PI = 3.141592653589793;
static const double MACH_EPS = 2.220446049250313e-16;

/* ------------------------------------------------- specFun.pyx:268-341 */
double orc_gammaincinv(double a, double p) {
    const double acc = 1.e-9, a1 = a - 1.;
    double eps = sqrt(acc), x, t, lna1 = 0., afac = 0.;
    if (!(a > 0)) return NAN;
    if (p >= 1.) return fmax(100., a + 100. * sqrt(a));
    if (p <= 0.) return 0.0;
    double gln = gsl_sf_lngamma(a);
    if (a > 1.) {
        lna1 = log(a1);
        afac = exp(a1 * (lna1 - 1.) - gln);
        double pp = p < 0.5 ? p : (1 - p);
        t = sqrt(-2. * log(pp));
        x = (2.30753 + t * 0.27061) / (1 + t * (0.99229 + t * 0.04481)) - t;
        if (p < 0.5) x = -x;
        x = fmax(1.e-3, a * pow(1. - 1. / (9. * a) - x / (3. * sqrt(a)), 3));
    } else {
        t = 1. - a * (0.253 + a * 0.12);
        x = (p < t) ? pow(p / t, 1. / a) : 1. - log(1. - (p - t) / (1. - t));
    }
    int j;
    for (j = 0; j < 20; ++j) {
        if (x <= 0.0) return 0.0;
        double err = gsl_sf_gamma_inc_P(a, x) - p;
        t = (a > 1.) ? afac * exp(-(x - a1) + a1 * (log(x) - lna1)) : exp(-x + a1 * log(x) - gln);
        double u = err / t;
        t = u / (1. - 0.5 * fmin(1., u * ((a - 1.) / x - 1.)));
        x -= t;
        if (x <= 0.) x = 0.5 * (x + t);
        if (fabs(t) < eps * x) { j = 0; break; }
    }
    if (j == 20) j = 19;
    if (j == 19 && x < a) {
        eps = eps * eps;
        double err = gsl_sf_gamma_inc_P(a, x) - p;
        double xr = x, xl;
        for (int g = 0; err <= 0 && g < 2000; ++g) { xr *= 2.; err = gsl_sf_gamma_inc_P(a, xr) - p; }
        xl = 0.;
        x = 0.5 * (xr + xl);
        for (int k = 0; k < 100; ++k) {
            err = gsl_sf_gamma_inc_P(a, x) - p;
            if (err <= 0.) xl = x; else xr = x;
            x = 0.5 * (xr + xl);
            if (0.5 * (xr - x) < eps * x) break;
            if (x < eps * a) { x = 0.; break; }
        }
    }
    return x;
}

/* --------------------------------------------------- specFun.pyx:53-253 */
double orc_betaincinv(double a, double b, double p) {
    const double acc = 1.e-12;
    double q = 1 - p, sqrt2 = sqrt(2), EPS = sqrt(acc), x = 0.;
    unsigned nh = (unsigned)((-log(acc) / log(10)) + 1.);
    int sw = 0;
    if (q <= MACH_EPS) return 1.;
    if (p <= MACH_EPS) return 0.;
    if (a == 1 && b == 1) return p;
    if (a == 0.5 && b == 0.5) return sin(p * 0.5 * PI);
    if (a == 0.5 && b >= 0.5) { x = gsl_cdf_tdist_Pinv(0.5 * q, 2. * b); return 1 - 2. * b / (2. * b + x * x); }
    if (a >= 0.5 && b == 0.5) { x = gsl_cdf_tdist_Pinv(0.5 * p, 2. * a); return 2. * a / (2. * a + x * x); }
    if (a > b) { double t = a; a = b; b = t; t = p; p = q; q = t; sw = 1; }
    if (a + b >= 5) {
        if ((b - a) <= sqrt(a)) {
            double e0 = -1. / sqrt(a) * gsl_cdf_ugaussian_Qinv(p), be = b - a;
            double E2 = e0 * e0, E3 = E2 * e0, E4 = E3 * e0, E5 = E4 * e0, E6 = E5 * e0;
            double p1 = (-0.5 * be * sqrt2 + 0.125 * (1. - 2. * be) * e0 - 1. / 48. * be * sqrt2 * E2 -
                         1. / 192. * E3 - 1. / 3840. * be * sqrt2 * E4);
            double p2 = (1. / 12. * be * sqrt2 * (3. * be - 2.) + 1. / 128. * (20. * be * be - 12 * be + 1.) * e0 +
                         1. / 960. * be * sqrt2 * (20. * be - 1.) * E2 + 1. / 4608. * (16. * be * be + 30. * be - 15.) * E3 +
                         1. / 53760. * be * sqrt2 * (21. * be + 32.) * E4 + 1. / 368640. * (-32. * be * be + 63.) * E5 +
                         1. / 25804480 * be * sqrt2 * (120. * be + 17.) * E6);
            double p3 = (1. / 480. * be * sqrt2 * (-75. * be * be + 80. * be - 16.) +
                         1. / 9216. * (-1080. * be * be * be + 868. * be * be - 90. * be * be - 45.) * e0 +
                         1. / 53760 * be * sqrt2 * (-1190. * be * be + 84. * be + 373.) * E2 +
                         1. / 368640. * (-2240. * be * be * be - 2508. * be * be + 2100. * be - 165.) * E3);
            double eta = e0 + (p1 / a + p2 / (a * a) + p3 / (a * a * a));
            double r = sqrt(0.25 - 0.25 * exp(-0.5 * eta * eta));
            x = eta > 0 ? 0.5 + r : 0.5 - r;
        } else if (0.2 <= a / (a + b) && a / (a + b) <= 0.8) {
            if (pow(p, 1. / a) < 0.0025) x = pow(a * p * gsl_sf_beta(a, b), 1. / a);
            else if (pow(q, 1. / b) < 0.0025) x = 1 - pow(b * q * gsl_sf_beta(a, b), 1. / b);
            else {
                double r = a + b, s2 = a / r, c2 = b / r, s = sqrt(s2), c = sqrt(c2);
                double e0 = -1. / sqrt(r) * gsl_cdf_ugaussian_Qinv(p), E2 = e0 * e0, E3 = E2 * e0, E4 = E3 * e0;
                double S4 = s2 * s2, S6 = S4 * s2, S8 = S6 * s2, S10 = S8 * s2, S12 = S10 * s2, S14 = S12 * s2;
                double C4 = c2 * c2, C6 = C4 * c2;
                double p1 = ((2. * s2 - 1) / (2 * s * c) - (5. * S4 - 5. * s2 - 1) / (36. * s2 * c2) * e0 +
                             (46. * S6 - 69. * S4 + 21. * s2 + 1) / (1620. * s2 * s * c2 * c) * E2 -
                             (-2. * s2 - 62. * S6 + 31. * S8 + 33. * S4 + 7.) / (6480. * S4 * pow(c, 4)) * E3 +
                             (88. * S6 - 52. * s2 - 115. * S8 + 46. * S10 - 17. * S4 + 25.) / (90720. * S4 * s * C4 * c) * E4);
                double p2 = (-(52. * S6 - 78. * S4 + 12. * s2 + 7.) / (405. * s2 * s * c2 * c) +
                             (2. * s2 - 370. * S6 + 185. * S8 + 183. * S4 - 7.) / (2592. * S4 * pow(c, 4)) * e0 -
                             (776. * s2 + 10240. * S6 - 13525. * S8 - 533. + 5410. * S10 - 1835. * S4) /
                                 (204120. * S4 * s * C4 * c) * E2 +
                             (3747. * s2 + 15071. * S12 - 15821. * S6 + 45588. * S8 - 45213. * S10 - 3372. * S4 - 1579.) /
                                 (2099520. * S6 * C6) * E3);
                double p3 = ((3704. * S10 - 9620. * S8 + 6686. * S6 - 769. * S4 - 1259. * s2 + 449.) /
                                 (102060. * S4 * s * C4 * c) -
                             (750479. * S12 - 151557. * s2 - 727469. * S6 + 2239932. * S8 - 2251437. * S10 + 140052. * S4 +
                              63149.) / (20995200. * S6 * C6) * e0 +
                             (729754. * S14 - 78755. * s2 - 2554139. * S12 + 146879. * S6 - 1602610. * S8 + 3195183. * S10 +
                              105222. * S4 + 29233.) / (36741600. * S6 * s * C6 * c) * E2);
                double eta = e0 + (p1 / r + p2 / (r * r) + p3 / (r * r * r));
                if (eta * eta < 0.49) {
                    x = (s2 + s * c * eta + (1. - 2. * s2) / 3. * eta * eta + (13. * S4 - 13. * s2 + 1.) / (36. * s * c) * eta * eta * eta +
                         (46. * S6 - 69. * S4 + 21. * s2 + 1.) / (270. * s2 * c2) * eta * eta * eta * eta);
                } else {
                    double al = eta < 0 ? c2 / s2 : s2 / c2;
                    double u = exp(1. / (eta < 0 ? s2 : c2) * (-0.5 * eta * eta + s2 * log(s2) + c2 * log(c2)));
                    x = (u + al * u * u + 3. * al * (3. * al + 1.) / 6. * u * u * u +
                         4. * al * (4. * al + 1.) * (4. * al + 2.) / 24. * u * u * u * u +
                         5 * al * (5. * al + 1.) * (5. * al + 2.) * (5. * al + 3.) / 120. * u * u * u * u * u);
                    if (eta >= 0) x = 1 - x;
                }
            }
        } else {
            double e0 = 1. / b * orc_gammaincinv(a, p), mu = a / b, w = sqrt(1. + mu);
            double w2 = w * w, w3 = w * w2, w4 = w3 * w, w5 = w4 * w, w6 = w5 * w, w7 = w6 * w, w8 = w7 * w, w9 = w8 * w,
                   w10 = w9 * w, q1 = w + 1, q2 = q1 * q1, q3 = q2 * q1, q4 = q3 * q1;
            double d1 = e0 - mu, d2 = d1 * d1, d3 = d2 * d1, d4 = d3 * d1;
            double p1 = ((w + 2.) * (w - 1.) / (3. * w) + (w3 + 9. * w2 + 21. * w + 5.) / (36. * w2 * q1) * d1 -
                         (w4 - 13. * w3 + 69. * w2 + 167. * w + 46.) / (1620. * q2 * w3) * d2 -
                         (7. * w5 + 21. * w4 + 70. * w3 + 26. * w2 - 93. * w - 31.) / (6480. * q3 * w4) * d3 -
                         (75. * w6 + 202. * w5 + 188. * w4 - 888. * w3 - 1345. * w2 + 118. * w + 138.) / (272160. * q4 * w5) * d4);
            double p2 = ((28. * w4 + 131. * w3 + 402. * w2 + 581. * w + 208.) * (w - 1.) / (1620. * q1 * w3) -
                         (35. * w6 - 154. * w5 - 623. * w4 - 1636. * w3 - 3983. * w2 - 3514. * w - 925.) / (12960. * q2 * w4) * d1 -
                         (2132. * w7 + 7915. * w6 + 16821. * w5 + 35066. * w4 + 87490. * w3 + 141183. * w2 + 95993. * w + 21640.) /
                             (816480. * w5 * q3) * d2 -
                         (11053. * w8 + 53308. * w7 + 117010. * w6 + 163924. * w5 + 116188. * w4 - 258428. * w3 - 677042. * w2 -
                          481940. * w - 105497.) / (14696640. * q4 * w6) * d3);
            double p3 = (-((3592. * w7 + 8375. * w6 - 1323. * w5 - 29198. * w4 - 89578. * w3 - 154413. * w2 - 116063. * w - 29632.) *
                           (w - 1.)) / (816480. * w5 * q2) -
                         (442043. * w9 + 2054169. * w8 + 3803094. * w7 + 3470754. * w6 + 2141568. * w5 - 2393568. * w4 -
                          19904934. * w3 - 34714674. * w2 - 23128299. * w - 5253353.) / (146966400. * w6 * q3) * d1 -
                         (116932. * w10 + 819281. * w9 + 2378172. * w8 + 4341330. * w7 + 6806004. * w6 + 10622748. * w5 +
                          18739500. * w4 + 30651894. * w3 + 30869976. * w2 + 15431867. * w + 2919016.) / (146966400. * q4 * w7) * d2);
            double eta = e0 + (p1 / b + p2 / (b * b) + p3 / (b * b * b));
            double u = exp(-eta + mu * log(eta) - (1 + mu) * log(1 + mu) + mu);
            if (eta == mu) x = 1. / (1. + mu);
            else {
                x = eta < mu ? 0.5 * (1. / (1. + mu) + 1.) : 0.5 / (1. + mu);
                for (unsigned j = 0; j < nh; ++j) {
                    if (x <= 0.0) return 0.0;
                    if (x >= 1.) return 1.0;
                    double err = x * pow(1 - x, mu) - u, y = 1. - x;
                    double der1 = pow(y, mu) - mu * x * pow(y, mu - 1), der2 = mu * (mu - 1.) * x * pow(y, mu - 2.);
                    double t = 2 * err * der1 / (2. * pow(der1, 2) - err * der2);
                    x -= t;
                    if (fabs(t) < 0.1 * x) break;
                }
            }
            x = 1 - x;
        }
    } else if (a < 1. && b < 1.) {
        if (p > gsl_sf_beta_inc(a, b, (1. - a) / (2. - a - b))) {
            double t = pow(b * q * gsl_sf_beta(b, a), 1. / b);
            x = 1 - t / (1 + t);
        } else {
            double t = pow(a * p * gsl_sf_beta(a, b), 1. / a);
            x = t / (1 + t);
        }
    } else if (a > 1. && b > 1.) {
        if (p > gsl_sf_beta_inc(b, a, (1. - b) / (2. - b - a))) {
            double t = pow(b * q * gsl_sf_beta(b, a), 1. / b);
            x = 1. - t + (a - 1.) / (b + 1.) * t * t + (a - 1.) * (b * b + 3. * a * b - b + 5. * a - 4.) / (2. * pow(b + 1., 2) * (b + 2.)) * t * t * t;
        } else {
            double t = pow(a * p * gsl_sf_beta(a, b), 1. / a);
            x = t + (b - 1.) / (a + 1.) * t * t + (b - 1.) * (a * a + 3. * b * a - a + 5. * b - 4.) / (2. * pow(a + 1., 2) * (a + 2.)) * t * t * t;
        }
    } else if (a <= 1. && b > 1.) {
        x = pow(1 - pow(q, a * gsl_sf_beta(b, a)), 1. / a);
    }
    if (x <= 0) x = 0.;
    else if (x >= 1.) x = 1.;
    double bfi = 1. / gsl_sf_beta(a, b), a1 = a - 1., a2 = a1 - 1., b1 = b - 1., b2 = b1 - 1.;
    for (unsigned j = 0; j < nh; ++j) {
        if (x <= 0.0) return 0.0;
        if (x >= 1.) return 1.0;
        double err = gsl_sf_beta_inc(a, b, x) - p, y = 1. - x;
        double xa1 = pow(x, a1), xa2 = pow(x, a2), yb1 = pow(y, b1), yb2 = pow(y, b2);
        double der1 = xa1 * yb1 * bfi, der2 = bfi * (xa2 * yb1 - xa1 * yb2);
        double t = 2 * err * der1 / (2. * pow(der1, 2) - err * der2);
        x -= t;
        if (fabs(t) < EPS * x) break;
    }
    return sw ? 1 - x : x;
}

/* ------------------------------------------------------------- Furman */
typedef struct {
    double p1EInf, p1Ehat, eEHat, w, p, e1, e2;
    double p1RInf, eR, r, r1, r2, q, sigmaE;
    double deltaTSHat, s, eHat0, t1, t2, t3, t4;
    double theta0max, deltaERmax;
    double epsN[10], pSmallN[10];
    double particle_mass;
    int32_t m, scaleSigmaE, compat_last, reserved;
} orc_furman_t;

typedef struct {
    int mode;
    const double *u;  /* mode 1: uniforms of the current particle */
    int d;
} Src;

static double s_rand(Src *s) { return s->mode == 0 ? orc_rand() : s->u[s->d++]; }
static double s_randn(Src *s) {
    if (s->mode == 0) return orc_randn();
    double u1 = 1.0 - s->u[s->d++], u2 = s->u[s->d++];
    return sqrt(-2.0 * log(u1)) * cos(2.0 * PI * u2);
}

static double clipd(double x, double lo, double hi) {
    if (x <= hi && x >= lo) return x;
    if (x < lo) return lo;
    return hi;
}

/* Returns the number of secondaries (written to out, at most out_cap rows).
 * mode 0: MT stream; mode 1: uniforms[32*n_abs].  warn[2]: warning counts. */
int64_t orc_furman_emit(const orc_furman_t *f, const double *ab, const double *nv, int64_t n0, int mode,
                        const double *uniforms, double *out, int64_t out_cap, int32_t *warn) {
    const double eF = 0.5 * f->particle_mass / 1.602176565e-19, eFi = 1. / eF;
    double *e0 = (double *)malloc(sizeof(double) * (n0 > 0 ? n0 : 1));
    int *ns = (int *)malloc(sizeof(int) * (n0 > 0 ? n0 : 1));
    double pN[11], dE = 0, dR = 0;
    Src src = {mode, NULL, 0};
    for (int64_t j = 0; j < n0; ++j) {
        const double *r = ab + 6 * j;
        double v0 = sqrt(r[2] * r[2] + r[3] * r[3] + r[4] * r[4]);
        e0[j] = eF * v0 * v0;
        double th = acos((r[2] * nv[2 * j] + r[3] * nv[2 * j + 1]) / v0);
        if (th > 0.5 * PI) th = PI - th;
        th = clipd(th, 0., f->theta0max);
        dE = (f->p1EInf + (f->p1Ehat - f->p1EInf) * exp(-pow(fabs(e0[j] - f->eEHat) / f->w, f->p) / f->p)) *
             (1 + f->e1 * (1 - pow(cos(th), f->e2)));
        dR = f->p1RInf * (1 - exp(-pow(e0[j] / f->eR, f->r))) * (1 + f->r1 * (1 - pow(cos(th), f->r2)));
        double eHat = f->eHat0 * (1 + f->t3 * (1 - pow(cos(th), f->t4)));
        double dTS = f->deltaTSHat * f->s * e0[j] / eHat / (f->s - 1 + pow(e0[j] / eHat, f->s)) *
                     (1 + f->t1 * (1 - pow(cos(th), f->t2)));
        double t = dE + dR;
        if (t >= f->deltaERmax) { dE = dE / t * f->deltaERmax; dR = dR / t * f->deltaERmax; warn[0]++; }
        double dTSp = dTS / (1 - dE - dR);
        if (dTSp >= f->m) { dTSp = f->m; warn[1]++; }
        else if (dTSp < 0) dTSp = 0;
        double pr = dTSp / f->m;
        for (int i = 0; i <= f->m; ++i) pN[i] = gsl_ran_binomial_pdf(i, pr, f->m) * (1 - dE - dR);
        pN[1] += dE + dR;
        if (mode == 1) { src.u = uniforms + 32 * j; src.d = 0; }
        double u = s_rand(&src), cum = 0;
        ns[j] = f->m;
        for (int i = 0; i < f->m; ++i) {
            cum += pN[i];
            if (u <= cum) { ns[j] = i; break; }
        }
    }
    /* pass 2; dE, dR, pN[1] are the last particle's (particleEmitter.pyx:245) */
    const double lastE = dE, lastR = dR, lastP1 = pN[1];
    int64_t cur = 0;
    double eSec[10], th[10], yk[10];
    for (int64_t j = 0; j < n0; ++j) {
        int n = ns[j];
        if (n == 0) continue;
        const double *r = ab + 6 * j;
        if (mode == 1) { src.u = uniforms + 32 * j; src.d = 1; }
        if (n == 1) {
            double myE = dE, myR = dR, myP1 = pN[1];
            if (!f->compat_last) {
                /* recompute this particle's own split (non-compat variant) */
                double v0 = sqrt(r[2] * r[2] + r[3] * r[3] + r[4] * r[4]);
                double thh = acos((r[2] * nv[2 * j] + r[3] * nv[2 * j + 1]) / v0);
                if (thh > 0.5 * PI) thh = PI - thh;
                thh = clipd(thh, 0., f->theta0max);
                myE = (f->p1EInf + (f->p1Ehat - f->p1EInf) * exp(-pow(fabs(e0[j] - f->eEHat) / f->w, f->p) / f->p)) *
                      (1 + f->e1 * (1 - pow(cos(thh), f->e2)));
                myR = f->p1RInf * (1 - exp(-pow(e0[j] / f->eR, f->r))) * (1 + f->r1 * (1 - pow(cos(thh), f->r2)));
                double eHat = f->eHat0 * (1 + f->t3 * (1 - pow(cos(thh), f->t4)));
                double dTS = f->deltaTSHat * f->s * e0[j] / eHat / (f->s - 1 + pow(e0[j] / eHat, f->s)) *
                             (1 + f->t1 * (1 - pow(cos(thh), f->t2)));
                double t = myE + myR;
                if (t >= f->deltaERmax) { myE = myE / t * f->deltaERmax; myR = myR / t * f->deltaERmax; }
                double dTSp = dTS / (1 - myE - myR);
                if (dTSp >= f->m) dTSp = f->m; else if (dTSp < 0) dTSp = 0;
                myP1 = gsl_ran_binomial_pdf(1, dTSp / f->m, f->m) * (1 - myE - myR) + (myE + myR);
            } else {
                myE = lastE; myR = lastR; myP1 = lastP1;
            }
            double aE = myE / myP1, aR = myR / myP1, u = s_rand(&src);
            if (u < aE) {
                double sig = f->scaleSigmaE ? f->sigmaE * sqrt(e0[j] / 300) : f->sigmaE;
                eSec[0] = e0[j] - fabs(sig * s_randn(&src));
                if (eSec[0] < 0.) eSec[0] = s_rand(&src) * e0[j];
            } else if (u < aE + aR) {
                eSec[0] = e0[j] * pow(s_rand(&src), 1. / (1. + f->q));
            } else {
                eSec[0] = f->epsN[0] * orc_gammaincinv(f->pSmallN[0], s_rand(&src) * gsl_sf_gamma_inc_P(f->pSmallN[0], e0[j] / f->epsN[0]));
            }
        } else {
            double P = f->pSmallN[n - 1], eps = f->epsN[n - 1];
            double p0 = gsl_sf_gamma_inc_P(n * P, e0[j] / eps);
            for (int i = 0; i < n - 1; ++i) th[i] = asin(sqrt(orc_betaincinv(P * (n - i - 1), P, s_rand(&src))));
            double y = sqrt(orc_gammaincinv(n * P, s_rand(&src) * p0));
            yk[0] = y * cos(th[0]);
            yk[n - 1] = y;
            for (int i = 0; i < n - 1; ++i) yk[n - 1] *= sin(th[i]);
            for (int i = 1; i < n - 1; ++i) {
                yk[i] = y * cos(th[i]);
                for (int k = 0; k < i; ++k) yk[i] *= sin(th[k]);
            }
            for (int i = 0; i < n; ++i) eSec[i] = eps * (yk[i] * yk[i]);
        }
        for (int i = 0; i < n; ++i) {
            double vs = sqrt(eFi * eSec[i]);
            double tS = asin(s_rand(&src)), cT = cos(tS), sT = sin(tS);
            double pS = s_rand(&src) * PI * 2., cP = cos(pS), sP = sin(pS);
            double n0 = nv[2 * j], n1 = nv[2 * j + 1];
            double t1 = cT * n0 - sT * n1, t2 = sT * n0 + cT * n1;
            if (cur < out_cap) {
                double *q = out + 6 * cur;
                q[0] = r[0];
                q[1] = r[1];
                q[5] = r[5];
                q[2] = vs * ((cP + n0 * n0 * (1 - cP)) * t1 + n0 * n1 * (1 - cP) * t2);
                q[3] = vs * ((cP + n1 * n1 * (1 - cP)) * t2 + n0 * n1 * (1 - cP) * t1);
                q[4] = vs * (-sP * n1 * t1 + sP * n0 * t2);
            }
            ++cur;
        }
    }
    free(e0);
    free(ns);
    return cur;
}

/* number of secondaries per absorbed row (pass 1 only), for tests */
void orc_furman_counts(const orc_furman_t *f, const double *ab, const double *nv, int64_t n0, const double *uniforms,
                       int32_t *counts) {
    double *tmp = (double *)malloc(sizeof(double) * 6 * 10 * (n0 > 0 ? n0 : 1));
    int32_t warn[2] = {0, 0};
    for (int64_t j = 0; j < n0; ++j) {
        int64_t k = orc_furman_emit(f, ab + 6 * j, nv + 2 * j, 1, 1, uniforms + 32 * j, tmp, 10, warn);
        counts[j] = (int32_t)k;
    }
    free(tmp);
}

/* homoLoader (particleEmitter.pyx:41-72) with the MT stream: kind 0 rect,
 * 1 ellipse (the cut-cell predicate is exercised through the reference). */
void orc_homo_loader(int kind, double lx, double ly, int64_t n, double w0, double vsigma, int randomize, double *pd) {
    for (int64_t i = 0; i < n; ++i) {
        double x, y;
        for (;;) {
            x = (orc_rand() - 0.5) * lx;
            y = (orc_rand() - 0.5) * ly;
            int in = kind == 0 ? !(x < -lx * 0.5 || x > lx * 0.5 || y < -ly * 0.5 || y > ly * 0.5)
                               : !(pow(x, 2) * (4. / pow(lx, 2)) + pow(y, 2) * (4. / pow(ly, 2)) >= 1.);
            if (in) break;
        }
        pd[6 * i] = x;
        pd[6 * i + 1] = y;
        pd[6 * i + 2] = orc_randn() * vsigma;
        pd[6 * i + 3] = orc_randn() * vsigma;
        pd[6 * i + 4] = orc_randn() * vsigma;
    }
    for (int64_t i = 0; i < n; ++i) pd[6 * i + 5] = randomize ? w0 * (0.5 + orc_rand()) : w0;
}

/* ------------------------------------------------------------------------
 * SecElecEmitter (particleEmitter.pyx:316-484) and SimpleSecEmitter
 * (:489-597).  orc_secelec_t holds the stainless parameters of stainlessMod
 * (:331-352) after seyMax / reflec.  Draw order (mode 0 = the reference's):
 * pass 1 per particle: E decision, R decision, TS rounding (3 draws, :387-394);
 * pass 2 per particle: R speed factor if R (:435), TS: n normal deviates for
 * the lognormal energies (:445), n uniforms if their sum exceeds E0 (:448-450),
 * then theta and phi per TS secondary (:456-458).  SimpleSecEmitter: R speed
 * factor (:567), n uniform energies (:577), no angles.  mode 1: 64 injected
 * uniforms per particle consumed in that order from draw 0 (normal = Box-Muller
 * of two), the GPU kernel's layout.
 * ------------------------------------------------------------------------ */
typedef struct {
    int32_t model; /* 0 SecElecEmitter, 1 SimpleSecEmitter */
    int32_t max_ts;
    double p1EInf, p1Ehat, eEHat, w, p, e1, e2, p1RInf, eR, r, r1, r2;
    double deltaTSHat, s, eHat0, t1, t2, t3, t4, sigmaETS, muETS, theta0max, deltaERmax, q;
    double particle_mass;
} orc_secelec_t;

int64_t orc_secelec_emit(const orc_secelec_t *f, const double *ab, const double *nv, int64_t n0, int mode,
                         const double *uniforms, double *out, int64_t out_cap) {
    const double qe = 1.602176565e-19;
    const double mass = f->model == 1 ? 9.10938291e-31 : f->particle_mass;
    const double eF = 0.5 * mass / qe, eFi = 1. / eF;
    double *e0 = (double *)malloc(sizeof(double) * (n0 > 0 ? n0 : 1));
    int *nE = (int *)calloc(n0 > 0 ? n0 : 1, sizeof(int));
    int *nR = (int *)calloc(n0 > 0 ? n0 : 1, sizeof(int));
    int *nT = (int *)calloc(n0 > 0 ? n0 : 1, sizeof(int));
    Src src = {mode, NULL, 0};
    for (int64_t j = 0; j < n0; ++j) {
        const double *r = ab + 6 * j;
        double v0 = sqrt(r[2] * r[2] + r[3] * r[3] + r[4] * r[4]);
        e0[j] = eF * v0 * v0;
        double dE, dR, dTS;
        if (f->model == 1) {
            const double s = 1.813, eHat = 310;
            dE = 0.05;
            dR = 0.5;
            dTS = 1.4 * s * e0[j] / eHat / (s - 1 + pow(e0[j] / eHat, s));
        } else {
            double th = acos((r[2] * nv[2 * j] + r[3] * nv[2 * j + 1]) / v0);
            if (th > 0.5 * PI) th = PI - th;
            th = clipd(th, 0., f->theta0max);
            dE = (f->p1EInf + (f->p1Ehat - f->p1EInf) * exp(-pow(fabs(e0[j] - f->eEHat) / f->w, f->p) / f->p)) *
                 (1 + f->e1 * (1 - pow(cos(th), f->e2)));
            dR = f->p1RInf * (1 - exp(-pow(e0[j] / f->eR, f->r))) * (1 + f->r1 * (1 - pow(cos(th), f->r2)));
            double eHat = f->eHat0 * (1 + f->t3 * (1 - pow(cos(th), f->t4)));
            dTS = f->deltaTSHat * f->s * e0[j] / eHat / (f->s - 1 + pow(e0[j] / eHat, f->s)) *
                  (1 + f->t1 * (1 - pow(cos(th), f->t2)));
            double t = dE + dR;
            if (t >= f->deltaERmax) { dE = dE / t * f->deltaERmax; dR = dR / t * f->deltaERmax; }
        }
        if (mode == 1) { src.u = uniforms + 64 * j; src.d = 0; }
        if (s_rand(&src) <= dE) nE[j] = 1;
        if (s_rand(&src) <= dR) nR[j] = 1;
        unsigned fl = (unsigned)dTS;
        nT[j] = s_rand(&src) <= (dTS - fl) ? (int)fl + 1 : (int)fl;
        if (nT[j] > f->max_ts) nT[j] = f->max_ts;
    }
    int64_t cur = 0;
    double eSec[64];
    for (int64_t j = 0; j < n0; ++j) {
        const double *r = ab + 6 * j;
        if (mode == 1) { src.u = uniforms + 64 * j; src.d = 3; }
        double *q;
        if (nE[j]) {
            if (cur < out_cap) {
                q = out + 6 * cur;
                q[0] = r[0]; q[1] = r[1]; q[5] = r[5];
                q[2] = -r[2]; q[3] = -r[3]; q[4] = -r[4];
            }
            ++cur;
        }
        if (nR[j]) {
            double vF = f->model == 1 ? sqrt(s_rand(&src)) : sqrt(pow(s_rand(&src), 1. / (1. + f->q)));
            if (cur < out_cap) {
                q = out + 6 * cur;
                q[0] = r[0]; q[1] = r[1]; q[5] = r[5];
                q[2] = -r[2] * vF; q[3] = -r[3] * vF; q[4] = -r[4] * vF;
            }
            ++cur;
        }
        int n = nT[j];
        if (n <= 0) continue;
        if (f->model == 1) {
            for (int i = 0; i < n; ++i) eSec[i] = s_rand(&src) * 5;
            for (int i = 0; i < n; ++i) {
                double vF = sqrt(eSec[i] / e0[j]);
                if (cur < out_cap) {
                    q = out + 6 * cur;
                    q[0] = r[0]; q[1] = r[1]; q[5] = r[5];
                    q[2] = -r[2] * vF; q[3] = -r[3] * vF; q[4] = -r[4] * vF;
                }
                ++cur;
            }
            continue;
        }
        double eSum = 0.;
        for (int i = 0; i < n; ++i) {
            eSec[i] = exp(f->sigmaETS * s_randn(&src) + f->muETS);
            eSum += eSec[i];
        }
        if (eSum > e0[j])
            for (int i = 0; i < n; ++i) eSec[i] = s_rand(&src) * e0[j] / n;
        for (int i = 0; i < n; ++i) {
            double vs = sqrt(eFi * eSec[i]);
            double tS = asin(s_rand(&src)), cT = cos(tS), sT = sin(tS);
            double pS = s_rand(&src) * PI * 2., cP = cos(pS), sP = sin(pS);
            double n0v = nv[2 * j], n1v = nv[2 * j + 1];
            double t1 = cT * n0v - sT * n1v, t2 = sT * n0v + cT * n1v;
            if (cur < out_cap) {
                q = out + 6 * cur;
                q[0] = r[0]; q[1] = r[1]; q[5] = r[5];
                q[2] = vs * ((cP + n0v * n0v * (1 - cP)) * t1 + n0v * n1v * (1 - cP) * t2);
                q[3] = vs * ((cP + n1v * n1v * (1 - cP)) * t2 + n0v * n1v * (1 - cP) * t1);
                q[4] = vs * (-sP * n1v * t1 + sP * n0v * t2);
            }
            ++cur;
        }
    }
    free(e0);
    free(nE);
    free(nR);
    free(nT);
    return cur;
}
