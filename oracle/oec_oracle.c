/*
 * oec_oracle.c -- CPU restatement of the openECLOUD per-step PIC algorithms,
 * in FP64, one function per reference routine.  TEST INFRASTRUCTURE ONLY:
 * called by tests/, by __graft_entry__.smoke() and by bench.py's CPU
 * baseline as the checker.  The product (openecloud_b200/) never links it.
 *
 * Pinning: the functions are checked against golden vectors produced by the
 * compiled reference itself (tests/golden/make_golden.py, oracle/_ref).
 * Particle data is the reference AoS layout: rows [x, y, vx, vy, vz, w].
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gsl/gsl_cdf.h"
#include "gsl/gsl_randist.h"
#include "gsl/gsl_rng.h"
#include "gsl/gsl_sf_gamma.h"

#define NC 6

/* ------------------------------------------------------------ RNG
 * One global MT19937 stream, as randomGen.pyx:22-35 keeps one. */
static gsl_rng *g_rng = NULL;

static gsl_rng *rng(void) {
    if (!g_rng) g_rng = gsl_rng_alloc(gsl_rng_mt19937);
    return g_rng;
}

void orc_seed(unsigned long s) { gsl_rng_set(rng(), s); }                       /* randomGen.pyx:25 */
double orc_rand(void) { return gsl_rng_uniform(rng()); }                         /* randomGen.pyx:28 */
double orc_randn(void) { return gsl_ran_gaussian_ziggurat(rng(), 1.0); }         /* randomGen.pyx:31 */
unsigned long orc_randi(unsigned long n) { return gsl_rng_uniform_int(rng(), n); } /* randomGen.pyx:34 */

/* ------------------------------------------------ particles.pyx:400-418 */
void orc_calc_grid_weights(const double *pd, int64_t n, double dxi, double dyi, double lxh, double lyh,
                           uint32_t nx, uint32_t *in_cell, double *w00, double *w10, double *w01,
                           double *w11) {
    for (int64_t i = 0; i < n; ++i) {
        double ux = (pd[NC * i] + lxh) * dxi;
        double uy = (pd[NC * i + 1] + lyh) * dyi;
        uint32_t ix = (uint32_t)ux, iy = (uint32_t)uy;
        in_cell[i] = ix + iy * nx;
        ux -= ix;
        uy -= iy;
        w00[i] = (1 - ux) * (1 - uy);
        w10[i] = ux * (1 - uy);
        w01[i] = (1 - ux) * uy;
        w11[i] = ux * uy;
    }
}

/* ------------------------------------------------ particles.pyx:336-351 */
void orc_charge_to_grid(const double *pd, int64_t n, const uint32_t *in_cell, const double *w00,
                        const double *w10, const double *w01, const double *w11, double charge,
                        uint32_t nx, uint32_t np, double *q) {
    for (uint32_t k = 0; k < np; ++k) q[k] = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        uint32_t c = in_cell[i];
        double wq = pd[NC * i + 5] * charge;
        q[c] += w00[i] * pd[NC * i + 5] * charge;
        q[c + 1] += w10[i] * pd[NC * i + 5] * charge;
        q[c + nx] += w01[i] * pd[NC * i + 5] * charge;
        q[c + nx + 1] += w11[i] * pd[NC * i + 5] * charge;
        (void)wq;
    }
}

/* ------------------------------------------- particles.pyx:354-397 (ncomp 2|3) */
void orc_field_to_particles(const double *field, int ncomp, const uint32_t *in_cell, const double *w00,
                            const double *w10, const double *w01, const double *w11, uint32_t nx,
                            uint32_t np, int64_t n, double *out) {
    for (int64_t i = 0; i < n; ++i) {
        uint32_t c = in_cell[i];
        for (int k = 0; k < ncomp; ++k) {
            const double *f = field + (size_t)k * np;
            double s = w00[i] * f[c];
            s += w10[i] * f[c + 1];
            s += w01[i] * f[c + nx];
            s += w11[i] * f[c + nx + 1];
            out[ncomp * i + k] = s;
        }
    }
}

/* --------------------------- particles.pyx:324-333 / :298-321 / :272-295 */
void orc_boris_push(double *pd, int64_t n, const double *e_at, const double *b_at, const double *bconst,
                    double dt, double qm, int type_b) {
    if (type_b == 0) {
        double k = qm * dt;
        for (int64_t i = 0; i < n; ++i) {
            double *r = pd + NC * i;
            r[2] += k * e_at[2 * i];
            r[3] += k * e_at[2 * i + 1];
            r[0] += dt * r[2];
            r[1] += dt * r[3];
        }
        return;
    }
    double h = 0.5 * qm * dt;
    for (int64_t i = 0; i < n; ++i) {
        double *r = pd + NC * i;
        double t0, t1, t2;
        if (type_b == 1) {
            t0 = h * bconst[0]; t1 = h * bconst[1]; t2 = h * bconst[2];
        } else {
            t0 = h * b_at[3 * i]; t1 = h * b_at[3 * i + 1]; t2 = h * b_at[3 * i + 2];
        }
        r[2] += h * e_at[2 * i];
        r[3] += h * e_at[2 * i + 1];
        double v0 = r[2] + r[3] * t2 - r[4] * t1;
        double v1 = r[3] + r[4] * t0 - r[2] * t2;
        double v2 = r[4] + r[2] * t1 - r[3] * t0;
        double f = 2. / (1. + t0 * t0 + t1 * t1 + t2 * t2);
        double s0 = t0 * f, s1 = t1 * f, s2 = t2 * f;
        r[2] += v1 * s2 - v2 * s1 + h * e_at[2 * i];
        r[3] += v2 * s0 - v0 * s2 + h * e_at[2 * i + 1];
        r[4] += v0 * s1 - v1 * s0;
        r[0] += dt * r[2];
        r[1] += dt * r[3];
    }
}

/* ------------------------------- particleBoundary.pyx inside predicates */
/* AbsorbRectangular.indexInside :84-97 */
void orc_index_inside_rect(const double *pd, int64_t n, double lx, double ly, uint16_t *inside) {
    double hx = lx * 0.5, hy = ly * 0.5;
    for (int64_t i = 0; i < n; ++i) {
        double x = pd[NC * i], y = pd[NC * i + 1];
        inside[i] = (x < -hx || x > hx || y < -hy || y > hy) ? 0 : 1;
    }
}

/* AbsorbElliptical.indexInside :227-242 */
void orc_index_inside_ellipse(const double *pd, int64_t n, double lx, double ly, uint16_t *inside) {
    double ax = 4. / (lx * lx), ay = 4. / (ly * ly);
    for (int64_t i = 0; i < n; ++i) {
        double x = pd[NC * i], y = pd[NC * i + 1];
        inside[i] = (x * x * ax + y * y * ay >= 1.) ? 0 : 1;
    }
}

/* _clipParticleDataToGrid :485-508; returns 1 if any row was clipped */
int orc_clip_to_grid(double *pd, int64_t n, double lxh, double lyh) {
    int flag = 0;
    for (int64_t i = 0; i < n; ++i) {
        double *r = pd + NC * i;
        if (r[0] > lxh) { r[0] = lxh; flag = 1; }
        else if (r[0] < -lxh) { r[0] = -lxh; flag = 1; }
        if (r[1] > lyh) { r[1] = lyh; flag = 1; }
        else if (r[1] < -lyh) { r[1] = -lyh; flag = 1; }
    }
    return flag;
}

/* AbsorbArbitraryCutCell.indexInside :336-370 (clip included) */
void orc_index_inside_cutcell(double *pd, int64_t n, double lxh_ext, double lyh_ext, double dx, double dy,
                              uint32_t nx, const uint16_t *faces, const double *bpts, const int32_t *cpi,
                              uint16_t *inside) {
    orc_clip_to_grid(pd, n, lxh_ext - 1.e-6 * dx, lyh_ext - 1.e-6 * dy);
    double dxi = 1. / dx, dyi = 1. / dy;
    for (int64_t i = 0; i < n; ++i) {
        double x = pd[NC * i], y = pd[NC * i + 1];
        uint32_t ix = (uint32_t)((x + lxh_ext) * dxi), iy = (uint32_t)((y + lyh_ext) * dyi);
        uint32_t c = ix + iy * nx;
        if (faces[c] == 8) inside[i] = 1;
        else if (faces[c] == 0) inside[i] = 0;
        else {
            int32_t a = cpi[2 * c], b = cpi[2 * c + 1];
            inside[i] = ((bpts[2 * a] - x) * (bpts[2 * b + 1] - y) > (bpts[2 * b] - x) * (bpts[2 * a + 1] - y)) ? 1 : 0;
        }
    }
}

/* ParticleBoundary.saveAbsorbed :38-65: rows with inside==0, in order. */
int64_t orc_save_absorbed(const double *pd, int64_t n, const uint16_t *inside, double *absorbed) {
    int64_t k = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (inside[i] == 0) {
            memcpy(absorbed + NC * k, pd + NC * i, NC * sizeof(double));
            ++k;
        }
    }
    return k;
}

/* AbsorbRectangular.calculateInteractionPoint :99-192 + calculateNormalVectors :195-221 */
void orc_interaction_rect(double *ab, int64_t n, double lx, double ly, double dx, double dy, double *normals) {
    double eps = 1e-6;
    double hx = lx * 0.5 - dx * eps, hy = ly * 0.5 - dy * eps;
    for (int64_t i = 0; i < n; ++i) {
        double *r = ab + NC * i;
        int xs = 1, ys = 1;  /* 0 below, 1 inside, 2 above */
        if (r[0] > hx) xs = 2; else if (r[0] < -hx) xs = 0;
        if (r[1] > hy) ys = 2; else if (r[1] < -hy) ys = 0;
        double t, tx, ty;
        int where;
        if (xs == 0 && ys == 1) { t = (r[0] + hx) / r[2]; where = 0; }
        else if (xs == 2 && ys == 1) { t = (r[0] - hx) / r[2]; where = 1; }
        else if (xs == 1 && ys == 0) { t = (r[1] + hy) / r[3]; where = 2; }
        else if (xs == 1 && ys == 2) { t = (r[1] - hy) / r[3]; where = 3; }
        else {
            tx = (xs == 0) ? (r[0] + hx) / r[2] : (r[0] - hx) / r[2];
            ty = (ys == 0) ? (r[1] + hy) / r[3] : (r[1] - hy) / r[3];
            /* the reference's corner labels (:163-190), kept as written */
            if (xs == 0 && ys == 0) where = (tx > ty) ? 0 : 1;
            else if (xs == 2 && ys == 0) where = (tx > ty) ? 2 : 1;
            else if (xs == 0 && ys == 2) where = (tx > ty) ? 0 : 3;
            else where = (tx > ty) ? 2 : 3;
            t = (tx > ty) ? tx : ty;
        }
        r[0] -= t * r[2];
        r[1] -= t * r[3];
        double nx_ = 0, ny_ = 0;
        if (where == 0) { nx_ = 1.; ny_ = 0.; }
        else if (where == 1) { nx_ = -1.; ny_ = 0.; }
        else if (where == 2) { nx_ = 0.; ny_ = 1.; }
        else { nx_ = 0.; ny_ = -1.; }
        normals[2 * i] = nx_;
        normals[2 * i + 1] = ny_;
    }
}

/* AbsorbElliptical.calculateInteractionPoint :252-274 + calculateNormalVectors :277-297 */
void orc_interaction_ellipse(double *ab, int64_t n, double lx, double ly, double dx, double dy,
                             double *normals) {
    double eps = 1.e-6;
    double ax = 4. / pow(lx - eps * dx, 2), ay = 4. / pow(ly - eps * dy, 2);
    for (int64_t i = 0; i < n; ++i) {
        double *r = ab + NC * i;
        double c = pow(r[0], 2) * ax + pow(r[1], 2) * ay - 1.;
        double b = r[0] * r[2] * ax + r[1] * r[3] * ay;
        double a = pow(r[2], 2) * ax + pow(r[3], 2) * ay;
        double t = (b - sqrt(b * b - a * c)) / a;
        r[0] -= t * r[2];
        r[1] -= t * r[3];
    }
    double nx2 = 4. / (lx * lx), ny2 = 4. / (ly * ly);
    double nx4 = nx2 * nx2, ny4 = ny2 * ny2;
    for (int64_t i = 0; i < n; ++i) {
        double *r = ab + NC * i;
        double inv = 1. / sqrt(pow(r[0], 2) * nx4 + pow(r[1], 2) * ny4);
        normals[2 * i] = -r[0] * nx2 * inv;
        normals[2 * i + 1] = -r[1] * ny2 * inv;
    }
}

/* AbsorbArbitraryCutCell.calculateInteractionPoint :373-446 + calculateNormalVectors :449-481.
 * Returns the number of particles whose wall intersection was not found. */
int64_t orc_interaction_cutcell(double *ab, int64_t n, double dt, double lxh_ext, double lyh_ext, double dx,
                                double dy, uint32_t nx, const uint16_t *faces, const double *bpts,
                                const int32_t *cpi, const double *cnorm, double *normals) {
    double dxi = 1. / dx, dyi = 1. / dy, eps = 1.e-6;
    int64_t missing = 0;
    for (int64_t i = 0; i < n; ++i) {
        double *r = ab + NC * i;
        uint32_t ix = (uint32_t)((r[0] + lxh_ext) * dxi), iy = (uint32_t)((r[1] + lyh_ext) * dyi);
        uint32_t cell = ix + iy * nx;
        double rx = -dt * r[2], ry = -dt * r[3];
        int xd[2] = {0, rx < 0. ? -1 : 1};
        int yd[2] = {0, ry < 0. ? -1 : 1};
        int found = 0;
        for (int a = 0; a < 2 && !found; ++a) {
            for (int b = 0; b < 2; ++b) {
                uint32_t cc = (uint32_t)((int64_t)cell + xd[a] + (int64_t)yd[b] * nx);
                if (faces[cc] == 0 || faces[cc] == 8) continue;
                int32_t p0 = cpi[2 * cc], p1 = cpi[2 * cc + 1];
                double sx = bpts[2 * p1] - bpts[2 * p0];
                double sy = bpts[2 * p1 + 1] - bpts[2 * p0 + 1];
                double rxs = rx * sy - ry * sx;
                if (rxs != 0.) {
                    double qx = bpts[2 * p0] - r[0], qy = bpts[2 * p0 + 1] - r[1];
                    double t = (qx * sy - qy * sx) / rxs;
                    double u = (qx * ry - qy * rx) / rxs;
                    if (-eps <= t && t <= 1. + eps && -eps <= u && u <= 1. + eps) {
                        r[0] += t * rx * (1. + eps);
                        r[1] += t * ry * (1. + eps);
                        found = 1;
                        break;
                    }
                }
            }
        }
        if (!found) ++missing;
    }
    for (int64_t i = 0; i < n; ++i) {
        double *r = ab + NC * i;
        uint32_t ix = (uint32_t)((r[0] + lxh_ext) * dxi), iy = (uint32_t)((r[1] + lyh_ext) * dyi);
        uint32_t cell = ix + iy * nx;
        normals[2 * i] = cnorm[2 * cell];
        normals[2 * i + 1] = cnorm[2 * cell + 1];
    }
    return missing;
}
