// pcg.cu -- iterative Poisson solve: f64 iterative refinement around an f32
// flexible preconditioned conjugate-gradient solve (FCG with one stored
// direction) on the 5-point FIT
// operator, with the LU back-substitution (poisson.cu) as judge and fallback.
//
// Reference operator: PoissonSolver.__init__ (poissonSolver.pyx:41-58) builds
// A = S diag(meps) S^T over the inside nodes; A is applied here matrix-free
// from its edge weights (oec_stencil_t).  The solve itself has no counterpart
// in the reference, which only has the direct solve (poissonSolver.pyx:85).
//
// Per inner iteration three bandwidth-bound kernels over the extended grid
// (operator, update, new direction); the dot products go through f64 atomics
// into one of two accumulator slots (the slot of iteration k is zeroed by the
// last kernel of iteration k-1), so the host only reads a residual norm every
// kCheck iterations.
#include <math.h>
#include <stdint.h>

#include "oec_common.cuh"

namespace oec {

// Preconditioner application of the learned network (cnn.cu): z = M r on the
// extended grid, zero outside.
int cnn_precond_apply(const void *ctx, const float *r_dev, float *z_dev, cudaStream_t s);

namespace {

constexpr int kT = 256;
constexpr int kCheck = 8;            // inner iterations between host checks
constexpr double kInnerFloor = 1e-6;  // tightest inner relative residual asked of f32
constexpr int kMaxRefine = 12;

struct Acc {
    double pq, rz, rr, rzn, zq, pad0, pad1, pad2;
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
    return v;
}

// Sum of v over the CTA added to *out (one atomic per CTA).
__device__ __forceinline__ void cta_add(double v, double *out) {
    __shared__ double sh[kT / 32];
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        double s = l < kT / 32 ? sh[l] : 0.0;
        s = warp_sum(s);
        if (l == 0 && s != 0.0) atomicAdd(out, s);
    }
}

template <typename T>
__device__ __forceinline__ T apply_at(int i, int nx, const T *__restrict__ ex, const T *__restrict__ ey,
                                      const T *__restrict__ x) {
    const T xi = x[i];
    return ex[i] * (xi - x[i + 1]) + ex[i - 1] * (xi - x[i - 1]) + ey[i] * (xi - x[i + nx]) +
           ey[i - nx] * (xi - x[i - nx]);
}

// The same with the neighbours' values masked by the inside flags, for
// vectors from outside the solver (nonzero outside values are ignored).
__device__ __forceinline__ double apply_masked(int i, int nx, const double *__restrict__ ex,
                                               const double *__restrict__ ey, const uint8_t *__restrict__ in,
                                               const double *__restrict__ x) {
    const double xi = x[i];
    const double xe = in[i + 1] ? x[i + 1] : 0.0, xw = in[i - 1] ? x[i - 1] : 0.0;
    const double xn = in[i + nx] ? x[i + nx] : 0.0, xs = in[i - nx] ? x[i - nx] : 0.0;
    return ex[i] * (xi - xe) + ex[i - 1] * (xi - xw) + ey[i] * (xi - xn) + ey[i - nx] * (xi - xs);
}

__global__ void __launch_bounds__(kT) k_stencil64(int nx, int G, const double *__restrict__ ex,
                                                  const double *__restrict__ ey, const uint8_t *__restrict__ in,
                                                  const double *__restrict__ x, double *__restrict__ y) {
    for (int i = blockIdx.x * kT + threadIdx.x; i < G; i += gridDim.x * kT)
        y[i] = in[i] ? apply_masked(i, nx, ex, ey, in, x) : 0.0;
}

// r = q - A phi on the inside nodes (0 outside); nrm[0] += |r|^2, nrm[1] += |q|^2.
__global__ void __launch_bounds__(kT) k_residual64(int nx, int G, const double *__restrict__ ex,
                                                   const double *__restrict__ ey, const uint8_t *__restrict__ in,
                                                   const double *__restrict__ q, const double *__restrict__ phi,
                                                   double *__restrict__ r, double *nrm) {
    double rr = 0.0, qq = 0.0;
    for (int i = blockIdx.x * kT + threadIdx.x; i < G; i += gridDim.x * kT) {
        double v = 0.0;
        if (in[i]) {
            const double qi = q[i];
            v = qi - apply_masked(i, nx, ex, ey, in, phi);
            qq += qi * qi;
        }
        r[i] = v;
        rr += v * v;
    }
    cta_add(rr, nrm);
    cta_add(qq, nrm + 1);
}

// r32 = s * r64; z = M r32 (Jacobi or identity) unless the network computes
// it; p = z; acc.rz += r.z.
__global__ void __launch_bounds__(kT) k_init32(int G, const double *__restrict__ r64, double s,
                                               const float *__restrict__ dinv, int precond, int z_given,
                                               float *__restrict__ r, float *__restrict__ z, float *__restrict__ p,
                                               float *__restrict__ d, Acc *acc) {
    double rz = 0.0;
    for (int i = blockIdx.x * kT + threadIdx.x; i < G; i += gridDim.x * kT) {
        float ri, zi;
        if (z_given) {
            ri = r[i];
            zi = z[i];
        } else {
            ri = (float)(r64[i] * s);
            zi = precond == OEC_PRECOND_JACOBI ? ri * dinv[i] : ri;
            r[i] = ri;
            z[i] = zi;
        }
        p[i] = zi;
        d[i] = 0.0f;
        rz += (double)ri * (double)zi;
    }
    cta_add(rz, &acc->rz);
}

__global__ void __launch_bounds__(kT) k_scale32(int G, const double *__restrict__ r64, double s,
                                                float *__restrict__ r) {
    for (int i = blockIdx.x * kT + threadIdx.x; i < G; i += gridDim.x * kT) r[i] = (float)(r64[i] * s);
}

// q = A32 p; acc.pq += p.q
__global__ void __launch_bounds__(kT) k_apply32(int nx, int G, const float *__restrict__ ex,
                                                const float *__restrict__ ey, const uint8_t *__restrict__ in,
                                                const float *__restrict__ p, float *__restrict__ q, Acc *acc) {
    double pq = 0.0;
    for (int i = blockIdx.x * kT + threadIdx.x; i < G; i += gridDim.x * kT) {
        float v = 0.0f;
        if (in[i]) {
            v = apply_at(i, nx, ex, ey, p);
            pq += (double)p[i] * (double)v;
        }
        q[i] = v;
    }
    cta_add(pq, &acc->pq);
}

// alpha = rz / pq (the exact line search along p: r.p = r.z because r is
// orthogonal to the previous direction); d += alpha p; r -= alpha q;
// acc.rr += |r|^2.  Without a network preconditioner also z = M r,
// acc.rzn += r.z, acc.zq += z.q.  A non-positive or non-finite curvature
// leaves every vector unchanged and marks rr as NaN for the host.
__global__ void __launch_bounds__(kT) k_update32(int G, const float *__restrict__ dinv, int precond,
                                                 const float *__restrict__ p, const float *__restrict__ q,
                                                 float *__restrict__ d, float *__restrict__ r,
                                                 float *__restrict__ z, Acc *acc) {
    const double pq = acc->pq, rzv = acc->rz;
    if (!(pq > 0.0) || !isfinite(rzv)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) acc->rr = __longlong_as_double(0x7ff8000000000000LL);
        return;
    }
    const float alpha = (float)(rzv / pq);
    double rr = 0.0, rzn = 0.0, zq = 0.0;
    for (int i = blockIdx.x * kT + threadIdx.x; i < G; i += gridDim.x * kT) {
        const float qi = q[i];
        d[i] = fmaf(alpha, p[i], d[i]);
        const float ri = fmaf(-alpha, qi, r[i]);
        r[i] = ri;
        rr += (double)ri * (double)ri;
        if (precond != OEC_PRECOND_CNN) {
            const float zn = precond == OEC_PRECOND_JACOBI ? ri * dinv[i] : ri;
            z[i] = zn;
            rzn += (double)ri * (double)zn;
            zq += (double)zn * (double)qi;
        }
    }
    cta_add(rr, &acc->rr);
    if (precond != OEC_PRECOND_CNN) {
        cta_add(rzn, &acc->rzn);
        cta_add(zq, &acc->zq);
    }
}

// Network preconditioner: acc.rzn += r.z, acc.zq += z.q with z = M r from
// the network (z_new), copied into z.
__global__ void __launch_bounds__(kT) k_zdots32(int G, const float *__restrict__ r, const float *__restrict__ zn,
                                                const float *__restrict__ q, float *__restrict__ z, Acc *acc) {
    double rzn = 0.0, zq = 0.0;
    for (int i = blockIdx.x * kT + threadIdx.x; i < G; i += gridDim.x * kT) {
        const float a = zn[i];
        rzn += (double)r[i] * (double)a;
        zq += (double)a * (double)q[i];
        z[i] = a;
    }
    cta_add(rzn, &acc->rzn);
    cta_add(zq, &acc->zq);
}

// beta = -(z.q) / (p.q): the new direction p = z + beta p is A-conjugate to
// the previous one whatever the preconditioner (flexible CG, one stored
// direction).  One thread prepares the next slot: rz = r.z, other sums zero.
__global__ void __launch_bounds__(kT) k_direction32(int G, const float *__restrict__ z, float *__restrict__ p,
                                                    Acc *acc, Acc *next) {
    const double rz = acc->rz;
    double b = -acc->zq / acc->pq;
    if (!isfinite(b)) b = 0.0;
    const float beta = (float)b;
    if (isfinite(acc->rr) && isfinite(rz) && acc->pq > 0.0) {
        for (int i = blockIdx.x * kT + threadIdx.x; i < G; i += gridDim.x * kT) p[i] = fmaf(beta, p[i], z[i]);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // a breakdown (rr NaN) propagates: the next update sees rz NaN
        next->rz = isfinite(acc->rr) ? acc->rzn : acc->rr;
        next->pq = next->rr = next->rzn = next->zq = 0.0;
    }
}

// phi += c d on the inside nodes.
__global__ void __launch_bounds__(kT) k_accumulate64(int G, double c, const float *__restrict__ d,
                                                     const uint8_t *__restrict__ in, double *__restrict__ phi) {
    for (int i = blockIdx.x * kT + threadIdx.x; i < G; i += gridDim.x * kT)
        phi[i] = in[i] ? fma(c, (double)d[i], phi[i]) : 0.0;
}

struct Work {
    double *r64, *nrm;
    float *r, *z, *p, *q, *d, *zn;
    Acc *acc;
};

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

Work carve(void *base, int G) {
    char *c = static_cast<char *>(base);
    Work w;
    w.r64 = reinterpret_cast<double *>(c);
    c += align256(sizeof(double) * G);
    float **f[] = {&w.r, &w.z, &w.p, &w.q, &w.d, &w.zn};
    for (float **x : f) {
        *x = reinterpret_cast<float *>(c);
        c += align256(sizeof(float) * G);
    }
    w.acc = reinterpret_cast<Acc *>(c);
    c += align256(sizeof(Acc) * 2);
    w.nrm = reinterpret_cast<double *>(c);
    return w;
}

bool valid_stencil(const oec_stencil_t *st) {
    return st && st->nx >= 3 && st->ny >= 3 && (int64_t)st->nx * st->ny < (1 << 28) && st->ex64 && st->ey64 &&
           st->ex32 && st->ey32 && st->dinv32 && st->inside && st->scale32 > 0.0;
}

}  // namespace
}  // namespace oec

using namespace oec;

extern "C" int64_t oec_pcg_work_bytes(int32_t nx, int32_t ny) {
    const size_t G = (size_t)nx * (size_t)ny;
    return (int64_t)(align256(sizeof(double) * G) + 6 * align256(sizeof(float) * G) + align256(sizeof(Acc) * 2) +
                     256);
}

extern "C" int oec_stencil_apply(const oec_stencil_t *st, const double *x_dev, double *y_dev, void *stream) {
    if (!valid_stencil(st) || !x_dev || !y_dev) return OEC_ERR_INVALID;
    const int G = st->nx * st->ny;
    k_stencil64<<<persistent_grid((G + kT - 1) / kT, 8), kT, 0, as_stream(stream)>>>(st->nx, G, st->ex64, st->ey64,
                                                                                     st->inside, x_dev, y_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_pcg_solve(const oec_stencil_t *st, const double *q_dev, double *phi_dev, double tol,
                             int32_t max_iter, int32_t precond, const void *precond_ctx, void *work_dev,
                             oec_pcg_stats_t *stats, void *stream) {
    if (!valid_stencil(st) || !q_dev || !phi_dev || !work_dev || !stats || !(tol > 0.0) || max_iter < 0)
        return OEC_ERR_INVALID;
    if (precond < OEC_PRECOND_NONE || precond > OEC_PRECOND_CNN) return OEC_ERR_INVALID;
    if (precond == OEC_PRECOND_CNN && !precond_ctx) return OEC_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    const int nx = st->nx, G = st->nx * st->ny;
    const int grid = persistent_grid((G + kT - 1) / kT, 4);
    Work w = carve(work_dev, G);
    *stats = oec_pcg_stats_t{};
    int total = 0;
    double prev_rel = 0.0;
    for (int refine = 0; refine <= kMaxRefine; ++refine) {
        OEC_CUDA_TRY(cudaMemsetAsync(w.nrm, 0, 2 * sizeof(double), s));
        k_residual64<<<grid, kT, 0, s>>>(nx, G, st->ex64, st->ey64, st->inside, q_dev, phi_dev, w.r64, w.nrm);
        OEC_LAUNCH_CHECK();
        double h[2];
        OEC_CUDA_TRY(cudaMemcpyAsync(h, w.nrm, sizeof(h), cudaMemcpyDeviceToHost, s));
        OEC_CUDA_TRY(cudaStreamSynchronize(s));
        stats->refinements = refine + 1;
        const double rel = h[1] > 0.0 ? sqrt(h[0] / h[1]) : 0.0;
        if (refine == 0) stats->rel_residual0 = rel;
        stats->rel_residual = rel;
        if (!isfinite(rel)) break;
        if (rel <= tol || h[1] == 0.0) {
            stats->converged = 1;
            break;
        }
        if (total >= max_iter || refine == kMaxRefine) break;
        if (refine > 0 && rel > 0.5 * prev_rel) break;  // refinement no longer pays: stagnation
        prev_rel = rel;
        const double rnorm = sqrt(h[0]);
        // aim the f32 solve at the target when it can get there, so a good warm
        // start needs a single refinement
        const double inner_tol = fmax(kInnerFloor, 0.5 * tol / rel);
        // ---- inner f32 solve of (scale32 A) d = r / ||r||
        OEC_CUDA_TRY(cudaMemsetAsync(w.acc, 0, 2 * sizeof(Acc), s));
        if (precond == OEC_PRECOND_CNN) {
            k_scale32<<<grid, kT, 0, s>>>(G, w.r64, 1.0 / rnorm, w.r);
            OEC_LAUNCH_CHECK();
            int rc = cnn_precond_apply(precond_ctx, w.r, w.z, s);
            if (rc != OEC_OK) return rc;
            k_init32<<<grid, kT, 0, s>>>(G, w.r64, 1.0 / rnorm, st->dinv32, precond, 1, w.r, w.z, w.p, w.d, w.acc);
        } else {
            k_init32<<<grid, kT, 0, s>>>(G, w.r64, 1.0 / rnorm, st->dinv32, precond, 0, w.r, w.z, w.p, w.d, w.acc);
        }
        OEC_LAUNCH_CHECK();
        int slot = 0, it = 0;
        double best = 1.0, best_at = 0.0;
        while (total < max_iter) {
            Acc *a = w.acc + slot, *nxt = w.acc + (slot ^ 1);
            k_apply32<<<grid, kT, 0, s>>>(nx, G, st->ex32, st->ey32, st->inside, w.p, w.q, a);
            k_update32<<<grid, kT, 0, s>>>(G, st->dinv32, precond, w.p, w.q, w.d, w.r, w.z, a);
            if (precond == OEC_PRECOND_CNN) {
                int rc = cnn_precond_apply(precond_ctx, w.r, w.zn, s);
                if (rc != OEC_OK) return rc;
                k_zdots32<<<grid, kT, 0, s>>>(G, w.r, w.zn, w.q, w.z, a);
            }
            k_direction32<<<grid, kT, 0, s>>>(G, w.z, w.p, a, nxt);
            OEC_LAUNCH_CHECK();
            slot ^= 1;
            ++it;
            ++total;
            if (it % kCheck == 0 || total >= max_iter) {
                double rr;
                OEC_CUDA_TRY(cudaMemcpyAsync(&rr, &a->rr, sizeof(double), cudaMemcpyDeviceToHost, s));
                OEC_CUDA_TRY(cudaStreamSynchronize(s));
                if (!isfinite(rr)) {
                    stats->breakdown = 1;
                    break;
                }
                const double rel_in = sqrt(rr);
                if (rel_in <= inner_tol) break;
                // f32 stagnation: the best residual did not drop by 10 % in
                // 1024 iterations (CG residual norms are not monotone)
                if (rel_in < 0.9 * best) {
                    best = rel_in;
                    best_at = it;
                } else if (it - best_at >= 1024) {
                    break;
                }
            }
        }
        stats->iterations = total;
        k_accumulate64<<<grid, kT, 0, s>>>(G, st->scale32 * rnorm, w.d, st->inside, phi_dev);
        OEC_LAUNCH_CHECK();
    }
    stats->iterations = total;
    return OEC_OK;
}
