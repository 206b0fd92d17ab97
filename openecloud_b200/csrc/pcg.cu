// pcg.cu -- iterative Poisson solve: f64 iterative refinement around an f32
// flexible preconditioned conjugate-gradient solve (FCG with one stored
// direction) on the 5-point FIT operator, with the LU back-substitution
// (poisson.cu) as its fallback and the reference its error is measured
// against.
//
// Reference operator: PoissonSolver.__init__ (poissonSolver.pyx:41-58) builds
// A = S diag(meps) S^T over the inside nodes; A is applied here matrix-free
// from its edge weights (oec_stencil_t).  The solve itself has no counterpart
// in the reference, which only has the direct solve (poissonSolver.pyx:85).
//
// Per inner iteration three bandwidth-bound kernels over the extended grid
// (operator, update, new direction) plus the preconditioner; the dot
// products go through f64 atomics into one of two accumulator slots (the
// slot of iteration k is zeroed by the last kernel of iteration k-1).  The
// whole solve -- refinement loop, inner loop, convergence checks and the
// optional LU fallback -- is one CUDA graph of conditional nodes whose
// conditions the kernels set, so it needs no host round trip and can itself
// be captured into a larger graph (a buildup time step).
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include <cooperative_groups.h>

#include <map>
#include <mutex>
#include <string>

#include "oec_common.cuh"

namespace oec {

// Preconditioner application of the learned network (cnn.cu): z = M r on the
// extended grid, zero outside.
int cnn_precond_apply(const void *ctx, const float *r_dev, float *z_dev, cudaStream_t s);

namespace {

constexpr int kT = 256;
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

// r = q - A phi on the inside nodes (0 outside); nrm[0] += |r|^2,
// nrm[1] += |q|^2.  First kernel of a refinement: it disarms the refinement
// loop, which only k_refine_begin re-arms.
__global__ void __launch_bounds__(kT) k_residual64(int nx, int G, const double *__restrict__ ex,
                                                   const double *__restrict__ ey, const uint8_t *__restrict__ in,
                                                   const double *__restrict__ q, const double *__restrict__ phi,
                                                   double *__restrict__ r, double *nrm,
                                                   cudaGraphConditionalHandle h_outer) {
    if (blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h_outer, 0);
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

// Device-side state of one solve (in the work area).  Every loop decision of
// the solve is taken on the device from these values, so a whole solve runs
// as one graph without host round trips.
struct Ctl {
    double nrm[2];             // |r|^2, |q|^2 of the refinement's f64 residual (atomics)
    double prev_rel;           // f64 relative residual at the previous refinement
    double inner_tol;          // relative residual asked of the current f32 solve
    double inv_rnorm;          // 1 / ||r|| of the current refinement
    double coef;               // scale32 * ||r||: weight of the f32 correction
    double best;               // best inner residual so far (stagnation window)
    double pq_prev;            // p.Ap of the previous inner iteration (k_cg_step)
    int slot, it, total, refine, best_at, ticket;
    oec_pcg_stats_t stats;     // stats of the synchronous entry point
};

// Start of a refinement (one thread), after k_residual64: record the f64
// residual, decide whether to stop (converged, iteration budget, refinement
// limit, or the last refinement gained less than 2x) and otherwise set up the
// f32 solve of (scale32 A) d = r / ||r|| with the inner tolerance aimed at
// tol.  h_outer continues the refinement loop, h_work runs this refinement.
__global__ void k_refine_begin(Ctl *c, Acc *acc, double tol, int max_iter, double scale32, oec_pcg_stats_t *stats,
                               cudaGraphConditionalHandle h_outer, cudaGraphConditionalHandle h_work) {
    if (threadIdx.x != 0) return;
    const double h0 = c->nrm[0], h1 = c->nrm[1];
    c->nrm[0] = c->nrm[1] = 0.0;
    const int refine = c->refine;
    const double rel = h1 > 0.0 ? sqrt(h0 / h1) : 0.0;
    stats->refinements = refine + 1;
    if (refine == 0) stats->rel_residual0 = rel;
    stats->rel_residual = rel;
    stats->iterations = c->total;
    int work = 0;
    if (isfinite(rel)) {
        if (rel <= tol || h1 == 0.0) {
            stats->converged = 1;
        } else if (c->total < max_iter && refine < kMaxRefine && !(refine > 0 && rel > 0.5 * c->prev_rel)) {
            work = 1;
            c->prev_rel = rel;
            const double rnorm = sqrt(h0);
            c->inner_tol = fmax(kInnerFloor, 0.5 * tol / rel);
            c->inv_rnorm = 1.0 / rnorm;
            c->coef = scale32 * rnorm;
            acc[0] = Acc{};
            acc[1] = Acc{};
            c->slot = 0;
            c->it = 0;
            c->best = 1.0;
            c->best_at = 0;
        }
    }
    c->refine = refine + 1;
    cudaGraphSetConditional(h_outer, work);
    cudaGraphSetConditional(h_work, work);
}

// r32 = r64 / ||r||; z = M r32 (Jacobi or identity) unless an external
// preconditioner computed it; p = z; d = 0; acc[0].rz += r.z.  Arms the
// inner loop.
__global__ void __launch_bounds__(kT) k_init32(int G, const double *__restrict__ r64, const Ctl *c,
                                               const float *__restrict__ dinv, int precond, int z_given,
                                               float *__restrict__ r, float *__restrict__ z, float *__restrict__ p,
                                               float *__restrict__ d, Acc *acc, cudaGraphConditionalHandle h_inner) {
    const double s = c->inv_rnorm;
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
    if (blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h_inner, 1);
}

__global__ void __launch_bounds__(kT) k_scale32(int G, const double *__restrict__ r64, const Ctl *c,
                                                float *__restrict__ r) {
    const double s = c->inv_rnorm;
    for (int i = blockIdx.x * kT + threadIdx.x; i < G; i += gridDim.x * kT) r[i] = (float)(r64[i] * s);
}

// q = A32 p; acc[slot].pq += p.q.  First kernel of an inner iteration: it
// disarms the loop, which only the convergence check re-arms.
__global__ void __launch_bounds__(kT) k_apply32(int nx, int G, const float *__restrict__ ex,
                                                const float *__restrict__ ey, const uint8_t *__restrict__ in,
                                                const float *__restrict__ p, float *__restrict__ q, Acc *acc,
                                                const Ctl *c, cudaGraphConditionalHandle h_inner) {
    pdl_wait();
    pdl_launch();
    Acc *a = acc + c->slot;
    if (blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h_inner, 0);
    double pq = 0.0;
    for (int i = blockIdx.x * kT + threadIdx.x; i < G; i += gridDim.x * kT) {
        float v = 0.0f;
        if (in[i]) {
            v = apply_at(i, nx, ex, ey, p);
            pq += (double)p[i] * (double)v;
        }
        q[i] = v;
    }
    cta_add(pq, &a->pq);
}

// alpha = rz / pq (the exact line search along p: r.p = r.z because r is
// orthogonal to the previous direction); d += alpha p; r -= alpha q;
// acc.rr += |r|^2.  Without an external preconditioner also z = M r,
// acc.rzn += r.z, acc.zq += z.q.  A non-positive or non-finite curvature
// leaves every vector unchanged and marks rr as NaN for the check.
__global__ void __launch_bounds__(kT) k_update32(int G, const float *__restrict__ dinv, int precond,
                                                 const float *__restrict__ p, const float *__restrict__ q,
                                                 float *__restrict__ d, float *__restrict__ r,
                                                 float *__restrict__ z, Acc *acc, const Ctl *c) {
    pdl_wait();
    pdl_launch();
    Acc *a = acc + c->slot;
    const double pq = a->pq, rzv = a->rz;
    if (!(pq > 0.0) || !isfinite(rzv)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) a->rr = __longlong_as_double(0x7ff8000000000000LL);
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
        if (precond <= OEC_PRECOND_JACOBI) {
            const float zn = precond == OEC_PRECOND_JACOBI ? ri * dinv[i] : ri;
            z[i] = zn;
            rzn += (double)ri * (double)zn;
            zq += (double)zn * (double)qi;
        }
    }
    cta_add(rr, &a->rr);
    if (precond <= OEC_PRECOND_JACOBI) {
        cta_add(rzn, &a->rzn);
        cta_add(zq, &a->zq);
    }
}

// Network preconditioner: acc.rzn += r.z, acc.zq += z.q with z = M r from
// the network (z_new), copied into z.
__global__ void __launch_bounds__(kT) k_zdots32(int G, const float *__restrict__ r, const float *__restrict__ zn,
                                                const float *__restrict__ q, float *__restrict__ z, Acc *acc,
                                                const Ctl *c) {
    pdl_wait();
    pdl_launch();
    Acc *a = acc + c->slot;
    double rzn = 0.0, zq = 0.0;
    for (int i = blockIdx.x * kT + threadIdx.x; i < G; i += gridDim.x * kT) {
        const float v = zn[i];
        rzn += (double)r[i] * (double)v;
        zq += (double)v * (double)q[i];
        z[i] = v;
    }
    cta_add(rzn, &a->rzn);
    cta_add(zq, &a->zq);
}

// beta = -(z.q) / (p.q): the new direction p = z + beta p is A-conjugate to
// the previous one whatever the preconditioner (flexible CG, one stored
// direction).  One thread prepares the next slot (rz = r.z, other sums
// zero).  The last CTA to finish checks convergence: the inner residual
// against the inner tolerance, a breakdown, the iteration budget and the
// stagnation window (the best residual did not drop by 10 % in 1024
// iterations; CG residual norms are not monotone), then moves to the next
// slot and re-arms the loop when it goes on.
__global__ void __launch_bounds__(kT) k_direction32(int G, const float *__restrict__ z, float *__restrict__ p,
                                                    Acc *acc, Ctl *c, int max_iter, oec_pcg_stats_t *stats,
                                                    cudaGraphConditionalHandle h_inner) {
    pdl_wait();
    pdl_launch();
    const int slot = c->slot;
    Acc *a = acc + slot, *next = acc + (slot ^ 1);
    const double rz = a->rz;
    double b = -a->zq / a->pq;
    if (!isfinite(b)) b = 0.0;
    const float beta = (float)b;
    if (isfinite(a->rr) && isfinite(rz) && a->pq > 0.0) {
        for (int i = blockIdx.x * kT + threadIdx.x; i < G; i += gridDim.x * kT) p[i] = fmaf(beta, p[i], z[i]);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // a breakdown (rr NaN) propagates: the next update sees rz NaN
        next->rz = isfinite(a->rr) ? a->rzn : a->rr;
        next->pq = next->rr = next->rzn = next->zq = 0.0;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    __threadfence();
    if (atomicAdd(&c->ticket, 1) != (int)gridDim.x - 1) return;
    __threadfence();
    c->ticket = 0;
    const double rr = *(volatile double *)&a->rr;
    const int it = c->it + 1, total = c->total + 1;
    c->it = it;
    c->total = total;
    stats->iterations = total;
    bool more = total < max_iter;
    if (!isfinite(rr)) {
        stats->breakdown = 1;
        more = false;
    } else {
        const double rel_in = sqrt(rr);
        if (rel_in <= c->inner_tol) {
            more = false;
        } else if (rel_in < 0.9 * c->best) {
            c->best = rel_in;
            c->best_at = it;
        } else if (it - c->best_at >= 1024) {
            more = false;
        }
    }
    c->slot = slot ^ 1;
    if (more) cudaGraphSetConditional(h_inner, 1);
}

// The inner iteration's CG part when the preconditioner runs first in the
// loop body (the multigrid V-cycle: z = M r with acc.rzn += r.z and
// acc.zq += z.q of the previous direction's q): the new direction
// p = z + beta p (beta = -(z.q)/(p.q), flexible CG; p = z in the first
// iteration), q = A p with p.q, the step alpha = (r.z)/(p.q) into d and r
// with |r|^2, and the convergence check of k_direction32 -- one cooperative
// launch with grid-wide barriers between the parts instead of three launches
// (all CTAs resident).  A non-positive or non-finite curvature leaves d and r
// unchanged and ends the loop as a breakdown.
__global__ void __launch_bounds__(kT) k_cg_step(int nx, int G, const float *__restrict__ ex,
                                                const float *__restrict__ ey, const uint8_t *__restrict__ in,
                                                const float *__restrict__ z, float *__restrict__ p,
                                                float *__restrict__ q, float *__restrict__ d, float *__restrict__ r,
                                                Acc *acc, Ctl *c, int max_iter, oec_pcg_stats_t *stats,
                                                cudaGraphConditionalHandle h_inner) {
    cooperative_groups::grid_group grid = cooperative_groups::this_grid();
    Acc *a = acc + c->slot;
    const int it = c->it;
    if (blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h_inner, 0);
    float beta = 0.f;
    if (it > 0) {
        double b = -a->zq / c->pq_prev;
        beta = isfinite(b) ? (float)b : 0.f;
    }
    const int stride = gridDim.x * kT;
    for (int i = blockIdx.x * kT + threadIdx.x; i < G; i += stride) p[i] = it > 0 ? fmaf(beta, p[i], z[i]) : z[i];
    grid.sync();
    double pq = 0.0;
    for (int i = blockIdx.x * kT + threadIdx.x; i < G; i += stride) {
        float v = 0.0f;
        if (in[i]) {
            v = apply_at(i, nx, ex, ey, p);
            pq += (double)p[i] * (double)v;
        }
        q[i] = v;
    }
    cta_add(pq, &a->pq);
    grid.sync();
    const double pqs = a->pq, rz = a->rzn;
    double rr = 0.0;
    if (pqs > 0.0 && isfinite(rz)) {
        const float alpha = (float)(rz / pqs);
        for (int i = blockIdx.x * kT + threadIdx.x; i < G; i += stride) {
            d[i] = fmaf(alpha, p[i], d[i]);
            const float ri = fmaf(-alpha, q[i], r[i]);
            r[i] = ri;
            rr += (double)ri * (double)ri;
        }
        cta_add(rr, &a->rr);
    } else if (blockIdx.x == 0 && threadIdx.x == 0) {
        a->rr = __longlong_as_double(0x7ff8000000000000LL);
    }
    grid.sync();
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const double rrs = a->rr;
    const int it1 = it + 1, total = c->total + 1;
    c->it = it1;
    c->total = total;
    stats->iterations = total;
    bool more = total < max_iter;
    if (!isfinite(rrs)) {
        stats->breakdown = 1;
        more = false;
    } else {
        const double rel_in = sqrt(rrs);
        if (rel_in <= c->inner_tol) {
            more = false;
        } else if (rel_in < 0.9 * c->best) {
            c->best = rel_in;
            c->best_at = it1;
        } else if (it1 - c->best_at >= 1024) {
            more = false;
        }
    }
    // the next V-cycle accumulates its dot products from zero
    c->pq_prev = pqs;
    a->pq = a->rr = a->rzn = a->zq = 0.0;
    if (more) cudaGraphSetConditional(h_inner, 1);
}

// Start of the inner loop of k_cg_step: d = 0, q = 0, arms the loop (r was
// scaled by k_scale32).
__global__ void __launch_bounds__(kT) k_init_cg(int G, float *__restrict__ d, float *__restrict__ q,
                                                cudaGraphConditionalHandle h_inner) {
    for (int i = blockIdx.x * kT + threadIdx.x; i < G; i += gridDim.x * kT) {
        d[i] = 0.0f;
        q[i] = 0.0f;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h_inner, 1);
}

// phi += coef d on the inside nodes.
__global__ void __launch_bounds__(kT) k_accumulate64(int G, const Ctl *c, const float *__restrict__ d,
                                                     const uint8_t *__restrict__ in, double *__restrict__ phi) {
    const double coef = c->coef;
    for (int i = blockIdx.x * kT + threadIdx.x; i < G; i += gridDim.x * kT)
        phi[i] = in[i] ? fma(coef, (double)d[i], phi[i]) : 0.0;
}

// LU fallback switch (one thread): runs the fallback when the solve missed
// tol and counts it.
__global__ void k_fallback_flag(const oec_pcg_stats_t *stats, int *count, cudaGraphConditionalHandle h) {
    if (threadIdx.x != 0) return;
    const int fb = stats->converged ? 0 : 1;
    if (fb && count) *count += 1;
    cudaGraphSetConditional(h, fb);
}

// ------------------------------------------------------------ multigrid
// Aggregation V-cycle (oec_mg_t).  Node i = row * nx + col on every level;
// a node is inside exactly when its 1/diagonal is nonzero (the operator's
// diagonal is positive on inside nodes).  Levels above the block level run
// as two tiled kernels each (down: two sweeps and the restricted residual;
// up: prolongation and two sweeps), every CTA computing a 32 x 16 tile of
// fine nodes with a halo of two nodes in shared memory, so no intermediate
// vector but the pre-smoothed x leaves the CTA.  The block level and all
// coarser ones run in one CTA with every level in shared memory.
constexpr int kTX = 32, kTY = 16;       // fine tile
constexpr int kBlockThreads = 1024;
constexpr int kMgMaxBlockLevels = 8;
constexpr int kMgFloatsPerNode = 7;     // ex, ey, leak, dinv, b, x, y
constexpr int kMgFloatsPerNodeLean = 3; // b, x, y (the operator read from global memory)
constexpr int kMgMaxCoarse = 1024;
constexpr size_t kMgMaxBlockSmem = 226 * 1024;  // dynamic, beside the level table

struct MgT {
    int nx, ny;
    const float *ex, *ey, *leak, *dinv;
};

// (A v) at fine node (gx, gy), i = gy * nx + gx, from a shared tile s with
// row stride S whose entry (sy, sx) holds node (gx, gy): leak v_i + sum over
// the 4 edges of w (v_i - v_j).  Nodes beyond the grid hold 0 in s.
template <int S>
__device__ __forceinline__ float tile_apply(const MgT &L, int i, int gx, int gy, const float *s, int sy, int sx) {
    const float c = s[sy * S + sx];
    float y = L.leak ? L.leak[i] * c : 0.f;
    y += L.ex[i] * (c - s[sy * S + sx + 1]);
    if (gx > 0) y += L.ex[i - 1] * (c - s[sy * S + sx - 1]);
    y += L.ey[i] * (c - s[(sy + 1) * S + sx]);
    if (gy > 0) y += L.ey[i - L.nx] * (c - s[(sy - 1) * S + sx]);
    return y;
}

// One damped-Jacobi sweep on the tile grown by `grow` (1 or 0) from the
// values in `src` (tile grown by grow + 1): dst = v + w D^-1 (b - A v).
template <int SS, int DS, int GROW>
__device__ __forceinline__ void tile_sweep(const MgT &L, float om, const float *__restrict__ b, int x0, int y0,
                                           const float *src, float *dst) {
    constexpr int W = kTX + 2 * GROW, H = kTY + 2 * GROW;
    for (int e = threadIdx.x; e < W * H; e += blockDim.x) {
        const int ly = e / W, lx = e - ly * W;
        const int gx = x0 + lx - GROW, gy = y0 + ly - GROW;
        float v = 0.f;
        if (gx >= 0 && gy >= 0 && gx < L.nx && gy < L.ny) {
            const int i = gy * L.nx + gx;
            const float d = L.dinv[i];
            if (d != 0.f) {
                const float c = src[(ly + 1) * SS + lx + 1];
                v = c + om * d * (b[i] - tile_apply<SS>(L, i, gx, gy, src, ly + 1, lx + 1));
            }
        }
        dst[ly * DS + lx] = v;
    }
}

// Down: x1 = w D^-1 b, x = x1 + w D^-1 (b - A x1) (written to x), and the
// coarse right-hand side bc[I] = sum over the inside children of (b - A x).
// Node (r, c) belongs to coarse node (r >> SY, c >> SX).
template <int SX, int SY>
__global__ void __launch_bounds__(kT) k_mg_down(MgT L, float om, const float *__restrict__ b, float *__restrict__ x,
                                                float *__restrict__ bc, int cnx, int cny) {
    pdl_wait();
    pdl_launch();
    __shared__ float s1[(kTY + 4) * (kTX + 4)];
    __shared__ float s2[(kTY + 2) * (kTX + 2)];
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
    for (int e = threadIdx.x; e < (kTY + 4) * (kTX + 4); e += kT) {
        const int ly = e / (kTX + 4), lx = e - ly * (kTX + 4);
        const int gx = x0 + lx - 2, gy = y0 + ly - 2;
        float v = 0.f;
        if (gx >= 0 && gy >= 0 && gx < L.nx && gy < L.ny) {
            const int i = gy * L.nx + gx;
            v = om * L.dinv[i] * b[i];
        }
        s1[e] = v;
    }
    __syncthreads();
    tile_sweep<kTX + 4, kTX + 2, 1>(L, om, b, x0, y0, s1, s2);
    __syncthreads();
    float *res = s1;  // [kTY][kTX]
    for (int e = threadIdx.x; e < kTY * kTX; e += kT) {
        const int ly = e / kTX, lx = e - ly * kTX;
        const int gx = x0 + lx, gy = y0 + ly;
        float v = 0.f;
        if (gx < L.nx && gy < L.ny) {
            const int i = gy * L.nx + gx;
            x[i] = s2[(ly + 1) * (kTX + 2) + lx + 1];
            if (L.dinv[i] != 0.f) v = b[i] - tile_apply<kTX + 2>(L, i, gx, gy, s2, ly + 1, lx + 1);
        }
        res[e] = v;
    }
    __syncthreads();
    constexpr int CW = kTX >> SX, CH = kTY >> SY;
    for (int e = threadIdx.x; e < CW * CH; e += kT) {
        const int cy = e / CW, cx = e - cy * CW;
        const int X = (x0 >> SX) + cx, Y = (y0 >> SY) + cy;
        if (X < cnx && Y < cny) {
            const float *r = res + (cy << SY) * kTX + (cx << SX);
            float v = r[0];
            if (SX) v += r[1];
            if (SY) v += SX ? r[kTX] + r[kTX + 1] : r[kTX];
            bc[Y * cnx + X] = v;
        }
    }
}

// Up: t = x + scale * yc[parent] (inside nodes), two sweeps, result to out.
// With acc, also acc[slot].rzn += b.out and acc[slot].zq += out.q (b is the
// level-0 residual r, out the preconditioned z).
template <int SX, int SY>
__global__ void __launch_bounds__(kT) k_mg_up(MgT L, float om, float scale, const float *__restrict__ b,
                                              const float *__restrict__ x, const float *__restrict__ yc, int cnx,
                                              float *__restrict__ out, const float *__restrict__ q, Acc *acc,
                                              const Ctl *ctl) {
    pdl_wait();
    pdl_launch();
    __shared__ float s1[(kTY + 4) * (kTX + 4)];
    __shared__ float s2[(kTY + 2) * (kTX + 2)];
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
    for (int e = threadIdx.x; e < (kTY + 4) * (kTX + 4); e += kT) {
        const int ly = e / (kTX + 4), lx = e - ly * (kTX + 4);
        const int gx = x0 + lx - 2, gy = y0 + ly - 2;
        float v = 0.f;
        if (gx >= 0 && gy >= 0 && gx < L.nx && gy < L.ny) {
            const int i = gy * L.nx + gx;
            if (L.dinv[i] != 0.f) v = x[i] + scale * yc[(gy >> SY) * cnx + (gx >> SX)];
        }
        s1[e] = v;
    }
    __syncthreads();
    tile_sweep<kTX + 4, kTX + 2, 1>(L, om, b, x0, y0, s1, s2);
    __syncthreads();
    double rz = 0.0, zq = 0.0;
    for (int e = threadIdx.x; e < kTY * kTX; e += kT) {
        const int ly = e / kTX, lx = e - ly * kTX;
        const int gx = x0 + lx, gy = y0 + ly;
        if (gx < L.nx && gy < L.ny) {
            const int i = gy * L.nx + gx;
            const float d = L.dinv[i];
            float v = 0.f;
            if (d != 0.f) {
                const float c = s2[(ly + 1) * (kTX + 2) + lx + 1];
                v = c + om * d * (b[i] - tile_apply<kTX + 2>(L, i, gx, gy, s2, ly + 1, lx + 1));
            }
            out[i] = v;
            if (acc) {
                rz += (double)b[i] * (double)v;
                zq += (double)v * (double)q[i];
            }
        }
    }
    if (acc) {
        Acc *a = acc + ctl->slot;
        cta_add(rz, &a->rzn);
        cta_add(zq, &a->zq);
    }
}

// Levels from the block level down, solved by one CTA (oec_mg_t levels
// block_level .. nlevels-1; the last one by its dense inverse).
struct MgBlock {
    int nb, m;
    int nx[kMgMaxBlockLevels], ny[kMgMaxBlockLevels];
    const float *ex[kMgMaxBlockLevels], *ey[kMgMaxBlockLevels], *leak[kMgMaxBlockLevels], *dinv[kMgMaxBlockLevels];
    const int32_t *idx;
    const float *inv;
    float om, scale;
};

struct SmLevel {
    int nx, ny, n;
    float *ex, *ey, *lk, *dv, *b, *x, *y;
};

__device__ __forceinline__ float sm_apply(const SmLevel &L, int i, const float *v) {
    const int r = i / L.nx, c = i - r * L.nx;
    const float vi = v[i];
    float y = L.lk[i] * vi;
    if (c + 1 < L.nx) y += L.ex[i] * (vi - v[i + 1]);
    if (c > 0) y += L.ex[i - 1] * (vi - v[i - 1]);
    if (r + 1 < L.ny) y += L.ey[i] * (vi - v[i + L.nx]);
    if (r > 0) y += L.ey[i - L.nx] * (vi - v[i - L.nx]);
    return y;
}

// dst = src + w D^-1 (b - A src) on the inside nodes, 0 outside.
__device__ __forceinline__ void sm_sweep(const SmLevel &L, float om, const float *src, float *dst) {
    for (int i = threadIdx.x; i < L.n; i += kBlockThreads) {
        const float d = L.dv[i];
        dst[i] = d != 0.f ? src[i] + om * d * (L.b[i] - sm_apply(L, i, src)) : 0.f;
    }
}

// coef_smem: the levels' operator is copied to shared memory (7 floats per
// node); otherwise it is read from its global arrays (3 floats per node in
// shared memory: b, x, y), which lets larger levels into this kernel.
__global__ void __launch_bounds__(kBlockThreads) k_mg_block(MgBlock P, const float *__restrict__ b_in,
                                                            float *__restrict__ y_out, int coef_smem) {
    pdl_wait();
    pdl_launch();
    extern __shared__ float sm[];
    __shared__ SmLevel Ls[kMgMaxBlockLevels];
    if (threadIdx.x == 0) {
        float *p = sm;
        for (int l = 0; l < P.nb; ++l) {
            SmLevel &L = Ls[l];
            L.nx = P.nx[l];
            L.ny = P.ny[l];
            L.n = L.nx * L.ny;
            if (coef_smem) {
                float **a[] = {&L.ex, &L.ey, &L.lk, &L.dv};
                for (float **q : a) {
                    *q = p;
                    p += L.n;
                }
            } else {
                L.ex = const_cast<float *>(P.ex[l]);
                L.ey = const_cast<float *>(P.ey[l]);
                L.lk = const_cast<float *>(P.leak[l]);
                L.dv = const_cast<float *>(P.dinv[l]);
            }
            float **a[] = {&L.b, &L.x, &L.y};
            for (float **q : a) {
                *q = p;
                p += L.n;
            }
        }
    }
    __syncthreads();
    for (int l = 0; l < P.nb; ++l) {
        const SmLevel &L = Ls[l];
        for (int i = threadIdx.x; i < L.n; i += kBlockThreads) {
            if (coef_smem) {
                L.ex[i] = P.ex[l][i];
                L.ey[i] = P.ey[l][i];
                L.lk[i] = P.leak[l][i];
                L.dv[i] = P.dinv[l][i];
            }
            L.b[i] = l == 0 ? b_in[i] : 0.f;
            L.x[i] = 0.f;
            L.y[i] = 0.f;
        }
    }
    __syncthreads();
    const float om = P.om;
    for (int l = 0; l + 1 < P.nb; ++l) {
        const SmLevel &L = Ls[l], &C = Ls[l + 1];
        const int sx = C.nx != L.nx, sy = C.ny != L.ny;
        for (int i = threadIdx.x; i < L.n; i += kBlockThreads) L.y[i] = om * L.dv[i] * L.b[i];
        __syncthreads();
        sm_sweep(L, om, L.y, L.x);
        __syncthreads();
        for (int I = threadIdx.x; I < C.n; I += kBlockThreads) {
            const int R = I / C.nx, Cc = I - R * C.nx;
            float s = 0.f;
#pragma unroll
            for (int d = 0; d < 4; ++d) {
                const int r = (R << sy) + (d >> 1), c = (Cc << sx) + (d & 1);
                if ((d >> 1) <= sy && (d & 1) <= sx && r < L.ny && c < L.nx) {
                    const int i = r * L.nx + c;
                    if (L.dv[i] != 0.f) s += L.b[i] - sm_apply(L, i, L.x);
                }
            }
            C.b[I] = s;
        }
        __syncthreads();
    }
    {  // bottom: y[idx[r]] = sum_c inv[r][c] b[idx[c]], one warp per row
        const SmLevel &B = Ls[P.nb - 1];
        const int lane = threadIdx.x & 31;
        for (int r = threadIdx.x >> 5; r < P.m; r += kBlockThreads / 32) {
            const float *row = P.inv + (size_t)r * P.m;
            float s = 0.f;
            for (int c = lane; c < P.m; c += 32) s = fmaf(row[c], B.b[P.idx[c]], s);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFullMask, s, o);
            if (lane == 0) B.y[P.idx[r]] = s;
        }
        __syncthreads();
    }
    for (int l = P.nb - 2; l >= 0; --l) {
        const SmLevel &L = Ls[l], &C = Ls[l + 1];
        const int sx = C.nx != L.nx, sy = C.ny != L.ny;
        for (int i = threadIdx.x; i < L.n; i += kBlockThreads) {
            const int r = i / L.nx, c = i - r * L.nx;
            L.y[i] = L.dv[i] != 0.f ? L.x[i] + P.scale * C.y[(r >> sy) * C.nx + (c >> sx)] : 0.f;
        }
        __syncthreads();
        sm_sweep(L, om, L.y, L.x);
        __syncthreads();
        sm_sweep(L, om, L.x, L.y);
        __syncthreads();
    }
    const SmLevel &T = Ls[0];
    for (int i = threadIdx.x; i < T.n; i += kBlockThreads) y_out[i] = T.y[i];
}

// ------------------------------------------------ one-cluster coarse levels
//
// The levels from the cluster level down, solved by one thread-block cluster
// of up to 16 CTAs (oec_mg_t.cluster_top): each level's rows are dealt out
// in bands of `rows` consecutive rows per CTA, and a CTA keeps its bands of
// b, x and y in its shared memory; the rows beyond a band (stencil
// neighbours, aggregation children and parents) are read from the other
// CTAs' shared memory through the cluster's distributed shared memory.  The
// phases of the V-cycle are separated by cluster barriers instead of kernel
// launches.  The arithmetic of every node is the one-CTA kernel's
// (k_mg_block), in the same order.

constexpr int kClusterMax = 16;
constexpr int kClusterLevels = 12;
constexpr int kClusterThreads = 1024;

struct MgCluster {
    int nl;       // levels, top (the cluster level) to bottom
    int ncta;     // CTAs of the cluster
    int m;        // inside nodes of the bottom level
    int nx[kClusterLevels], ny[kClusterLevels];
    int rows[kClusterLevels];  // rows of a band: ceil(ny / ncta)
    int off[kClusterLevels];   // float offset of the level's b band; x, y follow at +span, +2 span
    const float *ex[kClusterLevels], *ey[kClusterLevels], *leak[kClusterLevels], *dinv[kClusterLevels];
    const int32_t *idx;
    const float *inv;
    float om, scale;
    const float *b_top;  // right-hand side of the top level (global)
    float *out;          // result of the top level (global)
    const float *q;      // with acc: CG dots r.z and z.q of the top level
    Acc *acc;
    const Ctl *ctl;
};

size_t mg_cluster_floats(const MgCluster &P) {
    size_t n = 0;
    for (int l = 0; l < P.nl; ++l) n += 3 * (size_t)P.rows[l] * P.nx[l];
    return n;
}

struct ClLevel {
    int nx, ny, R, off;
    const float *ex, *ey, *lk, *dv;
};

// Pointer to node (r, 0) of array a (0 b, 1 x, 2 y) of level L, in the CTA
// that owns row r.
__device__ __forceinline__ float *cl_row(float *const *base, const ClLevel &L, int a, int r) {
    const int o = r / L.R;
    return base[o] + L.off + a * L.R * L.nx + (r - o * L.R) * L.nx;
}

// (A v)_i at node (r, c) of level L, the rows r-1, r, r+1 of v given.
__device__ __forceinline__ float cl_apply(const ClLevel &L, int i, int r, int c, const float *vm, const float *v0,
                                          const float *vp) {
    const float vi = v0[c];
    float y = L.lk[i] * vi;
    if (c + 1 < L.nx) y += L.ex[i] * (vi - v0[c + 1]);
    if (c > 0) y += L.ex[i - 1] * (vi - v0[c - 1]);
    if (r + 1 < L.ny) y += L.ey[i] * (vi - vp[c]);
    if (r > 0) y += L.ey[i - L.nx] * (vi - vm[c]);
    return y;
}

__device__ __forceinline__ void cl_sync() { cooperative_groups::this_cluster().sync(); }

__device__ __forceinline__ double cl_block_sum(double v, double *sh) {
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    double s = 0.0;
    if (w == 0) {
        s = l < kClusterThreads / 32 ? sh[l] : 0.0;
        s = warp_sum(s);
    }
    __syncthreads();
    return s;
}

__global__ void __launch_bounds__(kClusterThreads, 1) k_mg_cluster(MgCluster P) {
    pdl_wait();
    pdl_launch();
    extern __shared__ __align__(16) float smc[];
    __shared__ float *base[kClusterMax];
    __shared__ ClLevel Ls[kClusterLevels];
    __shared__ double red[kClusterThreads / 32];
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const unsigned me = cluster.block_rank();
    if (threadIdx.x < P.ncta) base[threadIdx.x] = cluster.map_shared_rank(smc, threadIdx.x);
    if (threadIdx.x < P.nl) {
        const int l = threadIdx.x;
        Ls[l] = ClLevel{P.nx[l], P.ny[l], P.rows[l], P.off[l], P.ex[l], P.ey[l], P.leak[l], P.dinv[l]};
    }
    __syncthreads();
    const float om = P.om;
    // own band of level L: rows [r0, r1), nodes [r0*nx, r1*nx)
    auto band = [&](const ClLevel &L, int &r0, int &r1) {
        r0 = min((int)me * L.R, L.ny);
        r1 = min(r0 + L.R, L.ny);
    };
    {  // top right-hand side into the band; bottom result cleared
        const ClLevel &T = Ls[0];
        int r0, r1;
        band(T, r0, r1);
        float *b = smc + T.off;
        for (int e = threadIdx.x; e < (r1 - r0) * T.nx; e += kClusterThreads) b[e] = P.b_top[r0 * T.nx + e];
        const ClLevel &B = Ls[P.nl - 1];
        band(B, r0, r1);
        float *y = smc + B.off + 2 * B.R * B.nx;
        for (int e = threadIdx.x; e < (r1 - r0) * B.nx; e += kClusterThreads) y[e] = 0.f;
    }
    cl_sync();
    // ---- down
    for (int l = 0; l + 1 < P.nl; ++l) {
        const ClLevel &L = Ls[l], &C = Ls[l + 1];
        const int sx = C.nx != L.nx, sy = C.ny != L.ny;
        int r0, r1;
        band(L, r0, r1);
        // x = y0 + w D^-1 (b - A y0), y0 = w D^-1 b (formed on the fly from b)
        for (int e = threadIdx.x; e < (r1 - r0) * L.nx; e += kClusterThreads) {
            const int lr = e / L.nx, c = e - lr * L.nx, r = r0 + lr, i = r * L.nx + c;
            float *x = smc + L.off + L.R * L.nx + lr * L.nx;
            const float d = L.dv[i];
            if (d == 0.f) {
                x[c] = 0.f;
                continue;
            }
            const float *b0 = cl_row(base, L, 0, r);
            const float *bm = r > 0 ? cl_row(base, L, 0, r - 1) : b0;
            const float *bp = r + 1 < L.ny ? cl_row(base, L, 0, r + 1) : b0;
            const float yi = om * d * b0[c];
            float ax = L.lk[i] * yi;
            if (c + 1 < L.nx) ax += L.ex[i] * (yi - om * L.dv[i + 1] * b0[c + 1]);
            if (c > 0) ax += L.ex[i - 1] * (yi - om * L.dv[i - 1] * b0[c - 1]);
            if (r + 1 < L.ny) ax += L.ey[i] * (yi - om * L.dv[i + L.nx] * bp[c]);
            if (r > 0) ax += L.ey[i - L.nx] * (yi - om * L.dv[i - L.nx] * bm[c]);
            x[c] = yi + om * d * (b0[c] - ax);
        }
        cl_sync();
        // coarse right-hand side: sum over the inside children of b - A x
        int R0, R1;
        band(C, R0, R1);
        for (int e = threadIdx.x; e < (R1 - R0) * C.nx; e += kClusterThreads) {
            const int lr = e / C.nx, Cc = e - lr * C.nx, R = R0 + lr;
            float s = 0.f;
#pragma unroll
            for (int dd = 0; dd < 4; ++dd) {
                const int r = (R << sy) + (dd >> 1), c = (Cc << sx) + (dd & 1);
                if ((dd >> 1) <= sy && (dd & 1) <= sx && r < L.ny && c < L.nx) {
                    const int i = r * L.nx + c;
                    if (L.dv[i] != 0.f) {
                        const float *x0 = cl_row(base, L, 1, r);
                        const float *xm = r > 0 ? cl_row(base, L, 1, r - 1) : x0;
                        const float *xp = r + 1 < L.ny ? cl_row(base, L, 1, r + 1) : x0;
                        s += cl_row(base, L, 0, r)[c] - cl_apply(L, i, r, c, xm, x0, xp);
                    }
                }
            }
            smc[C.off + lr * C.nx + Cc] = s;
        }
        cl_sync();
    }
    {  // bottom: y[idx[r]] = sum_c inv[r][c] b[idx[c]], one warp per row
        const ClLevel &B = Ls[P.nl - 1];
        const int lane = threadIdx.x & 31;
        const int warps = P.ncta * (kClusterThreads / 32);
        for (int r = (int)me * (kClusterThreads / 32) + (threadIdx.x >> 5); r < P.m; r += warps) {
            const float *row = P.inv + (size_t)r * P.m;
            float s = 0.f;
            for (int c = lane; c < P.m; c += 32) {
                const int j = P.idx[c], jr = j / B.nx;
                s = fmaf(row[c], cl_row(base, B, 0, jr)[j - jr * B.nx], s);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFullMask, s, o);
            if (lane == 0) {
                const int j = P.idx[r], jr = j / B.nx;
                cl_row(base, B, 2, jr)[j - jr * B.nx] = s;
            }
        }
        cl_sync();
    }
    // ---- up
    for (int l = P.nl - 2; l >= 0; --l) {
        const ClLevel &L = Ls[l], &C = Ls[l + 1];
        const int sx = C.nx != L.nx, sy = C.ny != L.ny;
        int r0, r1;
        band(L, r0, r1);
        const int n = (r1 - r0) * L.nx;
        float *bb = smc + L.off, *xx = bb + L.R * L.nx, *yy = xx + L.R * L.nx;
        // y = x + scale * (coarse result at the parent) on the inside nodes
        for (int e = threadIdx.x; e < n; e += kClusterThreads) {
            const int lr = e / L.nx, c = e - lr * L.nx, r = r0 + lr, i = r * L.nx + c;
            const int pr = r >> sy;
            yy[e] = L.dv[i] != 0.f ? xx[e] + P.scale * cl_row(base, C, 2, pr)[c >> sx] : 0.f;
        }
        cl_sync();
        // two sweeps: y -> x -> y
        for (int sweep = 0; sweep < 2; ++sweep) {
            const int src = sweep == 0 ? 2 : 1;
            float *dst = sweep == 0 ? xx : yy;
            const bool last = sweep == 1 && l == 0;
            double rz = 0.0, zq = 0.0;
            for (int e = threadIdx.x; e < n; e += kClusterThreads) {
                const int lr = e / L.nx, c = e - lr * L.nx, r = r0 + lr, i = r * L.nx + c;
                const float d = L.dv[i];
                float v = 0.f;
                if (d != 0.f) {
                    const float *v0 = cl_row(base, L, src, r);
                    const float *vm = r > 0 ? cl_row(base, L, src, r - 1) : v0;
                    const float *vp = r + 1 < L.ny ? cl_row(base, L, src, r + 1) : v0;
                    v = v0[c] + om * d * (bb[e] - cl_apply(L, i, r, c, vm, v0, vp));
                }
                if (last) {
                    P.out[i] = v;
                    if (P.acc) {
                        rz += (double)bb[e] * (double)v;
                        zq += (double)v * (double)P.q[i];
                    }
                } else {
                    dst[e] = v;
                }
            }
            if (last && P.acc) {
                Acc *a = P.acc + P.ctl->slot;
                rz = cl_block_sum(rz, red);
                zq = cl_block_sum(zq, red);
                if (threadIdx.x == 0) {
                    if (rz != 0.0) atomicAdd(&a->rzn, rz);
                    if (zq != 0.0) atomicAdd(&a->zq, zq);
                }
            }
            cl_sync();
        }
    }
    if (P.nl == 1) {  // the top level is the bottom: its result to out
        const ClLevel &B = Ls[0];
        int r0, r1;
        band(B, r0, r1);
        const float *y = smc + B.off + 2 * B.R * B.nx;
        double rz = 0.0, zq = 0.0;
        for (int e = threadIdx.x; e < (r1 - r0) * B.nx; e += kClusterThreads) {
            const int i = r0 * B.nx + e;
            P.out[i] = y[e];
            if (P.acc) {
                rz += (double)smc[B.off + e] * (double)y[e];
                zq += (double)y[e] * (double)P.q[i];
            }
        }
        if (P.acc) {
            Acc *a = P.acc + P.ctl->slot;
            rz = cl_block_sum(rz, red);
            zq = cl_block_sum(zq, red);
            if (threadIdx.x == 0) {
                if (rz != 0.0) atomicAdd(&a->rzn, rz);
                if (zq != 0.0) atomicAdd(&a->zq, zq);
            }
        }
        cl_sync();
    }
}

// acc[slot].rzn += r.z, acc[slot].zq += z.q (used when the block kernel
// writes z itself).
__global__ void __launch_bounds__(kT) k_dots32(int G, const float *__restrict__ r, const float *__restrict__ z,
                                               const float *__restrict__ q, Acc *acc, const Ctl *ctl) {
    pdl_wait();
    pdl_launch();
    acc += ctl->slot;
    double rzn = 0.0, zq = 0.0;
    for (int i = blockIdx.x * kT + threadIdx.x; i < G; i += gridDim.x * kT) {
        const float a = z[i];
        rzn += (double)r[i] * (double)a;
        zq += (double)a * (double)q[i];
    }
    cta_add(rzn, &acc->rzn);
    cta_add(zq, &acc->zq);
}

// Aggregation of level l into c: bit 0 set when columns pair up, bit 1 when
// rows do (a direction of size 1 counts as paired).
int mg_shift(const oec_mg_level_t &l, const oec_mg_level_t &c) {
    return (c.nx != l.nx || l.nx == 1 ? 1 : 0) | (c.ny != l.ny || l.ny == 1 ? 2 : 0);
}

MgT mg_t(const oec_mg_level_t &l, bool with_leak) { return MgT{l.nx, l.ny, l.ex, l.ey, with_leak ? l.leak : nullptr, l.dinv}; }

size_t mg_block_nodes(const oec_mg_t *mg) {
    size_t n = 0;
    for (int k = mg->block_level; k < mg->nlevels; ++k) n += (size_t)mg->levels[k].nx * mg->levels[k].ny;
    return n;
}

// Whether the one-CTA levels keep their operator (edge weights, leak,
// inverse diagonal) in shared memory too, or read it from global memory
// (L1/L2) so that larger levels fit.
bool mg_block_coef_smem(const oec_mg_t *mg) {
    return mg_block_nodes(mg) * kMgFloatsPerNode * sizeof(float) <= kMgMaxBlockSmem;
}

size_t mg_block_smem(const oec_mg_t *mg) {
    return mg_block_nodes(mg) * (mg_block_coef_smem(mg) ? kMgFloatsPerNode : kMgFloatsPerNodeLean) * sizeof(float);
}

bool valid_mg(const oec_mg_t *mg) {
    if (!mg || mg->nlevels < 1 || mg->nlevels > 16 || !mg->levels || mg->ncoarse < 1 ||
        mg->ncoarse > kMgMaxCoarse || !mg->coarse_idx || !mg->coarse_inv)
        return false;
    if (mg->block_level < 0 || mg->block_level >= mg->nlevels || mg->nlevels - mg->block_level > kMgMaxBlockLevels)
        return false;
    for (int k = 0; k < mg->nlevels; ++k) {
        const oec_mg_level_t &l = mg->levels[k];
        if (l.nx < 1 || l.ny < 1 || (int64_t)l.nx * l.ny >= (1 << 28) || !l.ex || !l.ey || !l.leak || !l.dinv ||
            !l.b || !l.x || !l.y)
            return false;
        if (k > 0) {  // each direction halves (rounded up) or keeps its size; the level shrinks
            const oec_mg_level_t &f = mg->levels[k - 1];
            if ((l.nx != (f.nx + 1) / 2 && l.nx != f.nx) || (l.ny != (f.ny + 1) / 2 && l.ny != f.ny) ||
                (int64_t)l.nx * l.ny >= (int64_t)f.nx * f.ny)
                return false;
        }
    }
    const oec_mg_level_t &bot = mg->levels[mg->nlevels - 1];
    if (mg->ncoarse > bot.nx * bot.ny) return false;
    return mg_block_smem(mg) <= kMgMaxBlockSmem;
}

// The cluster size used for the one-cluster levels on this device: 16 CTAs
// when a cluster of 16 with the largest shared-memory size can be resident,
// else 8 (portable); 0 when clusters cannot run.
int mg_cluster_ctas() {
    static std::atomic<int> cached[kMaxDevices];
    return per_device_cached(cached, [] {
        constexpr int smem = (int)kMgMaxBlockSmem;
        if (cudaFuncSetAttribute(k_mg_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
            return -1;
        for (int n : {16, 8}) {
            if (n > 8 && cudaFuncSetAttribute(k_mg_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                             cudaSuccess)
                continue;
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(n);
            cfg.blockDim = dim3(kClusterThreads);
            cfg.dynamicSmemBytes = smem;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = n;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            int clusters = 0;
            if (cudaOccupancyMaxActiveClusters(&clusters, k_mg_cluster, &cfg) == cudaSuccess && clusters >= 1)
                return n;
        }
        cudaGetLastError();
        return -1;
    });
}

// First level of the one-cluster solve: the first of at most
// mg->cluster_top nodes, no lower than the block level.
int mg_cluster_top_level(const oec_mg_t *mg) {
    for (int k = 0; k < mg->block_level; ++k)
        if ((int64_t)mg->levels[k].nx * mg->levels[k].ny <= mg->cluster_top) return k;
    return mg->block_level;
}

// The plan of the one-cluster levels (top level to the bottom): bands and
// shared-memory offsets.  False when the cluster path is off or does not
// fit; the one-CTA block path is used instead.
bool mg_cluster_plan(const oec_mg_t *mg, MgCluster &P) {
    if (mg->cluster_top <= 0) return false;
    const int ncta = mg_cluster_ctas();
    if (ncta <= 0) return false;
    const int top = mg_cluster_top_level(mg);
    if (mg->nlevels - top > kClusterLevels) return false;
    P = MgCluster{};
    P.nl = mg->nlevels - top;
    P.ncta = ncta;
    P.m = mg->ncoarse;
    int off = 0;
    for (int j = 0; j < P.nl; ++j) {
        const oec_mg_level_t &l = mg->levels[top + j];
        P.nx[j] = l.nx;
        P.ny[j] = l.ny;
        P.rows[j] = (l.ny + ncta - 1) / ncta;
        P.off[j] = off;
        off += 3 * P.rows[j] * l.nx;
        P.ex[j] = l.ex;
        P.ey[j] = l.ey;
        P.leak[j] = l.leak;
        P.dinv[j] = l.dinv;
    }
    if ((size_t)off * sizeof(float) > kMgMaxBlockSmem) return false;
    P.idx = mg->coarse_idx;
    P.inv = mg->coarse_inv;
    P.om = mg->omega;
    P.scale = mg->scale;
    return true;
}

int launch_mg_cluster(const MgCluster &P, cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(P.ncta);
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = mg_cluster_floats(P) * sizeof(float);
    cfg.stream = s;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = P.ncta;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl_enabled() ? 2 : 1;
    OEC_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_mg_cluster, P));
    return OEC_OK;
}

// One V-cycle z = M r; with acc, also the flexible-CG dot products r.z and
// z.q into acc[ctl->slot] (q the operator image of the current direction).
// Levels above the coarse solve run as tiled kernels over the whole GPU; the
// coarse levels run in one cluster (mg->cluster_top) or one CTA.
int mg_cycle(const oec_mg_t *mg, const float *r, float *z, const float *q, Acc *acc, const Ctl *ctl,
             cudaStream_t s) {
    const int L = mg->nlevels;
    MgCluster C;
    const bool clustered = mg_cluster_plan(mg, C);
    const int B = clustered ? mg_cluster_top_level(mg) : mg->block_level;
    const oec_mg_level_t *lv = mg->levels;
    for (int k = 0; k < B; ++k) {
        const oec_mg_level_t &l = lv[k], &c = lv[k + 1];
        const dim3 grid((l.nx + kTX - 1) / kTX, (l.ny + kTY - 1) / kTY);
        const MgT m = mg_t(l, k > 0);
        const float *b = k == 0 ? r : l.b;
        switch (mg_shift(l, c)) {
            case 3: OEC_CUDA_TRY(launch_overlapped(k_mg_down<1, 1>, grid, dim3(kT), 0, s, m, mg->omega, b, l.x, c.b, c.nx, c.ny)); break;
            case 2: OEC_CUDA_TRY(launch_overlapped(k_mg_down<0, 1>, grid, dim3(kT), 0, s, m, mg->omega, b, l.x, c.b, c.nx, c.ny)); break;
            case 1: OEC_CUDA_TRY(launch_overlapped(k_mg_down<1, 0>, grid, dim3(kT), 0, s, m, mg->omega, b, l.x, c.b, c.nx, c.ny)); break;
            default: return OEC_ERR_INVALID;
        }
    }
    if (clustered) {
        C.b_top = B == 0 ? r : lv[B].b;
        C.out = B == 0 ? z : lv[B].y;
        if (B == 0 && acc) {
            C.q = q;
            C.acc = acc;
            C.ctl = ctl;
        }
        OEC_TRY(launch_mg_cluster(C, s));
    } else {
        MgBlock P{};
        P.nb = L - B;
        P.m = mg->ncoarse;
        for (int k = B; k < L; ++k) {
            const int j = k - B;
            P.nx[j] = lv[k].nx;
            P.ny[j] = lv[k].ny;
            P.ex[j] = lv[k].ex;
            P.ey[j] = lv[k].ey;
            P.leak[j] = lv[k].leak;
            P.dinv[j] = lv[k].dinv;
        }
        P.idx = mg->coarse_idx;
        P.inv = mg->coarse_inv;
        P.om = mg->omega;
        P.scale = mg->scale;
        const size_t smem = mg_block_smem(mg);
        if (smem > 48 * 1024) {
            // the largest dynamic shared-memory size enabled so far, per device
            static std::atomic<size_t> attr_set[kMaxDevices];
            int dev = 0;
            OEC_CUDA_TRY(cudaGetDevice(&dev));
            if (dev < 0 || dev >= kMaxDevices) return OEC_ERR_INVALID;
            if (smem > attr_set[dev].load()) {
                OEC_CUDA_TRY(cudaFuncSetAttribute(k_mg_block, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)kMgMaxBlockSmem));
                attr_set[dev].store(kMgMaxBlockSmem);
            }
        }
        const float *bin = B == 0 ? r : lv[B].b;
        float *yout = B == 0 ? z : lv[B].y;
        OEC_CUDA_TRY(launch_overlapped(k_mg_block, dim3(1), dim3(kBlockThreads), smem, s, P, bin, yout,
                                       mg_block_coef_smem(mg) ? 1 : 0));
    }
    for (int k = B - 1; k >= 0; --k) {
        const oec_mg_level_t &l = lv[k], &c = lv[k + 1];
        const dim3 grid((l.nx + kTX - 1) / kTX, (l.ny + kTY - 1) / kTY);
        const MgT m = mg_t(l, k > 0);
        const float *b = k == 0 ? r : l.b;
        float *out = k == 0 ? z : l.y;
        const float *qq = k == 0 ? q : nullptr;
        Acc *a = k == 0 ? acc : nullptr;
        const float om = mg->omega, sc = mg->scale;
        switch (mg_shift(l, c)) {
            case 3: OEC_CUDA_TRY(launch_overlapped(k_mg_up<1, 1>, grid, dim3(kT), 0, s, m, om, sc, b, l.x, c.y, c.nx, out, qq, a, ctl)); break;
            case 2: OEC_CUDA_TRY(launch_overlapped(k_mg_up<0, 1>, grid, dim3(kT), 0, s, m, om, sc, b, l.x, c.y, c.nx, out, qq, a, ctl)); break;
            case 1: OEC_CUDA_TRY(launch_overlapped(k_mg_up<1, 0>, grid, dim3(kT), 0, s, m, om, sc, b, l.x, c.y, c.nx, out, qq, a, ctl)); break;
            default: return OEC_ERR_INVALID;
        }
    }
    if (acc && B == 0 && !clustered) {
        const int G = lv[0].nx * lv[0].ny;
        OEC_CUDA_TRY(launch_overlapped(k_dots32, dim3(persistent_grid((G + kT - 1) / kT, 4)), dim3(kT), 0, s, G, r, z,
                                       q, acc, ctl));
    }
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

// z = M r by the multigrid or the network; with acc (multigrid only) the
// V-cycle also adds r.z and z.q to acc[ctl->slot].
int external_apply(int precond, const void *ctx, const float *r, float *z, const float *q, Acc *acc, const Ctl *ctl,
                   cudaStream_t s) {
    if (precond == OEC_PRECOND_MG) return mg_cycle(static_cast<const oec_mg_t *>(ctx), r, z, q, acc, ctl, s);
    return cnn_precond_apply(ctx, r, z, s);
}

struct Work {
    double *r64;
    float *r, *z, *p, *q, *d, *zn;
    Acc *acc;
    Ctl *ctl;
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
    w.ctl = reinterpret_cast<Ctl *>(c);
    return w;
}

bool valid_stencil(const oec_stencil_t *st) {
    return st && st->nx >= 3 && st->ny >= 3 && (int64_t)st->nx * st->ny < (1 << 28) && st->ex64 && st->ey64 &&
           st->ex32 && st->ey32 && st->dinv32 && st->inside && st->scale32 > 0.0;
}

// ------------------------------------------------------------ solve graph
// One solve is a graph of conditional nodes:
//   memset(ctl, stats)
//   WHILE refine:                        (h_outer, set by k_refine_begin)
//     k_residual64, k_refine_begin
//     IF work:                           (h_work)
//       [k_scale32, M r] k_init32        (arms h_inner)
//       WHILE inner:                     (h_inner: disarmed by k_apply32,
//         k_apply32, k_update32,          re-armed by k_direction32's check)
//         [M r (+ dots)], k_direction32
//       k_accumulate64
//   [k_fallback_flag, IF fallback: LU solve]
// Every loop ends: each refinement raises the refinement count (at most
// kMaxRefine) and each inner iteration the iteration count (at most
// max_iter), and a loop whose check did not run is left disarmed.

struct SolveArgs {
    const oec_stencil_t *st;
    const double *q;
    double *phi;
    double tol;
    int max_iter, precond;
    const void *ctx;
    void *work;
    oec_pcg_stats_t *stats;  // device
    const oec_lu_t *lu;      // optional fallback
    double *lu_work;
    int *fb_count;
};

// Side streams used to fill the bodies of conditional nodes (per device);
// used only under g_cache_mu.
cudaStream_t g_side[kMaxDevices][4];

int side_stream(int k, cudaStream_t *out) {
    int dev = 0;
    OEC_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return OEC_ERR_INVALID;
    if (!g_side[dev][k]) OEC_CUDA_TRY(cudaStreamCreateWithFlags(&g_side[dev][k], cudaStreamNonBlocking));
    *out = g_side[dev][k];
    return OEC_OK;
}

// Ends a capture into a body graph if the builder leaves early.
struct BodyCapture {
    cudaStream_t s = nullptr;
    int begin(int k, cudaGraph_t body) {
        cudaStream_t t;
        if (side_stream(k, &t) != OEC_OK) return OEC_ERR_CUDA;
        OEC_CUDA_TRY(cudaStreamBeginCaptureToGraph(t, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        s = t;
        return OEC_OK;
    }
    int end() {
        cudaGraph_t g;
        cudaStream_t t = s;
        s = nullptr;
        OEC_CUDA_TRY(cudaStreamEndCapture(t, &g));
        return OEC_OK;
    }
    ~BodyCapture() {
        if (s) {
            cudaGraph_t g;
            cudaStreamEndCapture(s, &g);
        }
    }
};

// Adds a conditional node with handle h after the current capture position
// of the capturing stream s; s continues after the node.  Returns the body.
int add_conditional(cudaStream_t s, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                    cudaGraph_t *body) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t g;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    OEC_CUDA_TRY(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive) return OEC_ERR_INVALID;
    cudaGraphNodeParams p{};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = type;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    OEC_CUDA_TRY(cudaGraphAddNode(&node, g, deps, nd, &p));
    *body = p.conditional.phGraph_out[0];
    OEC_CUDA_TRY(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    return OEC_OK;
}

int capture_graph(cudaStream_t s, cudaGraph_t *g) {
    cudaStreamCaptureStatus cs;
    OEC_CUDA_TRY(cudaStreamGetCaptureInfo(s, &cs, nullptr, g, nullptr, nullptr));
    return cs == cudaStreamCaptureStatusActive ? OEC_OK : OEC_ERR_INVALID;
}

// Records the whole solve into the capture of s.
// Grids up to this many nodes take the cooperative k_cg_step: its grid
// barriers cost less than three launches only while the passes are short
// (measured cold solves, 15 / 23 iterations: 128^2 circle 0.826 -> 0.778 ms,
// 1024^2 ellipse 2.83 -> 3.24 ms).
constexpr int kCgStepMaxNodes = 1 << 17;

// Grid of the cooperative k_cg_step for G nodes on this device: at most two
// resident CTAs per SM, so that the whole grid fits beside other work (0:
// a grid above kCgStepMaxNodes, cooperative launches unavailable, or
// OEC_CG_STEP=0 in the environment; the iteration then runs as three
// kernels).
int cg_step_grid(int G) {
    if (G > kCgStepMaxNodes) return 0;
    static std::atomic<int> cached[kMaxDevices];
    const int per_sm = per_device_cached(cached, [] {
        const char *e = getenv("OEC_CG_STEP");
        if (e && e[0] == '0') return 0;
        int dev = 0, coop = 0, b = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_cg_step, kT, 0) != cudaSuccess)
            b = 0;
        cudaGetLastError();
        return b < 2 ? b : 2;
    });
    if (per_sm <= 0) return 0;
    return persistent_grid((G + kT - 1) / kT, per_sm);
}

int build_solve(const SolveArgs &a, cudaStream_t s) {
    const oec_stencil_t *st = a.st;
    const int nx = st->nx, G = st->nx * st->ny;
    const int grid = persistent_grid((G + kT - 1) / kT, 4);
    const int pc = a.precond;
    const bool external = pc == OEC_PRECOND_CNN || pc == OEC_PRECOND_MG;
    const int coop_grid = pc == OEC_PRECOND_MG ? cg_step_grid(G) : 0;
    Work w = carve(a.work, G);
    OEC_CUDA_TRY(cudaMemsetAsync(w.ctl, 0, sizeof(Ctl), s));
    OEC_CUDA_TRY(cudaMemsetAsync(a.stats, 0, sizeof(oec_pcg_stats_t), s));
    cudaGraph_t top, b_outer, b_work, b_inner;
    OEC_TRY(capture_graph(s, &top));
    cudaGraphConditionalHandle h_outer, h_work, h_inner;
    OEC_CUDA_TRY(cudaGraphConditionalHandleCreate(&h_outer, top, 1, cudaGraphCondAssignDefault));
    OEC_TRY(add_conditional(s, h_outer, cudaGraphCondTypeWhile, &b_outer));
    {
        BodyCapture c1;
        OEC_TRY(c1.begin(0, b_outer));
        k_residual64<<<grid, kT, 0, c1.s>>>(nx, G, st->ex64, st->ey64, st->inside, a.q, a.phi, w.r64, w.ctl->nrm,
                                            h_outer);
        OEC_CUDA_TRY(cudaGraphConditionalHandleCreate(&h_work, b_outer, 0, 0));
        k_refine_begin<<<1, 32, 0, c1.s>>>(w.ctl, w.acc, a.tol, a.max_iter, st->scale32, a.stats, h_outer, h_work);
        OEC_LAUNCH_CHECK();
        OEC_TRY(add_conditional(c1.s, h_work, cudaGraphCondTypeIf, &b_work));
        {
            BodyCapture c2;
            OEC_TRY(c2.begin(1, b_work));
            OEC_CUDA_TRY(cudaGraphConditionalHandleCreate(&h_inner, b_work, 0, 0));
            if (coop_grid > 0) {
                // multigrid: V-cycle first in the loop body, then the CG step
                k_scale32<<<grid, kT, 0, c2.s>>>(G, w.r64, w.ctl, w.r);
                k_init_cg<<<grid, kT, 0, c2.s>>>(G, w.d, w.q, h_inner);
                OEC_LAUNCH_CHECK();
                OEC_TRY(add_conditional(c2.s, h_inner, cudaGraphCondTypeWhile, &b_inner));
                BodyCapture c3;
                OEC_TRY(c3.begin(2, b_inner));
                OEC_TRY(external_apply(pc, a.ctx, w.r, w.z, w.q, w.acc, w.ctl, c3.s));
                int max_iter = a.max_iter;
                void *args[] = {(void *)&nx, (void *)&G, (void *)&st->ex32, (void *)&st->ey32, (void *)&st->inside,
                                (void *)&w.z, (void *)&w.p, (void *)&w.q, (void *)&w.d, (void *)&w.r,
                                (void *)&w.acc, (void *)&w.ctl, (void *)&max_iter, (void *)&a.stats,
                                (void *)&h_inner};
                OEC_CUDA_TRY(cudaLaunchCooperativeKernel((void *)k_cg_step, dim3(coop_grid), dim3(kT), args, 0, c3.s));
                OEC_TRY(c3.end());
            } else {
                if (external) {
                    k_scale32<<<grid, kT, 0, c2.s>>>(G, w.r64, w.ctl, w.r);
                    OEC_LAUNCH_CHECK();
                    OEC_TRY(external_apply(pc, a.ctx, w.r, w.z, nullptr, nullptr, nullptr, c2.s));
                }
                k_init32<<<grid, kT, 0, c2.s>>>(G, w.r64, w.ctl, st->dinv32, pc, external ? 1 : 0, w.r, w.z, w.p, w.d,
                                                w.acc, h_inner);
                OEC_LAUNCH_CHECK();
                OEC_TRY(add_conditional(c2.s, h_inner, cudaGraphCondTypeWhile, &b_inner));
                {
                    BodyCapture c3;
                    OEC_TRY(c3.begin(2, b_inner));
                    k_apply32<<<grid, kT, 0, c3.s>>>(nx, G, st->ex32, st->ey32, st->inside, w.p, w.q, w.acc, w.ctl,
                                                     h_inner);
                    OEC_CUDA_TRY(launch_overlapped(k_update32, dim3(grid), dim3(kT), 0, c3.s, G, st->dinv32, pc, w.p, w.q,
                                                   w.d, w.r, w.z, w.acc, w.ctl));
                    OEC_LAUNCH_CHECK();
                    if (pc == OEC_PRECOND_MG) {
                        OEC_TRY(external_apply(pc, a.ctx, w.r, w.z, w.q, w.acc, w.ctl, c3.s));
                    } else if (external) {
                        OEC_TRY(external_apply(pc, a.ctx, w.r, w.zn, nullptr, nullptr, nullptr, c3.s));
                        OEC_CUDA_TRY(launch_overlapped(k_zdots32, dim3(grid), dim3(kT), 0, c3.s, G, w.r, w.zn, w.q, w.z,
                                                       w.acc, w.ctl));
                    }
                    OEC_CUDA_TRY(launch_overlapped(k_direction32, dim3(grid), dim3(kT), 0, c3.s, G, w.z, w.p, w.acc, w.ctl,
                                                   a.max_iter, a.stats, h_inner));
                    OEC_LAUNCH_CHECK();
                    OEC_TRY(c3.end());
                }
            }
            k_accumulate64<<<grid, kT, 0, c2.s>>>(G, w.ctl, w.d, st->inside, a.phi);
            OEC_LAUNCH_CHECK();
            OEC_TRY(c2.end());
        }
        OEC_TRY(c1.end());
    }
    if (a.lu) {
        cudaGraphConditionalHandle h_fb;
        cudaGraph_t b_fb;
        OEC_CUDA_TRY(cudaGraphConditionalHandleCreate(&h_fb, top, 0, 0));
        k_fallback_flag<<<1, 32, 0, s>>>(a.stats, a.fb_count, h_fb);
        OEC_LAUNCH_CHECK();
        OEC_TRY(add_conditional(s, h_fb, cudaGraphCondTypeIf, &b_fb));
        BodyCapture c4;
        OEC_TRY(c4.begin(3, b_fb));
        OEC_TRY(oec_lu_solve(a.lu, a.q, a.phi, a.lu_work, c4.s));
        OEC_TRY(c4.end());
    }
    return OEC_OK;
}

// Instantiated solve graphs, keyed by everything a graph depends on: the
// argument values and the contents of the structures they point to.
struct KeyBuilder {
    std::string k;
    template <typename T>
    void add(const T &v) { k.append(reinterpret_cast<const char *>(&v), sizeof(T)); }
    void bytes(const void *p, size_t n) {
        if (p) k.append(static_cast<const char *>(p), n);
    }
};

std::string solve_key(const SolveArgs &a, int dev) {
    KeyBuilder kb;
    kb.add(dev);
    kb.bytes(a.st, sizeof(*a.st));
    kb.add(a.q);
    kb.add(a.phi);
    kb.add(a.tol);
    kb.add(a.max_iter);
    kb.add(a.precond);
    kb.add(a.ctx);
    if (a.precond == OEC_PRECOND_MG) {
        const oec_mg_t *mg = static_cast<const oec_mg_t *>(a.ctx);
        kb.bytes(mg, sizeof(*mg));
        kb.bytes(mg->levels, sizeof(oec_mg_level_t) * mg->nlevels);
    } else if (a.precond == OEC_PRECOND_CNN) {
        kb.bytes(a.ctx, sizeof(oec_cnn_t));
    }
    kb.add(a.work);
    kb.add(a.stats);
    kb.add(a.lu);
    if (a.lu) {
        kb.bytes(a.lu, sizeof(*a.lu));
        kb.bytes(a.lu->l_level_ptr, sizeof(int32_t) * (a.lu->l_nlevels + 1));
        kb.bytes(a.lu->u_level_ptr, sizeof(int32_t) * (a.lu->u_nlevels + 1));
        if (a.lu->l_level_lanes) kb.bytes(a.lu->l_level_lanes, (size_t)a.lu->l_nlevels);
        if (a.lu->u_level_lanes) kb.bytes(a.lu->u_level_lanes, (size_t)a.lu->u_nlevels);
    }
    kb.add(a.lu_work);
    kb.add(a.fb_count);
    return kb.k;
}

// Instantiated solve graphs keyed by their arguments; g_cache_mu also
// guards the per-device capture and side streams of build_solve.
constexpr size_t kMaxCachedSolves = 32;
std::mutex g_cache_mu;
std::map<std::string, cudaGraphExec_t> g_cache;

// Launches the solve as an instantiated graph on s (built on first use).
// The lock is held through the launch, so no other thread can evict the
// graph between the lookup and the launch; a graph destroyed by a later
// eviction still completes the launches already queued.
int launch_cached_solve(const SolveArgs &a, cudaStream_t s) {
    int dev = 0;
    OEC_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return OEC_ERR_INVALID;
    const std::string key = solve_key(a, dev);
    std::lock_guard<std::mutex> lock(g_cache_mu);
    auto it = g_cache.find(key);
    if (it == g_cache.end()) {
        if (g_cache.size() >= kMaxCachedSolves) {
            for (auto &e : g_cache) cudaGraphExecDestroy(e.second);
            g_cache.clear();
        }
        // a stream of its own for the top-level capture (the side streams
        // fill the bodies)
        static cudaStream_t g_cap[kMaxDevices] = {};
        if (!g_cap[dev]) OEC_CUDA_TRY(cudaStreamCreateWithFlags(&g_cap[dev], cudaStreamNonBlocking));
        cudaStream_t cap = g_cap[dev];
        OEC_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeRelaxed));
        const int rc = build_solve(a, cap);
        cudaGraph_t g = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(cap, &g);
        if (rc != OEC_OK || ec != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return rc != OEC_OK ? rc : OEC_ERR_CUDA;
        }
        cudaGraphExec_t exec;
        const cudaError_t ei = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        OEC_CUDA_TRY(ei);
        it = g_cache.emplace(key, exec).first;
    }
    OEC_CUDA_TRY(cudaGraphLaunch(it->second, s));
    return OEC_OK;
}

int check_solve_args(const SolveArgs &a) {
    if (!valid_stencil(a.st) || !a.q || !a.phi || !a.work || !a.stats || !(a.tol > 0.0) || a.max_iter < 0 ||
        a.max_iter > (1 << 24))
        return OEC_ERR_INVALID;
    if (a.precond < OEC_PRECOND_NONE || a.precond > OEC_PRECOND_MG) return OEC_ERR_INVALID;
    const bool external = a.precond == OEC_PRECOND_CNN || a.precond == OEC_PRECOND_MG;
    if (external && !a.ctx) return OEC_ERR_INVALID;
    if (a.precond == OEC_PRECOND_MG) {
        const oec_mg_t *mg = static_cast<const oec_mg_t *>(a.ctx);
        if (!valid_mg(mg) || mg->levels[0].nx != a.st->nx || mg->levels[0].ny != a.st->ny) return OEC_ERR_INVALID;
    }
    if (a.lu && (!a.lu_work || a.lu->n_nodes != a.st->nx * a.st->ny)) return OEC_ERR_INVALID;
    return OEC_OK;
}

// Enqueues the solve on s: into its capture when s is capturing, else as a
// launch of the cached graph.
int enqueue_solve(const SolveArgs &a, cudaStream_t s) {
    OEC_TRY(check_solve_args(a));
    cudaStreamCaptureStatus cs;
    OEC_CUDA_TRY(cudaStreamIsCapturing(s, &cs));
    // building a graph may set kernel attributes on first use; allow that
    // while another capture is under way
    cudaStreamCaptureMode mode = cudaStreamCaptureModeRelaxed;
    OEC_CUDA_TRY(cudaThreadExchangeStreamCaptureMode(&mode));
    int rc;
    if (cs == cudaStreamCaptureStatusActive) {
        std::lock_guard<std::mutex> lock(g_cache_mu);  // the side streams are shared per device
        rc = build_solve(a, s);
    } else if (cs == cudaStreamCaptureStatusNone) {
        rc = launch_cached_solve(a, s);
    } else {
        rc = OEC_ERR_INVALID;
    }
    cudaThreadExchangeStreamCaptureMode(&mode);
    return rc;
}

// phi <- 2 phi - prev, prev <- phi (the old phi): the linear extrapolation
// in time of the last two solutions, in one pass over both vectors.  While
// fewer than two solutions exist (*hist < 2) phi is kept and only copied to
// prev.  The count advances in a separate launch so that every CTA of this one
// reads the same value.
__global__ void k_extrapolate(double *__restrict__ phi, double *__restrict__ prev, int64_t n,
                              const int32_t *__restrict__ hist) {
    const bool extrapolate = hist == nullptr || *hist >= 2;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double a = phi[i];
        if (extrapolate) phi[i] = 2.0 * a - prev[i];
        prev[i] = a;
    }
}

__global__ void k_history_advance(int32_t *hist) { *hist = min(*hist + 1, 2); }

}  // namespace
}  // namespace oec

using namespace oec;

extern "C" int oec_warm_start_extrapolate(double *phi_dev, double *phi_prev_dev, int64_t n, int32_t *history_dev,
                                          void *stream) {
    if (!phi_dev || !phi_prev_dev || n < 0) return OEC_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    if (n > 0)
        k_extrapolate<<<persistent_grid((n + 255) / 256, 4), 256, 0, s>>>(phi_dev, phi_prev_dev, n, history_dev);
    if (history_dev) k_history_advance<<<1, 1, 0, s>>>(history_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int64_t oec_pcg_work_bytes(int32_t nx, int32_t ny) {
    const size_t G = (size_t)nx * (size_t)ny;
    return (int64_t)(align256(sizeof(double) * G) + 6 * align256(sizeof(float) * G) + align256(sizeof(Acc) * 2) +
                     align256(sizeof(Ctl)));
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
    if (!valid_stencil(st) || !work_dev || !stats) return OEC_ERR_INVALID;
    Work w = carve(work_dev, st->nx * st->ny);
    SolveArgs a{st, q_dev, phi_dev, tol, max_iter, precond, precond_ctx, work_dev, &w.ctl->stats,
                nullptr, nullptr, nullptr};
    cudaStream_t s = as_stream(stream);
    cudaStreamCaptureStatus cs;
    OEC_CUDA_TRY(cudaStreamIsCapturing(s, &cs));
    if (cs != cudaStreamCaptureStatusNone) return OEC_ERR_INVALID;  // reports to the host: use the async form
    OEC_TRY(enqueue_solve(a, s));
    OEC_CUDA_TRY(cudaMemcpyAsync(stats, &w.ctl->stats, sizeof(*stats), cudaMemcpyDeviceToHost, s));
    OEC_CUDA_TRY(cudaStreamSynchronize(s));
    return OEC_OK;
}

extern "C" int oec_pcg_solve_async(const oec_stencil_t *st, const double *q_dev, double *phi_dev, double tol,
                                   int32_t max_iter, int32_t precond, const void *precond_ctx, void *work_dev,
                                   oec_pcg_stats_t *stats_dev, const oec_lu_t *fallback, double *lu_work_dev,
                                   int32_t *fallback_count_dev, void *stream) {
    SolveArgs a{st, q_dev, phi_dev, tol, max_iter, precond, precond_ctx, work_dev, stats_dev,
                fallback, lu_work_dev, fallback_count_dev};
    return enqueue_solve(a, as_stream(stream));
}

extern "C" int oec_mg_apply(const oec_mg_t *mg, const float *r_dev, float *z_dev, void *stream) {
    if (!valid_mg(mg) || !r_dev || !z_dev) return OEC_ERR_INVALID;
    return mg_cycle(mg, r_dev, z_dev, nullptr, nullptr, nullptr, as_stream(stream));
}
