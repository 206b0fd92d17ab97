// poisson.cu -- Poisson solve on the device: the FP64 LU back-substitution
// (the direct solve, and the fallback and error reference of the iterative
// one) and the sparse E = phiToE * phi product.
//
// Reference: poissonSolver.pyx:83-88 (phi[inside] = lu.solve(q[inside]);
// E = phiToE . phi).  SuperLU's factors P_r A P_c = L U are produced on the
// host at setup with the reference's options (poissonSolver.pyx:59).
//
// Triangular solves.  The factors of a 2-D FIT operator under a minimum-degree
// ordering have a wide bottom (many independent rows per dependency level)
// and a long thin top: the separator rows, one or two rows per level.  The
// rows are split at setup into a "head", solved level by level, and a
// "tail" of the last m rows, whose triangular block is inverted densely at
// setup and applied as a matrix-vector product, turning hundreds of one-row
// levels into one bandwidth-bound pass.  Of the head levels, runs of narrow
// ones go to one CTA each (a __syncthreads between levels), and the wide
// ones between the runs to one cooperative launch per segment of 2-64 levels
// or a launch per level (or, on request, each whole triangle to one CTA with
// the vector in shared memory).
#include <math.h>
#include <stdint.h>

#include <cooperative_groups.h>

#include <algorithm>
#include <vector>

#include "oec_common.cuh"

namespace oec {
namespace {

constexpr int kWarps = 8;  // warps per CTA in the row kernels

// The head CSR is stored in level order: position w holds factor row
// rows[w] (its entries ptr[w]..ptr[w+1], its diagonal diag[w]), so a row's
// record is read with independent loads rather than through rows[w].
//
// x[r] = (x[r] - sum_j A[r,j] x[j]) / d[r] for the rows [w0, w1) of one level.
__global__ void __launch_bounds__(kWarps * 32)
    k_trsv_rows(const int32_t *__restrict__ rows, int w0, int w1, const int32_t *__restrict__ ptr,
                const int32_t *__restrict__ idx, const double *__restrict__ val, const double *__restrict__ diag,
                double *__restrict__ x) {
    const int w = w0 + blockIdx.x * kWarps + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (w >= w1) return;
    const int r = rows[w], k1 = ptr[w + 1];
    double s = 0.0;
    for (int k = ptr[w] + lane; k < k1; k += 32) s += val[k] * x[idx[k]];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFullMask, s, o);
    if (lane == 0) {
        double v = x[r] - s;
        x[r] = diag ? v / diag[w] : v;
    }
}

// Every level of one triangle in one cooperative launch: the warps of the
// grid share each level's rows and a grid-wide barrier separates the levels
// (the launch guarantees that every CTA is resident, so the barrier is the
// hardware's, not a spin).  x is read through L2 (__ldcg): a row's inputs were
// written by other SMs after this SM's L1 may have cached their lines.
// Up to this many levels one cooperative launch replaces the launches of a
// segment (128^2: 40 levels in 0.17 ms against 0.22 ms as launches); the
// level pointers travel in the parameter block.
constexpr int kCoopMaxLevels = 64;
struct LevelPtr {
    int n;
    int ptr[kCoopMaxLevels + 1];
};

__global__ void __launch_bounds__(kWarps * 32)
    k_trsv_levels(const int32_t *__restrict__ rows, LevelPtr lv, const int32_t *__restrict__ ptr,
                  const int32_t *__restrict__ idx, const double *__restrict__ val, const double *__restrict__ diag,
                  double *x) {
    cooperative_groups::grid_group grid = cooperative_groups::this_grid();
    const int lane = threadIdx.x & 31;
    const int w0 = blockIdx.x * kWarps + (threadIdx.x >> 5), nw = gridDim.x * kWarps;
    for (int l = 0; l < lv.n; ++l) {
        for (int w = lv.ptr[l] + w0; w < lv.ptr[l + 1]; w += nw) {
            const int r = rows[w], k1 = ptr[w + 1];
            double s = 0.0;
            for (int k = ptr[w] + lane; k < k1; k += 32) s += val[k] * __ldcg(&x[idx[k]]);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFullMask, s, o);
            if (lane == 0) {
                const double v = __ldcg(&x[r]) - s;
                x[r] = diag ? v / diag[w] : v;
            }
        }
        if (l + 1 < lv.n) grid.sync();
    }
}

// Small systems (every unknown fits one CTA's shared memory as f64), on
// request: each triangle is solved by one 1024-thread CTA with the solution
// vector in shared memory and __syncthreads between the levels, a fraction of
// a grid barrier's cost.  One SM has too few loads in flight for the factors'
// entries, though: at 128^2 (12644 unknowns, 20 levels) it ties with the
// cooperative launch on a warm L2 (0.172 against 0.166 ms) and loses inside a
// buildup step, where the other kernels have evicted the factors (2500 steps:
// 0.78 against 0.71 s), so the automatic choice does not take it.  A level's
// rows are spread over the CTA with g lanes per row, g the largest power of
// two up to 32 that keeps the level in one pass
// (1 for the wide bottom levels; the narrow top levels have the long rows).
// A level's cost is the latency of its loads, so the record of a thread's
// first row in the next level (row, entry range, diagonal; none of it
// depends on x) is loaded while the current level computes.
constexpr int kBlockThreads = 1024;
constexpr int kBlockMaxRows = 28672;  // 224 KB of f64

struct RowRec {
    int r, k0, k1;
    double d;
};

__device__ __forceinline__ int level_lanes(int nrows) {
    int g = 1;
    while (g < 32 && nrows * (2 * g) <= kBlockThreads) g *= 2;
    return g;
}

__device__ __forceinline__ RowRec row_rec(int w, int w1, const int32_t *__restrict__ rows,
                                          const int32_t *__restrict__ ptr, const double *__restrict__ diag) {
    RowRec rc{-1, 0, 0, 1.0};
    if (w < w1) {
        rc.r = rows[w];
        rc.k0 = ptr[w];
        rc.k1 = ptr[w + 1];
        if (diag) rc.d = diag[w];
    }
    return rc;
}

__device__ __forceinline__ void block_levels(const int32_t *__restrict__ rows, const LevelPtr &lv, int l0,
                                             const int32_t *__restrict__ ptr, const int32_t *__restrict__ idx,
                                             const double *__restrict__ val, const double *__restrict__ diag,
                                             double *xs) {
    if (l0 >= lv.n) return;
    int g = level_lanes(lv.ptr[l0 + 1] - lv.ptr[l0]);
    RowRec nxt = row_rec(lv.ptr[l0] + (int)threadIdx.x / g, lv.ptr[l0 + 1], rows, ptr, diag);
    for (int l = l0; l < lv.n; ++l) {
        const int r0 = lv.ptr[l], r1 = lv.ptr[l + 1];
        const int sub = threadIdx.x & (g - 1), groups = kBlockThreads / g;
        RowRec cur = nxt;
        const int gn = l + 1 < lv.n ? level_lanes(lv.ptr[l + 2] - lv.ptr[l + 1]) : 1;
        if (l + 1 < lv.n) nxt = row_rec(lv.ptr[l + 1] + (int)threadIdx.x / gn, lv.ptr[l + 2], rows, ptr, diag);
        for (int base = r0; base < r1; base += groups) {  // same trip count in every thread
            if (base != r0) cur = row_rec(base + (int)threadIdx.x / g, r1, rows, ptr, diag);
            double s = 0.0;
            for (int k = cur.k0 + sub; k < cur.k1; k += g) s += val[k] * xs[idx[k]];
            for (int o = g >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(kFullMask, s, o);
            if (cur.r >= 0 && sub == 0) {
                const double v = xs[cur.r] - s;
                xs[cur.r] = diag ? v / cur.d : v;
            }
        }
        g = gn;
        __syncthreads();
    }
}

// Forward half: gather the permuted right-hand side (c = P_r q), solve the
// unit-lower head and write y_head to c[0, h) (the tail's rows of c keep
// their right-hand side).  The first level of a strictly lower triangle has
// no entries (any entry would be a dependency), so it is skipped.
__global__ void __launch_bounds__(kBlockThreads)
    k_lu_block_lower(int n, int h, const int32_t *__restrict__ rhs_node, const double *__restrict__ q,
                     const int32_t *__restrict__ rows, LevelPtr lv, const int32_t *__restrict__ ptr,
                     const int32_t *__restrict__ idx, const double *__restrict__ val, double *__restrict__ c) {
    extern __shared__ double xs[];
#pragma unroll 4
    for (int i = threadIdx.x; i < n; i += kBlockThreads) xs[i] = q[rhs_node[i]];
    __syncthreads();
    block_levels(rows, lv, 1, ptr, idx, val, nullptr, xs);
#pragma unroll 4
    for (int i = threadIdx.x; i < n; i += kBlockThreads) c[i] = xs[i];
}

// Backward half: z_head from y_head (c[0, h)) and the solved tail (z_tail),
// then phi[node of unknown i] = z[perm_c[i]] straight from shared memory.
__global__ void __launch_bounds__(kBlockThreads)
    k_lu_block_upper(int n, int h, const double *__restrict__ c, const double *__restrict__ ztail,
                     const int32_t *__restrict__ rows, LevelPtr lv, const int32_t *__restrict__ ptr,
                     const int32_t *__restrict__ idx, const double *__restrict__ val,
                     const double *__restrict__ diag, const int32_t *__restrict__ sol_src,
                     const int32_t *__restrict__ sol_node, double *__restrict__ phi) {
    extern __shared__ double xs[];
#pragma unroll 4
    for (int i = threadIdx.x; i < n; i += kBlockThreads) xs[i] = i < h ? c[i] : ztail[i - h];
    __syncthreads();
    block_levels(rows, lv, 0, ptr, idx, val, diag, xs);
#pragma unroll 4
    for (int i = threadIdx.x; i < n; i += kBlockThreads) phi[sol_node[i]] = xs[sol_src[i]];
}

// t[i] = b[i] - sum_j C[i,j] x[j]   (the tail's right-hand side after the head)
__global__ void __launch_bounds__(kWarps * 32)
    k_spmv_rhs(int nrows, const int32_t *__restrict__ ptr, const int32_t *__restrict__ idx,
               const double *__restrict__ val, const double *__restrict__ x, const double *__restrict__ b,
               double *__restrict__ t) {
    int w = blockIdx.x * kWarps + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (w >= nrows) return;
    double s = 0.0;
    for (int k = ptr[w] + lane; k < ptr[w + 1]; k += 32) s += val[k] * x[idx[k]];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFullMask, s, o);
    if (lane == 0) t[w] = b[w] - s;
}

// Runs of narrow head levels in one CTA.  Most levels of a large factor hold
// a few rows with short entry lists, so a launch per level costs its launch
// and drain (~8.5 us at 1024^2) for a chain of three dependent loads; one CTA
// runs a whole run of such levels with a __syncthreads between them.  The
// setup marks a level for this when its rows fit one pass of the CTA and its
// longest row needs few loads per lane; lanes[l] is the lanes per row (a
// power of two up to 32).  x is read and written in global memory: the
// earlier levels of the run were written by this CTA (same SM), the rest by
// earlier launches.
constexpr int kThinMaxLevels = 2048;
struct ThinLevels {
    int n;
    int ptr[kThinMaxLevels + 1];
    int8_t lanes[kThinMaxLevels];
};

// A lane's share of one row of a run level: the row, its entry range and
// diagonal, and its first kThinPre entries.  None of it depends on x, so the
// next level's share is loaded while the current level computes and a level
// waits only for its x values.
constexpr int kThinPre = 4;
struct ThinRow {
    int r, k0, k1;
    double d;
    double v[kThinPre];
    int c[kThinPre];
};

__device__ __forceinline__ void thin_fetch(ThinRow &t, int w, int w1, int sub, int g,
                                           const int32_t *__restrict__ rows, const int32_t *__restrict__ ptr,
                                           const int32_t *__restrict__ idx, const double *__restrict__ val,
                                           const double *__restrict__ diag) {
    t.r = -1;
    if (w < w1) {
        t.r = rows[w];
        t.k0 = ptr[w] + sub;
        t.k1 = ptr[w + 1];
        t.d = diag ? diag[w] : 1.0;
#pragma unroll
        for (int j = 0; j < kThinPre; ++j) {
            const int k = t.k0 + j * g;
            if (k < t.k1) {
                t.v[j] = val[k];
                t.c[j] = idx[k];
            }
        }
    }
}

__global__ void __launch_bounds__(kBlockThreads)
    k_trsv_thin(const int32_t *__restrict__ rows, ThinLevels lv, const int32_t *__restrict__ ptr,
                const int32_t *__restrict__ idx, const double *__restrict__ val, const double *__restrict__ diag,
                double *x) {
    const int tid = threadIdx.x;
    ThinRow nxt;
    {
        const int g0 = lv.lanes[0];
        thin_fetch(nxt, lv.ptr[0] + tid / g0, lv.ptr[1], tid & (g0 - 1), g0, rows, ptr, idx, val, diag);
    }
    for (int l = 0; l < lv.n; ++l) {
        const int g = lv.lanes[l];
        const int sub = tid & (g - 1), groups = kBlockThreads / g;
        const int r0 = lv.ptr[l], r1 = lv.ptr[l + 1];
        ThinRow cur = nxt;
        if (l + 1 < lv.n) {
            const int gn = lv.lanes[l + 1];
            thin_fetch(nxt, lv.ptr[l + 1] + tid / gn, lv.ptr[l + 2], tid & (gn - 1), gn, rows, ptr, idx, val, diag);
        }
        for (int base = r0; base < r1; base += groups) {  // one pass as set up; same trip count in every thread
            if (base != r0) thin_fetch(cur, base + tid / g, r1, sub, g, rows, ptr, idx, val, diag);
            double s = 0.0;
            if (cur.r >= 0) {
#pragma unroll
                for (int j = 0; j < kThinPre; ++j)
                    if (cur.k0 + j * g < cur.k1) s += cur.v[j] * x[cur.c[j]];
                for (int k = cur.k0 + kThinPre * g; k < cur.k1; k += g) s += val[k] * x[idx[k]];
            }
            for (int o = g >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(kFullMask, s, o);
            if (cur.r >= 0 && sub == 0) {
                const double v = x[cur.r] - s;
                x[cur.r] = diag ? v / cur.d : v;
            }
        }
        __syncthreads();
    }
}

// out[i] = sum_{j in tri(i)} T[i*m + j] in[j]; lower: j <= i, upper: j >= i.
// One CTA per row; rows are contiguous in memory so the loads coalesce.  The
// inverse is read once per solve with evict-first loads, so its streaming
// (up to 1 GB a triangle) leaves the head factors and the vector in L2
// (c1 passage 0.62 -> 0.59 s, 512^2 solve 1.63 -> 1.53 ms).
template <bool LOWER>
__global__ void __launch_bounds__(256)
    k_dense_tri(int m, const double *__restrict__ T, const double *__restrict__ in, double *__restrict__ out) {
    __shared__ double red[8];
    int i = blockIdx.x;
    const double *row = T + (int64_t)i * m;
    int j0 = LOWER ? 0 : i, j1 = LOWER ? i + 1 : m;
    double s = 0.0;
    for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) s += __ldcs(row + j) * in[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFullMask, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFullMask, s, o);
        if (threadIdx.x == 0) out[i] = s;
    }
}

__global__ void k_lu_gather(int n, const int32_t *__restrict__ node, const double *__restrict__ q,
                            double *__restrict__ c) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) c[k] = q[node[k]];
}

__global__ void k_lu_scatter(int n, const int32_t *__restrict__ src, const int32_t *__restrict__ node,
                             const double *__restrict__ z, double *__restrict__ phi) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        phi[node[i]] = z[src[i]];
}

// y = A x (CSR), a thread per row: the field operator phiToE has 0-6
// entries per row (1.6 on average), which a warp per row would leave 30 of
// 32 lanes idle on (1024^2: 334 us against a 75 MB pass).  Adjacent rows'
// entries are adjacent, so the loads of a warp stay within a few lines.
__global__ void __launch_bounds__(256)
    k_spmv(int nrows, const int32_t *__restrict__ ptr, const int32_t *__restrict__ idx,
           const double *__restrict__ val, const double *__restrict__ x, double *__restrict__ y) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += gridDim.x * blockDim.x) {
        const int k1 = ptr[r + 1];
        double s = 0.0;
        for (int k = ptr[r]; k < k1; ++k) s += val[k] * x[idx[k]];
        y[r] = s;
    }
}

inline unsigned warp_blocks(int rows) { return (unsigned)((rows + kWarps - 1) / kWarps); }

}  // namespace
}  // namespace oec

using namespace oec;

namespace oec {
namespace {

LevelPtr level_ptrs(const int32_t *level_ptr, int nlevels) {
    LevelPtr lv;
    lv.n = nlevels;
    for (int l = 0; l <= nlevels; ++l) lv.ptr[l] = level_ptr[l];
    return lv;
}

// The whole solve of a small system (n <= kBlockMaxRows, both triangles of at
// most kCoopMaxLevels head levels): the two one-CTA triangle kernels around
// the tail's right-hand side and its two dense products.
int lu_solve_block(const oec_lu_t *lu, const double *q, double *phi, double *c, double *t, cudaStream_t s) {
    const int n = lu->n, h = lu->head, m = n - h;
    const size_t smem = sizeof(double) * (size_t)n;
    static size_t attr_set = 0;  // largest dynamic shared-memory size enabled so far
    if (smem > 48 * 1024 && smem > attr_set) {
        OEC_CUDA_TRY(cudaFuncSetAttribute(k_lu_block_lower, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        OEC_CUDA_TRY(cudaFuncSetAttribute(k_lu_block_upper, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr_set = smem;
    }
    OEC_CUDA_TRY(cudaMemsetAsync(phi, 0, sizeof(double) * (size_t)lu->n_nodes, s));
    k_lu_block_lower<<<1, kBlockThreads, smem, s>>>(n, h, lu->rhs_node, q, lu->l_rows,
                                                    level_ptrs(lu->l_level_ptr, lu->l_nlevels), lu->l_ptr, lu->l_idx,
                                                    lu->l_val, c);
    if (m > 0) {
        k_spmv_rhs<<<warp_blocks(m), kWarps * 32, 0, s>>>(m, lu->lc_ptr, lu->lc_idx, lu->lc_val, c, c + h, t);
        k_dense_tri<true><<<m, 256, 0, s>>>(m, lu->tl_inv, t, c + h);   // y_tail
        k_dense_tri<false><<<m, 256, 0, s>>>(m, lu->tu_inv, c + h, t);  // z_tail
    }
    k_lu_block_upper<<<1, kBlockThreads, smem, s>>>(n, h, c, t, lu->u_rows,
                                                    level_ptrs(lu->u_level_ptr, lu->u_nlevels), lu->u_ptr, lu->u_idx,
                                                    lu->u_val, lu->u_diag, lu->sol_src, lu->sol_node, phi);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

inline bool thin_lanes_ok(int g) { return g == 1 || g == 2 || g == 4 || g == 8 || g == 16 || g == 32; }

// Levels [a, b) of one triangle, each its own launch, or one cooperative
// launch when `coop` allows it, they are at least two and fit the parameter
// block and the device supports it.
int solve_wide(const int32_t *rows, const int32_t *level_ptr, int a, int b, const int32_t *ptr, const int32_t *idx,
               const double *val, const double *diag, double *x, bool coop_ok, cudaStream_t s) {
    // resident CTAs per SM of the cooperative kernel, per device (0: no cooperative launch)
    static std::atomic<int> cached[kMaxDevices];
    const int per_sm = per_device_cached(cached, [] {
        int dev = 0, coop = 0, b = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_trsv_levels, kWarps * 32, 0) != cudaSuccess)
            b = 0;
        cudaGetLastError();
        return b;
    });
    const int n = b - a;
    if (coop_ok && per_sm > 0 && n >= 2 && n <= kCoopMaxLevels) {
        LevelPtr lv = level_ptrs(level_ptr + a, n);
        int widest = 0;
        for (int l = a; l < b; ++l) widest = std::max(widest, level_ptr[l + 1] - level_ptr[l]);
        // one CTA per SM: a wider grid makes every barrier dearer than the
        // extra warps save on the few wide levels
        const int grid = std::max(1, std::min(sm_count(), (widest + kWarps - 1) / kWarps));
        void *args[] = {(void *)&rows, (void *)&lv, (void *)&ptr, (void *)&idx, (void *)&val, (void *)&diag,
                        (void *)&x};
        OEC_CUDA_TRY(cudaLaunchCooperativeKernel((void *)k_trsv_levels, dim3(grid), dim3(kWarps * 32), args, 0, s));
        return OEC_OK;
    }
    for (int l = a; l < b; ++l) {
        const int r0 = level_ptr[l], r1 = level_ptr[l + 1];
        if (r1 > r0) k_trsv_rows<<<warp_blocks(r1 - r0), kWarps * 32, 0, s>>>(rows, r0, r1, ptr, idx, val, diag, x);
    }
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

// The levels of one triangle: runs of two or more levels that `lanes` (host,
// per level; optional) marks for one CTA go to k_trsv_thin, the levels
// between them to solve_wide.
int solve_levels(const int32_t *rows, const int32_t *level_ptr, int nlevels, const int8_t *lanes,
                 const int32_t *ptr, const int32_t *idx, const double *val, const double *diag, double *x,
                 bool coop_ok, cudaStream_t s) {
    if (nlevels <= 0) return OEC_OK;
    auto thin = [&](int l) { return lanes && l < nlevels && thin_lanes_ok(lanes[l]); };
    int l = 0;
    while (l < nlevels) {
        int e = l;
        while (thin(e) && e - l < kThinMaxLevels) ++e;
        if (e - l >= 2) {
            ThinLevels tl;
            tl.n = e - l;
            for (int k = 0; k <= tl.n; ++k) tl.ptr[k] = level_ptr[l + k];
            for (int k = 0; k < tl.n; ++k) tl.lanes[k] = lanes[l + k];
            k_trsv_thin<<<1, kBlockThreads, 0, s>>>(rows, tl, ptr, idx, val, diag, x);
            OEC_LAUNCH_CHECK();
            l = e;
            continue;
        }
        // up to the next run of two marked levels
        e = l + 1;
        while (e < nlevels && !(thin(e) && thin(e + 1))) ++e;
        const int rc = solve_wide(rows, level_ptr, l, e, ptr, idx, val, diag, x, coop_ok, s);
        if (rc != OEC_OK) return rc;
        l = e;
    }
    return OEC_OK;
}

}  // namespace
}  // namespace oec

extern "C" int oec_lu_solve(const oec_lu_t *lu, const double *q_dev, double *phi_dev, double *work_dev,
                            void *stream) {
    if (!lu || !q_dev || !phi_dev || !work_dev || lu->n <= 0 || lu->head < 0 || lu->head > lu->n)
        return OEC_ERR_INVALID;
    const int n = lu->n, h = lu->head, m = n - h;
    if (m > 0 && (!lu->tl_inv || !lu->tu_inv)) return OEC_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    double *c = work_dev;      // n: right-hand side, then y, then z (in place)
    double *t = work_dev + n;  // m: tail scratch
    const int path = lu->head_path;
    if (path < OEC_LU_HEAD_AUTO || path > OEC_LU_HEAD_ONE_CTA) return OEC_ERR_INVALID;
    const bool few_levels = lu->l_nlevels <= kCoopMaxLevels && lu->u_nlevels <= kCoopMaxLevels;
    if (path == OEC_LU_HEAD_ONE_CTA && n <= kBlockMaxRows && few_levels)
        return lu_solve_block(lu, q_dev, phi_dev, c, t, s);
    const bool coop = path != OEC_LU_HEAD_PER_LEVEL;
    const bool runs = path == OEC_LU_HEAD_AUTO || path == OEC_LU_HEAD_ONE_CTA;  // one-CTA runs of marked levels
    k_lu_gather<<<persistent_grid((n + 255) / 256, 4), 256, 0, s>>>(n, lu->rhs_node, q_dev, c);
    OEC_LAUNCH_CHECK();
    // forward, head levels (unit lower: no diagonal).  The first level of a
    // strictly lower triangle has no entries (any entry would be a
    // dependency): its rows keep their right-hand side, so it is skipped.
    const int l_skip = lu->l_nlevels > 0 ? 1 : 0;
    int rc = solve_levels(lu->l_rows, lu->l_level_ptr + l_skip, lu->l_nlevels - l_skip,
                          runs && lu->l_level_lanes ? lu->l_level_lanes + l_skip : nullptr, lu->l_ptr, lu->l_idx,
                          lu->l_val, nullptr, c, coop, s);
    if (rc != OEC_OK) return rc;
    if (m > 0) {
        // t = c_tail - L[tail, head] y_head ; y_tail = TLinv t ; z_tail = TUinv y_tail
        k_spmv_rhs<<<warp_blocks(m), kWarps * 32, 0, s>>>(m, lu->lc_ptr, lu->lc_idx, lu->lc_val, c, c + h, t);
        k_dense_tri<true><<<m, 256, 0, s>>>(m, lu->tl_inv, t, c + h);
        k_dense_tri<false><<<m, 256, 0, s>>>(m, lu->tu_inv, c + h, t);
        OEC_CUDA_TRY(cudaMemcpyAsync(c + h, t, sizeof(double) * m, cudaMemcpyDeviceToDevice, s));
        OEC_LAUNCH_CHECK();
    }
    // backward, head levels (rows use every column > row, tail included)
    rc = solve_levels(lu->u_rows, lu->u_level_ptr, lu->u_nlevels, runs ? lu->u_level_lanes : nullptr, lu->u_ptr,
                      lu->u_idx, lu->u_val, lu->u_diag, c, coop, s);
    if (rc != OEC_OK) return rc;
    OEC_CUDA_TRY(cudaMemsetAsync(phi_dev, 0, sizeof(double) * (size_t)lu->n_nodes, s));
    k_lu_scatter<<<persistent_grid((n + 255) / 256, 4), 256, 0, s>>>(n, lu->sol_src, lu->sol_node, c, phi_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_spmv_csr(int32_t nrows, const int32_t *ptr_dev, const int32_t *idx_dev, const double *val_dev,
                            const double *x_dev, double *y_dev, void *stream) {
    if (nrows < 0 || !ptr_dev || !idx_dev || !val_dev || !x_dev || !y_dev) return OEC_ERR_INVALID;
    if (nrows == 0) return OEC_OK;
    k_spmv<<<persistent_grid((nrows + 255) / 256, 8), 256, 0, as_stream(stream)>>>(nrows, ptr_dev, idx_dev, val_dev,
                                                                                  x_dev, y_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

// --------------------------------------------------------- host: levels
// Dependency level of every row of a triangular CSR matrix (restricted to
// rows [0, nrows) and columns [0, ncols_dep)): level(r) = 1 + max level of
// the rows it reads.  lower: columns < r, else columns > r (processed from
// the last row).  Returns the number of levels.
extern "C" int oec_trsv_levels(int32_t nrows, const int32_t *ptr, const int32_t *idx, int32_t lower,
                               int32_t ncols_dep, int32_t *level_out, int32_t *nlevels_out) {
    if (nrows < 0 || !ptr || !idx || !level_out || !nlevels_out) return OEC_ERR_INVALID;
    int32_t maxl = 0;
    if (lower) {
        for (int32_t r = 0; r < nrows; ++r) {
            int32_t l = 0;
            for (int32_t k = ptr[r]; k < ptr[r + 1]; ++k) {
                int32_t j = idx[k];
                if (j < r && j < ncols_dep) l = std::max(l, level_out[j]);
            }
            level_out[r] = l + 1;
            maxl = std::max(maxl, l + 1);
        }
    } else {
        for (int32_t r = nrows - 1; r >= 0; --r) {
            int32_t l = 0;
            for (int32_t k = ptr[r]; k < ptr[r + 1]; ++k) {
                int32_t j = idx[k];
                if (j > r && j < ncols_dep) l = std::max(l, level_out[j]);
            }
            level_out[r] = l + 1;
            maxl = std::max(maxl, l + 1);
        }
    }
    *nlevels_out = maxl;
    return OEC_OK;
}
