// manage.cu -- macro-particle management on the device: stable radix sort
// (sortByColumn, cell ordering), Russian roulette (globalRandom) and the
// cell-binned phase-space merge (localRandom).
//
// Reference: particles.pyx sortByColumn (:49-50, :431-459),
// particleManagement.pyx globalRandom (:35-67) and localRandom (:74-238).
//  * Sorting is a stable least-significant-digit radix sort of 32-bit keys
//    (8-bit digits): per pass a per-tile digit histogram, one exclusive scan
//    over (digit, tile), and a stable scatter in which each tile ranks its
//    elements by 1-bit split passes.
//  * globalRandom removes n - target particles chosen uniformly without
//    replacement (each thread throws darts at free slots with atomicOr on the
//    removal bitmask, as the reference redraws until it hits a particle it has
//    not removed), or appends target - n copies of particles drawn with
//    replacement; weights are scaled by n/target in both cases.
//  * localRandom keeps the reference's bookkeeping (weight thresholds, split
//    and merge counts, typical velocity, phase-space metric with
//    lambda = ds / v_typical) but replaces the sequential kd-tree search by
//    binning: the merge candidates (the lightest particles) are ordered along
//    a 5-D Morton curve of (x, y, lambda v) and neighbours in that order are
//    merged when their phase-space distance passes the reference's test.
#include <math.h>
#include <stdint.h>

#include "oec_common.cuh"
#include "specfun.cuh"

namespace oec {
namespace {

constexpr int kSortThreads = 256;                      // threads per sort CTA (8 warps)
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kPerLane = 16;                            // keys per thread
constexpr int kTile = kSortThreads * kPerLane;          // keys per sort tile (one CTA): 4096
constexpr int kWarpKeys = 32 * kPerLane;                // a warp's consecutive keys in the tile

__device__ __forceinline__ int blk_scan(int v, int *tot, int *sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(kFullMask, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int s = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(kFullMask, s, o);
            if (lane >= o) s += y;
        }
        sh[lane] = s;
    }
    __syncthreads();
    int ex = (wid > 0 ? sh[wid - 1] : 0) + x - v;
    if (tot) *tot = sh[(blockDim.x >> 5) - 1];
    __syncthreads();
    return ex;
}

// ----------------------------------------------------------- radix sort

// Digit counts of one tile (kTile keys): per-warp counters in shared memory
// (fewer same-address conflicts), summed per digit at the end; written
// digit-major, hist[d * ntiles + tile].
__global__ void __launch_bounds__(kSortThreads) k_digit_hist(const uint32_t *__restrict__ keys, const int32_t *n_p,
                                                             int shift, int ntiles, int *__restrict__ hist) {
    __shared__ int h[kSortWarps][256];
    const int n = *n_p;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int d = threadIdx.x; d < kSortWarps * 256; d += kSortThreads) (&h[0][0])[d] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kTile + w * kWarpKeys + lane;
#pragma unroll 4
    for (int r = 0; r < kPerLane; ++r) {
        const int64_t i = base + r * 32;
        if (i < n) atomicAdd(&h[w][(keys[i] >> shift) & 255u], 1);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += kSortThreads) {
        int c = 0;
#pragma unroll
        for (int k = 0; k < kSortWarps; ++k) c += h[k][d];
        hist[d * ntiles + blockIdx.x] = c;
    }
}

// exclusive scan of `len` ints in one CTA (len <= 1024 * chunks)
__global__ void k_scan_serial_chunks(int *a, int len) {
    __shared__ int sh[32];
    int carry = 0;
    for (int base = 0; base < len; base += blockDim.x) {
        int i = base + threadIdx.x;
        int v = i < len ? a[i] : 0;
        int tot;
        int ex = blk_scan(v, &tot, sh);
        if (i < len) a[i] = ex + carry;
        carry += tot;
        __syncthreads();
    }
}

// Exclusive scan of a[0, len) in place by 1024-element blocks (each block's
// total to partial[block]), then the scan of the block totals, then the add:
// the digit histograms of a large sort are millions of entries long.
__global__ void k_scan_tiles(int *a, int len, int *partial) {
    __shared__ int sh[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = i < len ? a[i] : 0;
    int tot;
    const int ex = blk_scan(v, &tot, sh);
    if (i < len) a[i] = ex;
    if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

__global__ void k_scan_add_tiles(int *a, int len, const int *partial) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < len) a[i] += partial[blockIdx.x];
}

// Stable scatter of one tile (kTile keys) by the digit at `shift`.  Warp w
// owns the tile's keys w*512 .. w*512+511 and walks them in 16 rounds of 32
// consecutive keys (coalesced loads); a key's place among the equal digits
// of its warp is the warp's running count of that digit (shared memory, one
// counter row per warp) plus the lanes below it in the round with the same
// digit (a warp match).  After the rounds the counts of the lower warps give
// each warp's start inside the tile's run of a digit, and the scanned tile
// histogram the run's start in the output, so the order is (digit, tile,
// warp, round, lane) = stable.
__global__ void __launch_bounds__(kSortThreads) k_scatter(const uint32_t *__restrict__ keys,
                                                          const int32_t *__restrict__ vals, const int32_t *n_p,
                                                          int shift, int ntiles, const int *__restrict__ offs,
                                                          uint32_t *__restrict__ okeys, int32_t *__restrict__ ovals) {
    __shared__ int cnt[kSortWarps][256];  // running digit counts, then each warp's start in a digit's run
    const int n = *n_p;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    for (int e = threadIdx.x; e < kSortWarps * 256; e += kSortThreads) (&cnt[0][0])[e] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kTile + w * kWarpKeys + lane;
    uint32_t k[kPerLane];
    int32_t v[kPerLane];
    int dr[kPerLane];  // digit << 16 | rank among the warp's equal digits, -1: no key
#pragma unroll
    for (int r = 0; r < kPerLane; ++r) {
        const int64_t i = base + r * 32;
        const bool valid = i < n;
        k[r] = valid ? keys[i] : 0u;
        v[r] = valid ? vals[i] : 0;
    }
#pragma unroll
    for (int r = 0; r < kPerLane; ++r) {
        const bool valid = base + r * 32 < n;
        const int d = valid ? (int)((k[r] >> shift) & 255u) : 256;
        const unsigned peers = __match_any_sync(kFullMask, d);
        int rank = 0;
        if (valid) rank = cnt[w][d] + __popc(peers & below);
        __syncwarp();
        if (valid && (peers & below) == 0) cnt[w][d] += __popc(peers);
        __syncwarp();
        dr[r] = valid ? (d << 16 | rank) : -1;
    }
    __syncthreads();
    // each warp's start inside the tile's run of digit d: the counts of the lower warps
    for (int d = threadIdx.x; d < 256; d += kSortThreads) {
        int run = 0;
#pragma unroll
        for (int q = 0; q < kSortWarps; ++q) {
            const int c = cnt[q][d];
            cnt[q][d] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kPerLane; ++r) {
        if (dr[r] < 0) continue;
        const int d = dr[r] >> 16, rank = dr[r] & 0xffff;
        const int dst = offs[d * ntiles + blockIdx.x] + cnt[w][d] + rank;
        okeys[dst] = k[r];
        ovals[dst] = v[r];
    }
}

// float -> order-preserving uint32
__device__ __forceinline__ uint32_t float_key(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void k_make_keys(oec_particles_t p, int column, uint32_t *__restrict__ keys, int32_t *__restrict__ vals) {
    int n = *p.count;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t k;
        switch (column) {
            case 6: k = (uint32_t)p.cell[i]; break;  // cell order
            case 2: k = float_key(p.vx[i]); break;
            case 3: k = float_key(p.vy[i]); break;
            case 4: k = float_key(p.vz[i]); break;
            case 5: k = float_key(p.w[i]); break;
            default: k = (uint32_t)p.cell[i]; break;
        }
        keys[i] = k;
        vals[i] = i;
    }
}

// gather every SoA array through the permutation into `q`
__global__ void k_permute(oec_particles_t p, const int32_t *__restrict__ perm, oec_particles_t q) {
    int n = *p.count;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int s = perm[i];
        q.cell[i] = p.cell[s];
        q.ox[i] = p.ox[s];
        q.oy[i] = p.oy[s];
        q.vx[i] = p.vx[s];
        q.vy[i] = p.vy[s];
        q.vz[i] = p.vz[s];
        q.w[i] = p.w[s];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *q.count = n;
}

// ------------------------------------------------------- weight search
// _searchSorted (particleManagement.pyx:244-262) on the weight-sorted store,
// one thread per threshold, the reference's loop as written (it answers 0 as
// soon as a[0] >= value): the first index with a[i] > value.
__global__ void k_search_sorted2(const float *__restrict__ w, const int32_t *count, double lo, double hi,
                                 int32_t *out) {
    const int t = threadIdx.x;
    if (t > 1) return;
    const double value = t == 0 ? lo : hi;
    const int n = *count;
    int r;
    if (n <= 0) {
        r = 0;
    } else if ((double)w[n - 1] <= value) {
        r = n;
    } else if ((double)w[0] >= value) {
        r = 0;
    } else {
        int i0 = 0, i2 = n - 1, i1 = (int)((i2 + i0) * 0.5);
        while (i1 != i0) {
            if ((double)w[i1] > value)
                i2 = i1;
            else
                i0 = i1;
            i1 = (int)((i2 + i0) * 0.5);
        }
        r = i1 + 1;
    }
    out[t] = r;
}

// -------------------------------------------------------------- roulette

__global__ void k_scale_w(oec_particles_t p, double factor) {
    int n = *p.count;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        p.w[i] = (float)((double)p.w[i] * factor);
}

__global__ void k_zero_words(uint32_t *m, int nwords) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nwords; i += gridDim.x * blockDim.x) m[i] = 0u;
}

// Mark `k` distinct uniformly chosen indices in [0, n) in `mask`.
__global__ void k_darts(int n, int k, uint32_t *mask, uint2 key, uint32_t call, int max_tries, int *fails) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < k; t += gridDim.x * blockDim.x) {
        bool done = false;
        for (int a = 0; a < max_tries && !done; ++a) {
            uint4 r = sf::philox4x32_10(make_uint4((uint32_t)t, call, (uint32_t)a, 0x7011u), key);
            uint32_t idx = (uint32_t)(((uint64_t)r.x * (uint64_t)n) >> 32);
            uint32_t bit = 1u << (idx & 31);
            uint32_t old = atomicOr(&mask[idx >> 5], bit);
            done = (old & bit) == 0u;
        }
        if (!done) atomicAdd(fails, 1);
    }
}

// mask = ~mask on [0, n)
__global__ void k_invert_valid(uint32_t *mask, int n) {
    int nw = (n + 31) >> 5;
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += gridDim.x * blockDim.x) {
        uint32_t valid = (w * 32 + 32 <= n) ? 0xffffffffu : ((1u << (n - w * 32)) - 1u);
        mask[w] = (~mask[w]) & valid;
    }
}

// rows of particles drawn with replacement (clone step of globalRandom)
__global__ void k_clone_rows(oec_particles_t p, int n, int k, uint2 key, uint32_t call, int nx, float inv_nx,
                             double dx, double dy, double lxh, double lyh, double *rows) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < k; t += gridDim.x * blockDim.x) {
        uint4 r = sf::philox4x32_10(make_uint4((uint32_t)t, call, 0u, 0xc10eu), key);
        int s = (int)(((uint64_t)r.x * (uint64_t)n) >> 32);
        int ix, iy;
        split_cell(p.cell[s], nx, inv_nx, ix, iy);
        double *q = rows + 6 * (int64_t)t;
        q[0] = abs_coord(ix, p.ox[s], dx, lxh);
        q[1] = abs_coord(iy, p.oy[s], dy, lyh);
        q[2] = p.vx[s];
        q[3] = p.vy[s];
        q[4] = p.vz[s];
        q[5] = p.w[s];
    }
}

// ------------------------------------------------------------ local merge

// Stats over particles [0, n): sum w, sum |v|^2 w^2 (f64, atomics).
__global__ void k_wstats(oec_particles_t p, double *acc) {
    int n = *p.count;
    double sw = 0, sv = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double w = p.w[i], vx = p.vx[i], vy = p.vy[i], vz = p.vz[i];
        sw += w;
        sv += (vx * vx + vy * vy + vz * vz) * w * w;
    }
    for (int o = 16; o > 0; o >>= 1) {
        sw += __shfl_xor_sync(kFullMask, sw, o);
        sv += __shfl_xor_sync(kFullMask, sv, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&acc[0], sw);
        atomicAdd(&acc[1], sv);
    }
}

struct MergeArgs {
    oec_particles_t p;         // weight-sorted store
    int n_cand;                // merge candidates: the lightest n_cand particles
    int n_merge_target;        // merges wanted
    const int32_t *order;      // candidates ordered by (cell, velocity key)
    double lam2;               // (ds / v_typical)^2 * lambda_factor^2
    double limit;              // factorDisLimit * ds (compared with the squared distance, as the reference)
    double dx, dy;
    int nx;
    float inv_nx;
    uint2 key;
    uint32_t call;
    int scheme;
    uint32_t *mask;            // removal bits
    int *counters;             // [0] qualifying pairs, [1] merges done
};

// Pair (2k, 2k+1) of the ordered candidates: qualifies when the weighted
// phase-space distance passes the reference's test.
__global__ void k_pair_count(MergeArgs a) {
    int npairs = a.n_cand / 2;
    int q = 0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < npairs; k += gridDim.x * blockDim.x) {
        int i = a.order[2 * k], j = a.order[2 * k + 1];
        int ix, iy, jx, jy;
        split_cell(a.p.cell[i], a.nx, a.inv_nx, ix, iy);
        split_cell(a.p.cell[j], a.nx, a.inv_nx, jx, jy);
        double ddx = ((double)(ix - jx) + ((double)a.p.ox[i] - a.p.ox[j])) * a.dx;
        double ddy = ((double)(iy - jy) + ((double)a.p.oy[i] - a.p.oy[j])) * a.dy;
        double dvx = (double)a.p.vx[i] - a.p.vx[j], dvy = (double)a.p.vy[i] - a.p.vy[j],
               dvz = (double)a.p.vz[i] - a.p.vz[j];
        double d2 = ddx * ddx + ddy * ddy + a.lam2 * (dvx * dvx + dvy * dvy + dvz * dvz);
        if (d2 < a.limit) ++q;
    }
    for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(kFullMask, q, o);
    if ((threadIdx.x & 31) == 0 && q) atomicAdd(&a.counters[0], q);
}

__global__ void k_pair_merge(MergeArgs a) {
    int npairs = a.n_cand / 2;
    int qual = a.counters[0];
    double paccept = qual > 0 ? fmin(1.0, (double)a.n_merge_target / (double)qual) : 0.0;
    int done = 0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < npairs; k += gridDim.x * blockDim.x) {
        int i = a.order[2 * k], j = a.order[2 * k + 1];
        int ix, iy, jx, jy;
        split_cell(a.p.cell[i], a.nx, a.inv_nx, ix, iy);
        split_cell(a.p.cell[j], a.nx, a.inv_nx, jx, jy);
        double ddx = ((double)(ix - jx) + ((double)a.p.ox[i] - a.p.ox[j])) * a.dx;
        double ddy = ((double)(iy - jy) + ((double)a.p.oy[i] - a.p.oy[j])) * a.dy;
        double dvx = (double)a.p.vx[i] - a.p.vx[j], dvy = (double)a.p.vy[i] - a.p.vy[j],
               dvz = (double)a.p.vz[i] - a.p.vz[j];
        double d2 = ddx * ddx + ddy * ddy + a.lam2 * (dvx * dvx + dvy * dvy + dvz * dvz);
        if (!(d2 < a.limit)) continue;
        uint4 r = sf::philox4x32_10(make_uint4((uint32_t)k, a.call, 0u, 0x3e59u), a.key);
        double u0 = r.x * (1.0 / 4294967296.0), u1 = r.y * (1.0 / 4294967296.0);
        if (u0 >= paccept) continue;
        double wi = a.p.w[i], wj = a.p.w[j];
        int keep = (u1 < wi / (wi + wj)) ? i : j;  // keep with probability proportional to weight
        int drop = keep == i ? j : i;
        if (a.scheme == 1) {
            // scale the kept velocity to conserve kinetic energy (particleManagement.pyx:200-236)
            double wk = a.p.w[keep], wd = a.p.w[drop];
            double vk2 = (double)a.p.vx[keep] * a.p.vx[keep] + (double)a.p.vy[keep] * a.p.vy[keep] +
                         (double)a.p.vz[keep] * a.p.vz[keep];
            double vd2 = (double)a.p.vx[drop] * a.p.vx[drop] + (double)a.p.vy[drop] * a.p.vy[drop] +
                         (double)a.p.vz[drop] * a.p.vz[drop];
            double f = vk2 > 0 ? wk / (wk + wd) + vd2 / vk2 * wd / (wk + wd) : 1.0;
            a.p.vx[keep] = (float)(a.p.vx[keep] * f);
            a.p.vy[keep] = (float)(a.p.vy[keep] * f);
            a.p.vz[keep] = (float)(a.p.vz[keep] * f);
        }
        a.p.w[keep] = (float)(wi + wj);
        atomicOr(&a.mask[drop >> 5], 1u << (drop & 31));
        ++done;
    }
    for (int o = 16; o > 0; o >>= 1) done += __shfl_xor_sync(kFullMask, done, o);
    if ((threadIdx.x & 31) == 0 && done) atomicAdd(&a.counters[1], done);
}

// Weighted phase-space coordinates of the merge metric (localRandom :166-171):
// (x, y, lambda vx, lambda vy, lambda vz), positions relative to the grid corner.
__device__ __forceinline__ void phase5(const oec_particles_t &p, int i, int nx, float inv_nx, double dx, double dy,
                                       double lam, float c[5]) {
    int ix, iy;
    split_cell(p.cell[i], nx, inv_nx, ix, iy);
    c[0] = (float)(((double)ix + p.ox[i]) * dx);
    c[1] = (float)(((double)iy + p.oy[i]) * dy);
    c[2] = (float)(lam * p.vx[i]);
    c[3] = (float)(lam * p.vy[i]);
    c[4] = (float)(lam * p.vz[i]);
}

// Bounding box of the candidates' weighted coordinates (order-preserving
// float keys, atomic min / max): bbox[0..4] minima, bbox[5..9] maxima.
__global__ void k_cand_bbox(oec_particles_t p, int n_cand, int nx, float inv_nx, double dx, double dy, double lam,
                            uint32_t *bbox) {
    uint32_t mn[5], mx[5];
    for (int d = 0; d < 5; ++d) {
        mn[d] = 0xffffffffu;
        mx[d] = 0u;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_cand; i += gridDim.x * blockDim.x) {
        float c[5];
        phase5(p, i, nx, inv_nx, dx, dy, lam, c);
        for (int d = 0; d < 5; ++d) {
            uint32_t k = float_key(c[d]);
            mn[d] = min(mn[d], k);
            mx[d] = max(mx[d], k);
        }
    }
    for (int d = 0; d < 5; ++d) {
        for (int o = 16; o > 0; o >>= 1) {
            mn[d] = min(mn[d], __shfl_xor_sync(kFullMask, mn[d], o));
            mx[d] = max(mx[d], __shfl_xor_sync(kFullMask, mx[d], o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&bbox[d], mn[d]);
            atomicMax(&bbox[5 + d], mx[d]);
        }
    }
}

__device__ __forceinline__ float key_float(uint32_t k) {
    uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    return __uint_as_float(u);
}

// Candidate keys: 5-D Morton order (6 bits per axis, one common scale for all
// axes so that the order follows the isotropic weighted metric): neighbours in
// key order are close in (x, y, lambda v).
__global__ void k_cand_keys(oec_particles_t p, int n_cand, int nx, float inv_nx, double dx, double dy, double lam,
                            const uint32_t *bbox, uint32_t *keys, int32_t *vals) {
    float lo[5], span = 0.f;
    for (int d = 0; d < 5; ++d) {
        lo[d] = key_float(bbox[d]);
        span = fmaxf(span, key_float(bbox[5 + d]) - lo[d]);
    }
    float inv = span > 0.f ? 64.0f / span : 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_cand; i += gridDim.x * blockDim.x) {
        float c[5];
        phase5(p, i, nx, inv_nx, dx, dy, lam, c);
        uint32_t q[5];
        for (int d = 0; d < 5; ++d) q[d] = (uint32_t)fminf(fmaxf((c[d] - lo[d]) * inv, 0.f), 63.f);
        uint32_t key = 0;
        for (int b = 5; b >= 0; --b)
            for (int d = 0; d < 5; ++d) key = (key << 1) | ((q[d] >> b) & 1u);
        keys[i] = key;
        vals[i] = i;
    }
}

// rows: duplicates at half weight of the heaviest `k` (the last k in weight order)
__global__ void k_split_rows(oec_particles_t p, int n, int k, int nx, float inv_nx, double dx, double dy, double lxh,
                             double lyh, double *rows) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < k; t += gridDim.x * blockDim.x) {
        int s = n - k + t;
        p.w[s] = p.w[s] * 0.5f;
        int ix, iy;
        split_cell(p.cell[s], nx, inv_nx, ix, iy);
        double *q = rows + 6 * (int64_t)t;
        q[0] = abs_coord(ix, p.ox[s], dx, lxh);
        q[1] = abs_coord(iy, p.oy[s], dy, lyh);
        q[2] = p.vx[s];
        q[3] = p.vy[s];
        q[4] = p.vz[s];
        q[5] = p.w[s];
    }
}

}  // namespace
}  // namespace oec

using namespace oec;

static bool vp2(const oec_particles_t *p) {
    return p && p->cell && p->ox && p->oy && p->vx && p->vy && p->vz && p->w && p->count && p->capacity > 0;
}

// Blocks of the histogram scan (256 digits x tiles entries, 1024 per block).
static int64_t hist_scan_blocks(int64_t capacity) {
    const int64_t tiles = (capacity + kTile - 1) / kTile;
    return (256 * tiles + 1023) / 1024;
}

extern "C" int64_t oec_sort_work_bytes(int64_t capacity) {
    int64_t tiles = (capacity + kTile - 1) / kTile;
    // keys, vals (twice) | histogram | 256-byte slack (merge counters) | block totals
    return 4 * capacity * 4 + 256 * tiles * 4 + 256 + 4 * hist_scan_blocks(capacity) + 256;
}

// Stable radix sort of (keys, vals) pairs, keys in work; `bits` significant key bits.
static int radix_sort(uint32_t *keys, int32_t *vals, uint32_t *k2, int32_t *v2, int *hist, const int32_t *n_dev,
                      int64_t cap, int bits, cudaStream_t s, uint32_t **kout, int32_t **vout) {
    int ntiles = (int)((cap + kTile - 1) / kTile);
    const int len = 256 * ntiles, nb = (int)hist_scan_blocks(cap);
    // block totals after the histogram and its 256-byte slack
    int *partial = reinterpret_cast<int *>(reinterpret_cast<char *>(hist) + 4 * (int64_t)len + 256);
    for (int shift = 0; shift < bits; shift += 8) {
        k_digit_hist<<<ntiles, kSortThreads, 0, s>>>(keys, n_dev, shift, ntiles, hist);
        k_scan_tiles<<<nb, 1024, 0, s>>>(hist, len, partial);
        k_scan_serial_chunks<<<1, 1024, 0, s>>>(partial, nb);
        k_scan_add_tiles<<<nb, 1024, 0, s>>>(hist, len, partial);
        k_scatter<<<ntiles, kSortThreads, 0, s>>>(keys, vals, n_dev, shift, ntiles, hist, k2, v2);
        uint32_t *tk = keys;
        keys = k2;
        k2 = tk;
        int32_t *tv = vals;
        vals = v2;
        v2 = tv;
    }
    *kout = keys;
    *vout = vals;
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_sort_particles(oec_particles_t *p, oec_particles_t *tmp, int32_t column, void *work_dev,
                                  void *stream) {
    if (!vp2(p) || !vp2(tmp) || !work_dev || tmp->capacity < p->capacity) return OEC_ERR_INVALID;
    if (column < 2 || column > 6) return OEC_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    int64_t cap = p->capacity;
    uint32_t *keys = static_cast<uint32_t *>(work_dev);
    int32_t *vals = reinterpret_cast<int32_t *>(keys + cap);
    uint32_t *k2 = reinterpret_cast<uint32_t *>(vals + cap);
    int32_t *v2 = reinterpret_cast<int32_t *>(k2 + cap);
    int *hist = reinterpret_cast<int *>(v2 + cap);
    int g = persistent_grid((cap + 255) / 256, 8);
    k_make_keys<<<g, 256, 0, s>>>(*p, column, keys, vals);
    OEC_LAUNCH_CHECK();
    int bits = 32;
    if (column == 6) {
        // cell keys: only as many digits as the largest cell index needs
        bits = 24;
    }
    uint32_t *kout;
    int32_t *vout;
    int rc = radix_sort(keys, vals, k2, v2, hist, p->count, cap, bits, s, &kout, &vout);
    if (rc != OEC_OK) return rc;
    k_permute<<<g, 256, 0, s>>>(*p, vout, *tmp);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_weight_thresholds(const oec_particles_t *p, double lo, double hi, int32_t *out_dev,
                                     void *stream) {
    if (!vp2(p) || !out_dev) return OEC_ERR_INVALID;
    k_search_sorted2<<<1, 32, 0, as_stream(stream)>>>(p->w, p->count, lo, hi, out_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_scale_weights(oec_particles_t *p, double factor, void *stream) {
    if (!vp2(p)) return OEC_ERR_INVALID;
    k_scale_w<<<persistent_grid((p->capacity + 255) / 256, 8), 256, 0, as_stream(stream)>>>(*p, factor);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_roulette_select(int32_t n, int32_t n_remove, uint32_t *mask_dev, int64_t mask_words,
                                   uint64_t seed, uint32_t call, int32_t *fails_dev, void *stream) {
    if (n < 0 || n_remove < 0 || n_remove > n || !mask_dev || !fails_dev || mask_words * 32 < n)
        return OEC_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
    int nw = (n + 31) / 32;
    k_zero_words<<<persistent_grid((mask_words + 255) / 256, 8), 256, 0, s>>>(mask_dev, (int)mask_words);
    OEC_CUDA_TRY(cudaMemsetAsync(fails_dev, 0, sizeof(int32_t), s));
    // choose the smaller of the removed and the kept sets by darts
    bool invert = n_remove > n / 2;
    int k = invert ? n - n_remove : n_remove;
    if (k > 0)
        k_darts<<<persistent_grid((k + 255) / 256, 8), 256, 0, s>>>(n, k, mask_dev, key, call, 4096, fails_dev);
    if (invert) k_invert_valid<<<persistent_grid((nw + 255) / 256, 8), 256, 0, s>>>(mask_dev, n);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_clone_rows(const oec_grid_t *grid, const oec_particles_t *p, int32_t n, int32_t k, uint64_t seed,
                              uint32_t call, double *rows_dev, void *stream) {
    if (!grid || !vp2(p) || n <= 0 || k < 0 || !rows_dev) return OEC_ERR_INVALID;
    GridConst gc = make_grid_const(*grid);
    uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
    if (k > 0)
        k_clone_rows<<<persistent_grid((k + 255) / 256, 8), 256, 0, as_stream(stream)>>>(
            *p, n, k, key, call, gc.nx, 1.0f / (float)gc.nx, gc.dx, gc.dy, gc.lxh, gc.lyh, rows_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_weight_stats(const oec_particles_t *p, double *acc_dev, void *stream) {
    if (!vp2(p) || !acc_dev) return OEC_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    OEC_CUDA_TRY(cudaMemsetAsync(acc_dev, 0, 2 * sizeof(double), s));
    k_wstats<<<persistent_grid((p->capacity + 255) / 256, 4), 256, 0, s>>>(*p, acc_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_split_rows(const oec_grid_t *grid, oec_particles_t *p, int32_t n, int32_t k, double *rows_dev,
                              void *stream) {
    if (!grid || !vp2(p) || k < 0 || k > n || (k > 0 && !rows_dev)) return OEC_ERR_INVALID;
    GridConst gc = make_grid_const(*grid);
    if (k > 0)
        k_split_rows<<<persistent_grid((k + 255) / 256, 8), 256, 0, as_stream(stream)>>>(
            *p, n, k, gc.nx, 1.0f / (float)gc.nx, gc.dx, gc.dy, gc.lxh, gc.lyh, rows_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_cell_merge(const oec_grid_t *grid, oec_particles_t *p, int32_t n_cand, int32_t n_merge,
                              double lambda, double limit, int32_t scheme, uint64_t seed, uint32_t call,
                              double vscale, uint32_t *mask_dev, int32_t *counters_dev, void *work_dev,
                              void *stream) {
    if (!grid || !vp2(p) || n_cand < 0 || n_cand > p->capacity || n_merge < 0 || !mask_dev || !counters_dev ||
        !work_dev)
        return OEC_ERR_INVALID;
    GridConst gc = make_grid_const(*grid);
    (void)vscale;
    cudaStream_t s = as_stream(stream);
    int64_t cap = p->capacity;
    uint32_t *keys = static_cast<uint32_t *>(work_dev);
    int32_t *vals = reinterpret_cast<int32_t *>(keys + cap);
    uint32_t *k2 = reinterpret_cast<uint32_t *>(vals + cap);
    int32_t *v2 = reinterpret_cast<int32_t *>(k2 + cap);
    int *hist = reinterpret_cast<int *>(v2 + cap);
    int32_t *ncand_dev = reinterpret_cast<int32_t *>(hist + 256 * ((cap + kTile - 1) / kTile));
    uint32_t *bbox = reinterpret_cast<uint32_t *>(ncand_dev + 1);  // 10 words (inside the 256-byte slack)
    uint32_t init[10] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u, 0u, 0u};
    OEC_CUDA_TRY(cudaMemcpyAsync(ncand_dev, &n_cand, sizeof(int32_t), cudaMemcpyHostToDevice, s));
    OEC_CUDA_TRY(cudaMemcpyAsync(bbox, init, sizeof(init), cudaMemcpyHostToDevice, s));
    OEC_CUDA_TRY(cudaMemsetAsync(counters_dev, 0, 2 * sizeof(int32_t), s));
    int g = persistent_grid((n_cand + 255) / 256 + 1, 8);
    k_cand_bbox<<<g, 256, 0, s>>>(*p, n_cand, gc.nx, 1.0f / (float)gc.nx, gc.dx, gc.dy, lambda, bbox);
    k_cand_keys<<<g, 256, 0, s>>>(*p, n_cand, gc.nx, 1.0f / (float)gc.nx, gc.dx, gc.dy, lambda, bbox, keys, vals);
    uint32_t *kout;
    int32_t *vout;
    int rc = radix_sort(keys, vals, k2, v2, hist, ncand_dev, cap, 32, s, &kout, &vout);
    if (rc != OEC_OK) return rc;
    MergeArgs a{};
    a.p = *p;
    a.n_cand = n_cand;
    a.n_merge_target = n_merge;
    a.order = vout;
    a.lam2 = lambda * lambda;
    a.limit = limit;
    a.dx = gc.dx;
    a.dy = gc.dy;
    a.nx = gc.nx;
    a.inv_nx = 1.0f / (float)gc.nx;
    a.key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
    a.call = call;
    a.scheme = scheme;
    a.mask = mask_dev;
    a.counters = counters_dev;
    k_pair_count<<<g, 256, 0, s>>>(a);
    k_pair_merge<<<g, 256, 0, s>>>(a);
    OEC_LAUNCH_CHECK();
    OEC_CUDA_TRY(cudaStreamSynchronize(s));  // n_cand lives on this stack frame
    return OEC_OK;
}
