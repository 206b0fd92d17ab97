// boundary.cu -- absorbed particles, wall intersection and wall normals,
// and the removal/insertion of particles in the reference's slot order.
//
// Reference: particleBoundary.pyx (saveAbsorbed :38-65, AbsorbRectangular
// :99-221, AbsorbElliptical :252-297, AbsorbArbitraryCutCell :373-481) and
// particles.pyx addAndRemoveParticles (:94-121, :201-269).
//
// The absorbed set arrives as one bit per particle (from the fused push
// kernel or oec_index_inside).  A three-kernel scan turns the bits into the
// ascending list of absorbed indices, so the set, its order and everything
// derived from it is deterministic.  Wall geometry is evaluated in FP64 on
// the FP32 state widened exactly to FP64.
#include <math.h>
#include <stdint.h>

#include "oec_common.cuh"

namespace oec {
namespace {

constexpr int kScanThreads = 1024;            // words per scan block
constexpr int kMaxScanBlocks = 1024;          // -> up to 2^25 particles

__device__ __forceinline__ int block_excl_scan(int v, int *tot, int *sh) {
    // sh: >= 32 ints.  Exclusive scan over the CTA (blockDim multiple of 32).
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
        int nw = blockDim.x >> 5;
        int s = lane < nw ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(kFullMask, s, o);
            if (lane >= o) s += y;
        }
        sh[lane] = s;
    }
    __syncthreads();
    int before = (wid > 0 ? sh[wid - 1] : 0) + x - v;
    if (tot) *tot = sh[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before;
}

__device__ __forceinline__ uint32_t valid_bits(int word, int n) {
    int base = word * 32;
    if (base + 32 <= n) return 0xffffffffu;
    if (base >= n) return 0u;
    return (1u << (n - base)) - 1u;
}

__global__ void k_mask_count(const uint32_t *__restrict__ mask, const int32_t *count, int *partial) {
    __shared__ int sh[32];
    int n = *count;
    int nwords = (n + 31) >> 5;
    int w = blockIdx.x * kScanThreads + threadIdx.x;
    int c = (w < nwords) ? __popc(mask[w] & valid_bits(w, n)) : 0;
    int tot;
    block_excl_scan(c, &tot, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

__global__ void k_partial_scan(int *partial, int nblocks, int32_t *total_out, int32_t *total_out2) {
    __shared__ int sh[32];
    int v = threadIdx.x < nblocks ? partial[threadIdx.x] : 0;
    int tot;
    int ex = block_excl_scan(v, &tot, sh);
    if (threadIdx.x < nblocks) partial[threadIdx.x] = ex;
    if (threadIdx.x == 0) {
        *total_out = tot;
        if (total_out2) *total_out2 = tot;
    }
}

__global__ void k_mask_scatter(const uint32_t *__restrict__ mask, const int32_t *count, const int *partial,
                               int32_t *__restrict__ index, int cap) {
    __shared__ int sh[32];
    int n = *count;
    int nwords = (n + 31) >> 5;
    int w = blockIdx.x * kScanThreads + threadIdx.x;
    uint32_t bits = (w < nwords) ? (mask[w] & valid_bits(w, n)) : 0u;
    int off = block_excl_scan(__popc(bits), nullptr, sh) + partial[blockIdx.x];
    while (bits) {
        int b = __ffs(bits) - 1;
        bits &= bits - 1;
        if (off < cap) index[off] = w * 32 + b;
        ++off;
    }
}

// The same index in one CTA for small stores (a few scan blocks): the words
// are taken 1024 at a time with a running carry, so the three launches above
// (count, block scan, scatter; ~3.5 us each at 1e5 particles) become one.
constexpr int kSmallScanBlocks = 8;  // up to 8 * 1024 words = 262,144 particles

__global__ void __launch_bounds__(kScanThreads)
    k_mask_index_small(const uint32_t *__restrict__ mask, const int32_t *count, int32_t *__restrict__ index,
                       int cap, int32_t *total_out, int32_t *total_out2) {
    __shared__ int sh[32];
    const int n = *count;
    const int nwords = (n + 31) >> 5;
    int carry = 0;
    for (int base = 0; base < nwords; base += kScanThreads) {  // same trip count in every thread
        const int w = base + threadIdx.x;
        uint32_t bits = (w < nwords) ? (mask[w] & valid_bits(w, n)) : 0u;
        int tot;
        int off = block_excl_scan(__popc(bits), &tot, sh) + carry;
        while (bits) {
            const int b = __ffs(bits) - 1;
            bits &= bits - 1;
            if (off < cap) index[off] = w * 32 + b;
            ++off;
        }
        carry += tot;
    }
    if (threadIdx.x == 0) {
        *total_out = carry;
        if (total_out2) *total_out2 = carry;
    }
}

// Absorbed rows in the reference layout [x, y, vx, vy, vz, w] (f64).
__global__ void k_gather_rows(oec_particles_t p, const int32_t *__restrict__ index, const int32_t *n_abs, int cap,
                              int nx, float inv_nx, double dx, double dy, double lxh, double lyh,
                              double *__restrict__ rows) {
    int na = *n_abs < cap ? *n_abs : cap;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < na; i += gridDim.x * blockDim.x) {
        int k = index[i];
        if (!OEC_IN_BOUNDS(k, *p.count)) continue;
        int ix, iy;
        split_cell(p.cell[k], nx, inv_nx, ix, iy);
        double *r = rows + 6 * (int64_t)i;
        r[0] = abs_coord(ix, p.ox[k], dx, lxh);
        r[1] = abs_coord(iy, p.oy[k], dy, lyh);
        r[2] = (double)p.vx[k];
        r[3] = (double)p.vy[k];
        r[4] = (double)p.vz[k];
        r[5] = (double)p.w[k];
    }
}

// ------------------------------------------------------------ wall geometry

struct WallConst {
    int kind;
    double dxi, dyi, lxh_ext, lyh_ext, dt;
    double rect_hx, rect_hy;             // lx/2 - 1e-6 dx, ly/2 - 1e-6 dy
    double ell_ax, ell_ay;               // 4/(lx - 1e-6 dx)^2, 4/(ly - 1e-6 dy)^2
    double ell_nx2, ell_ny2, ell_nx4, ell_ny4;  // 4/lx^2, 4/ly^2 and squares
    int nx;
    const uint16_t *faces;
    const double *bpts;
    const int32_t *cpi;
    const double *cnorm;
};

// AbsorbRectangular.calculateInteractionPoint + calculateNormalVectors.
__device__ bool wall_rect(const WallConst &c, double *r, double *nrm) {
    const double hx = c.rect_hx, hy = c.rect_hy;
    int xs = 1, ys = 1;
    if (r[0] > hx) xs = 2; else if (r[0] < -hx) xs = 0;
    if (r[1] > hy) ys = 2; else if (r[1] < -hy) ys = 0;
    double t;
    int where;
    if (ys == 1 && xs != 1) {
        t = (xs == 0) ? (r[0] + hx) / r[2] : (r[0] - hx) / r[2];
        where = (xs == 0) ? 0 : 1;
    } else if (xs == 1 && ys != 1) {
        t = (ys == 0) ? (r[1] + hy) / r[3] : (r[1] - hy) / r[3];
        where = (ys == 0) ? 2 : 3;
    } else {
        double tx = (xs == 0) ? (r[0] + hx) / r[2] : (r[0] - hx) / r[2];
        double ty = (ys == 0) ? (r[1] + hy) / r[3] : (r[1] - hy) / r[3];
        // corner labels as written in particleBoundary.pyx:163-190
        if (xs == 0 && ys == 0) where = (tx > ty) ? 0 : 1;
        else if (xs == 2 && ys == 0) where = (tx > ty) ? 2 : 1;
        else if (xs == 0 && ys == 2) where = (tx > ty) ? 0 : 3;
        else where = (tx > ty) ? 2 : 3;
        t = (tx > ty) ? tx : ty;
    }
    bool found = true;
    if (isfinite(t)) {
        r[0] = __dsub_rn(r[0], __dmul_rn(t, r[2]));
        r[1] = __dsub_rn(r[1], __dmul_rn(t, r[3]));
    } else {
        // no velocity across the crossed side (the back step divides by a
        // zero component and the reference's point is NaN): the point is
        // clamped onto the wall instead
        r[0] = fmin(fmax(r[0], -hx), hx);
        r[1] = fmin(fmax(r[1], -hy), hy);
        found = false;
    }
    nrm[0] = where == 0 ? 1. : (where == 1 ? -1. : 0.);
    nrm[1] = where == 2 ? 1. : (where == 3 ? -1. : 0.);
    return found;
}

// AbsorbElliptical.calculateInteractionPoint + calculateNormalVectors.
__device__ bool wall_ellipse(const WallConst &c, double *r, double *nrm) {
    const double ax = c.ell_ax, ay = c.ell_ay;
    double cc = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(r[0], r[0]), ax), __dmul_rn(__dmul_rn(r[1], r[1]), ay)), -1.);
    double b = __dadd_rn(__dmul_rn(__dmul_rn(r[0], r[2]), ax), __dmul_rn(__dmul_rn(r[1], r[3]), ay));
    double a = __dadd_rn(__dmul_rn(__dmul_rn(r[2], r[2]), ax), __dmul_rn(__dmul_rn(r[3], r[3]), ay));
    const double disc = __dsub_rn(__dmul_rn(b, b), __dmul_rn(a, cc));
    bool found = true;
    if (disc >= 0. && a > 0.) {
        double t = __ddiv_rn(__dsub_rn(b, __dsqrt_rn(disc)), a);
        r[0] = __dsub_rn(r[0], __dmul_rn(t, r[2]));
        r[1] = __dsub_rn(r[1], __dmul_rn(t, r[3]));
    } else {
        // the back step along the velocity misses the wall (or there is no
        // transverse velocity) and the reference's point is NaN: the point
        // is projected radially onto the wall instead
        const double s = __dsqrt_rn(__dadd_rn(cc, 1.));
        if (s > 0.) {
            r[0] = __ddiv_rn(r[0], s);
            r[1] = __ddiv_rn(r[1], s);
        }
        found = false;
    }
    const double nx2 = c.ell_nx2, ny2 = c.ell_ny2, nx4 = c.ell_nx4, ny4 = c.ell_ny4;
    double inv = __ddiv_rn(1., __dsqrt_rn(__dadd_rn(__dmul_rn(__dmul_rn(r[0], r[0]), nx4),
                                                    __dmul_rn(__dmul_rn(r[1], r[1]), ny4))));
    nrm[0] = __dmul_rn(__dmul_rn(-r[0], nx2), inv);
    nrm[1] = __dmul_rn(__dmul_rn(-r[1], ny2), inv);
    return found;
}

__device__ __forceinline__ int cell_of(const WallConst &c, double x, double y) {
    int ix = (int)((x + c.lxh_ext) * c.dxi);
    int iy = (int)((y + c.lyh_ext) * c.dyi);
    return ix + iy * c.nx;
}

// AbsorbArbitraryCutCell.calculateInteractionPoint + calculateNormalVectors:
// segment-segment intersection of the back step with the cut segments of the
// 2x2 cells around the particle.  Returns false if no intersection is found.
__device__ bool wall_cutcell(const WallConst &c, double *r, double *nrm, int G) {
    const double eps = 1.e-6;
    int cell = cell_of(c, r[0], r[1]);
    double rx = -c.dt * r[2], ry = -c.dt * r[3];
    int xd[2] = {0, rx < 0. ? -1 : 1};
    int yd[2] = {0, ry < 0. ? -1 : 1};
    bool found = false;
    for (int a = 0; a < 2 && !found; ++a) {
        for (int b = 0; b < 2; ++b) {
            int cc = cell + xd[a] + yd[b] * c.nx;
            if (cc < 0 || cc >= G) continue;
            unsigned f = c.faces[cc];
            if (f == 0 || f == 8) continue;
            int p0 = c.cpi[2 * cc], p1 = c.cpi[2 * cc + 1];
            if (p0 < 0 || p1 < 0) continue;
            double sx = c.bpts[2 * p1] - c.bpts[2 * p0];
            double sy = c.bpts[2 * p1 + 1] - c.bpts[2 * p0 + 1];
            double rxs = __dsub_rn(__dmul_rn(rx, sy), __dmul_rn(ry, sx));
            if (rxs != 0.) {
                double qx = c.bpts[2 * p0] - r[0], qy = c.bpts[2 * p0 + 1] - r[1];
                double t = __ddiv_rn(__dsub_rn(__dmul_rn(qx, sy), __dmul_rn(qy, sx)), rxs);
                double u = __ddiv_rn(__dsub_rn(__dmul_rn(qx, ry), __dmul_rn(qy, rx)), rxs);
                if (-eps <= t && t <= 1. + eps && -eps <= u && u <= 1. + eps) {
                    r[0] = __dadd_rn(r[0], __dmul_rn(__dmul_rn(t, rx), 1. + eps));
                    r[1] = __dadd_rn(r[1], __dmul_rn(__dmul_rn(t, ry), 1. + eps));
                    found = true;
                    break;
                }
            }
        }
    }
    int cn = cell_of(c, r[0], r[1]);
    if (cn >= 0 && cn < G) {
        nrm[0] = c.cnorm[2 * cn];
        nrm[1] = c.cnorm[2 * cn + 1];
    } else {
        nrm[0] = 0.;
        nrm[1] = 0.;
    }
    return found;
}

__global__ void k_wall(WallConst c, double *__restrict__ rows, const int32_t *n_abs, int cap,
                       double *__restrict__ normals, int G, oec_status_t *status) {
    const int total = *n_abs;
    int na = total < cap ? total : cap;
    // rows past the capacity were never gathered: those particles leave the
    // store without a wall point, so they emit nothing; count them
    if (blockIdx.x == 0 && threadIdx.x == 0 && total > cap) atomicAdd(&status->n_rows_dropped, total - cap);
    int missing = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < na; i += gridDim.x * blockDim.x) {
        double *r = rows + 6 * (int64_t)i;
        double *nrm = normals + 2 * (int64_t)i;
        bool found;
        if (c.kind == OEC_BOUNDARY_RECT)
            found = wall_rect(c, r, nrm);
        else if (c.kind == OEC_BOUNDARY_ELLIPSE)
            found = wall_ellipse(c, r, nrm);
        else
            found = wall_cutcell(c, r, nrm, G);
        if (!found) ++missing;
    }
    if (missing) atomicAdd(&status->n_not_found, missing);
}

// ------------------------------------------------------------- add/remove
//
// addAndRemoveParticles (particles.pyx:94-121) places the particles by one
// of four rules, chosen from the counts (N old particles, A holes = removed
// particles, S added rows, K = N - A kept, N_new = K + S):
//  * remove only (S = 0, particles.pyx:254-269): each hole below N_new, in
//    ascending order, takes the LAST kept particle not yet moved, so the
//    kept particles of the tail [N_new, N) land in descending order;
//  * a larger array (S > 0 and N_new above the row count of the reference's
//    particle array, particles.pyx:109-116, :201-219): the kept particles in
//    order, then the added rows; the array then holds int(1.1 N_new) rows;
//  * in place with S >= A (particles.pyx:224-232, :245-252): added row k
//    fills hole k, the rest are appended after N;
//  * in place with S < A (particles.pyx:224-244): added row k fills hole k
//    for k < S, then every kept particle after hole S-1 shifts down over the
//    A - S holes left, in order.
// The order matters beyond bookkeeping: the reference's Furman emission
// reads the yields of the last absorbed particle of the store for every
// single-secondary split (particleEmitter.pyx:245-246), so the same store
// order gives the same physics.  The row count of the reference's array is
// emulated in a device integer (array_len); without one the larger-array
// rule is never taken.
//
// The two shifting rules move a region [r0, N) whose kept particles land at
// r0 + rank; they go through a scratch store (gather, then scatter back),
// since destinations overlap sources.  The remove-only rule moves tail
// particles into holes below N_new, disjoint from the sources, directly.
enum ArMode : int { kArNothing = 0, kArRemove = 1, kArFillAppend = 2, kArShift = 3, kArNewArray = 4 };

__device__ __forceinline__ void copy_particle(oec_particles_t &p, int dst, int src) {
    p.cell[dst] = p.cell[src];
    p.ox[dst] = p.ox[src];
    p.oy[dst] = p.oy[src];
    p.vx[dst] = p.vx[src];
    p.vy[dst] = p.vy[src];
    p.vz[dst] = p.vz[src];
    p.w[dst] = p.w[src];
}

__device__ __forceinline__ void copy_across(oec_particles_t &d, int dst, const oec_particles_t &s, int src) {
    d.cell[dst] = s.cell[src];
    d.ox[dst] = s.ox[src];
    d.oy[dst] = s.oy[src];
    d.vx[dst] = s.vx[src];
    d.vy[dst] = s.vy[src];
    d.vz[dst] = s.vz[src];
    d.w[dst] = s.w[src];
}

// Row [x,y,vx,vy,vz,w] (f64) -> SoA slot k.
__device__ __forceinline__ void store_row(oec_particles_t &p, int k, const double *r, int nx, int ny, double dxi,
                                          double dyi, double lxh, double lyh) {
    double ux = (r[0] + lxh) * dxi, uy = (r[1] + lyh) * dyi;
    int ix = (int)fmax(fmin(floor(ux), (double)(nx - 2)), 0.0);
    int iy = (int)fmax(fmin(floor(uy), (double)(ny - 2)), 0.0);
    p.cell[k] = ix + iy * nx;
    p.ox[k] = fminf(fmaxf((float)(ux - (double)ix), 0.0f), 0x1.fffffep-1f);
    p.oy[k] = fminf(fmaxf((float)(uy - (double)iy), 0.0f), 0x1.fffffep-1f);
    p.vx[k] = (float)r[2];
    p.vy[k] = (float)r[3];
    p.vz[k] = (float)r[4];
    p.w[k] = (float)r[5];
}

struct AddArgs {
    oec_particles_t p;
    oec_particles_t tmp;       // scratch store for the shifting rules
    const int32_t *holes;      // ascending absorbed indices
    const int32_t *n_holes;
    int holes_cap;
    const double *add_rows;    // (n_add, 6)
    const int32_t *n_add;
    int add_cap;
    int32_t *array_len;        // emulated row count of the reference's array (optional)
    int nx, ny;
    double dxi, dyi, lxh, lyh;
    unsigned long long *rho;   // optional deposit of the added rows
    const double *wscale;
    oec_status_t *status;
};

// First index in the ascending holes[0, n) that is >= v.
__device__ __forceinline__ int holes_lower_bound(const int32_t *__restrict__ holes, int n, int v) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (holes[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// The rule and the region of one call, computed alike by every thread of
// every launch (the count changes only in the last launch).
struct ArPlan {
    int N, A, S, Nnew;
    int mode;
    int r0;     // start of the region whose kept particles move
    int kept;   // kept particles in [r0, N)
    int below;  // holes below r0
};

__device__ __forceinline__ ArPlan ar_plan(const AddArgs &a) {
    ArPlan q;
    q.N = *a.p.count;
    q.A = min(*a.n_holes, a.holes_cap);
    q.S = min(*a.n_add, a.add_cap);
    const int K = q.N - q.A;
    q.Nnew = K + q.S;
    q.mode = kArFillAppend;
    q.r0 = q.kept = q.below = 0;
    if (q.S == 0) {
        // the kept tail [N_new, N) holds as many particles as there are holes below N_new
        q.mode = q.A == 0 ? kArNothing : kArRemove;
        q.r0 = q.Nnew;
        q.below = holes_lower_bound(a.holes, q.A, q.Nnew);
        q.kept = q.below;
    } else if (a.array_len && q.Nnew > *a.array_len) {
        q.mode = kArNewArray;
        q.kept = K;
    } else if (q.S < q.A) {
        q.mode = kArShift;
        q.r0 = a.holes[q.S];  // the first hole left open: everything below it stays
        q.below = q.S;
        q.kept = q.N - q.r0 - (q.A - q.S);
    }
    return q;
}

// Added row k -> slot dst, with its deposit when rho is given.  Slots at or
// beyond the capacity are dropped (counted by the caller).
__device__ __forceinline__ bool place_row(AddArgs &a, int dst, int k) {
    if (dst >= a.p.capacity) return false;
    store_row(a.p, dst, a.add_rows + 6 * (int64_t)k, a.nx, a.ny, a.dxi, a.dyi, a.lxh, a.lyh);
    if (a.rho && OEC_IN_BOUNDS(a.p.cell[dst] + a.nx + 1, a.nx * a.ny)) {
        const int c = a.p.cell[dst];
        const double q = (double)llrint((double)a.p.w[dst] * *a.wscale);
        const double gx = (double)a.p.ox[dst], gy = (double)a.p.oy[dst];
        const long long v0 = llrint(q * ((1.0 - gx) * (1.0 - gy)));
        const long long v1 = llrint(q * (gx * (1.0 - gy)));
        const long long v2 = llrint(q * ((1.0 - gx) * gy));
        const long long v3 = (long long)q - v0 - v1 - v2;
        atomicAdd(a.rho + c, (unsigned long long)v0);
        atomicAdd(a.rho + c + 1, (unsigned long long)v1);
        atomicAdd(a.rho + c + a.nx, (unsigned long long)v2);
        atomicAdd(a.rho + c + a.nx + 1, (unsigned long long)v3);
    }
    return true;
}

// One launch, two loops.  First the in-place rules' added rows: row k fills
// hole k (k < A), the rest are appended after the old count (with S < A only
// holes are filled, all below r0).  Then the kept particles of the region
// [r0, N), each with its rank among them: (p - r0) minus the holes in
// [r0, p), which a CTA takes for its chunk's start from the ascending holes
// array (a binary search; the 32 warps search the starts of 32 successive
// chunk iterations at once, so the dependent loads of one search are paid
// once per 32 chunks) and within the chunk from a scan of the absorbed bits,
// so the chunks run independently.  Remove-only: rank r goes to hole
// kept-1-r (descending into ascending holes, all below N_new <= r0).
// Shifting rules: rank r goes to tmp[r].  The two loops touch disjoint
// slots (holes below r0 or slots from N on, against [r0, N)).
constexpr int kGatherThreads = 1024;  // 32 warps: one hole search per warp

__global__ void __launch_bounds__(kGatherThreads) k_place_gather(AddArgs a, const uint32_t *__restrict__ mask) {
    __shared__ int sh[32];
    __shared__ int holes_before[32];  // holes in [r0, chunk start) of 32 successive chunk iterations
    const ArPlan q = ar_plan(a);
    const int mode = q.mode, N = q.N, r0 = q.r0, kept = q.kept, below = q.below, Nnew = q.Nnew, A = q.A;
    if (mode == kArFillAppend || mode == kArShift) {
        int dropped = 0;
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < q.S; k += gridDim.x * blockDim.x) {
            const int dst = (k < A) ? a.holes[k] : N + (k - A);
            if (!place_row(a, dst, k)) ++dropped;
        }
        if (dropped) atomicAdd(&a.status->n_capacity_drop, dropped);
    }
    if (mode != kArRemove && mode != kArShift && mode != kArNewArray) return;
    if (r0 + (int)blockIdx.x * (int)blockDim.x >= N) return;  // whole CTA, before any barrier
    const int stride = gridDim.x * blockDim.x;
    int iter = 0;
    for (int c0 = r0 + blockIdx.x * blockDim.x; c0 < N; c0 += stride, ++iter) {
        if ((iter & 31) == 0 && (threadIdx.x & 31) == 0) {
            // warp w: the start of chunk iteration iter + w (rewritten only
            // after the barrier that ends iteration iter - 1)
            const int64_t cw = (int64_t)c0 + (int64_t)(threadIdx.x >> 5) * stride;
            holes_before[threadIdx.x >> 5] = cw < N ? holes_lower_bound(a.holes, A, (int)cw) - below : 0;
        }
        const int p = c0 + threadIdx.x;
        const int absorbed = p < N ? (int)((mask[p >> 5] >> (p & 31)) & 1u) : 1;
        const int before = block_excl_scan(absorbed, nullptr, sh);  // its barriers publish holes_before
        if (!absorbed) {
            const int r = (p - r0) - (holes_before[iter & 31] + before);
            if (r < kept) {
                if (mode == kArRemove) {
                    const int dst = a.holes[kept - 1 - r];
                    if (OEC_IN_BOUNDS(dst, Nnew)) copy_particle(a.p, dst, p);
                } else {
                    copy_across(a.tmp, r, a.p, p);
                }
            }
        }
        __syncthreads();  // holes_before is rewritten 32 chunk iterations later
    }
}

// Shifting rules, second half: tmp[i] -> slot r0 + i; for the larger-array
// rule the added rows follow the kept particles (slot K + k = r0 + kept + k).
__global__ void k_region_scatter(AddArgs a) {
    const ArPlan q = ar_plan(a);
    if (q.mode != kArShift && q.mode != kArNewArray) return;
    const int r0 = q.r0, kept = q.kept;
    const int items = kept + (q.mode == kArNewArray ? q.S : 0);
    int dropped = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < items; i += gridDim.x * blockDim.x) {
        if (i < kept) copy_across(a.p, r0 + i, a.tmp, i);
        else if (!place_row(a, r0 + i, i - kept)) ++dropped;
    }
    if (dropped) atomicAdd(&a.status->n_capacity_drop, dropped);
}

__global__ void k_set_count(AddArgs a) {
    const ArPlan q = ar_plan(a);
    long long nn = q.Nnew;
    if (nn > a.p.capacity) nn = a.p.capacity;
    *a.p.count = (int32_t)nn;
    // numpy.empty((<unsigned int> (newParticleCount*1.1), nCoords)): truncation
    if (q.mode == kArNewArray) *a.array_len = (int32_t)(uint32_t)((double)q.Nnew * 1.1);
}

__global__ void k_mask_from_keep(const uint16_t *__restrict__ keep, int n, uint32_t *__restrict__ mask, int nwords) {
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < nwords; w += gridDim.x * blockDim.x) {
        uint32_t bits = 0;
        for (int b = 0; b < 32; ++b) {
            int i = w * 32 + b;
            if (i < n && keep[i] == 0) bits |= 1u << b;
        }
        mask[w] = bits;
    }
}

}  // namespace

OEC_BOUND_QUERY(bound_violations_boundary)

}  // namespace oec

using namespace oec;

static bool vstore(const oec_particles_t *p) {
    return p && p->cell && p->ox && p->oy && p->vx && p->vy && p->vz && p->w && p->capacity > 0;
}

static bool vp(const oec_particles_t *p) { return vstore(p) && p->count; }

extern "C" int oec_absorbed_index(const oec_particles_t *p, const uint32_t *absorbed_mask_dev, int32_t *index_dev,
                                  int32_t index_cap, int32_t *n_abs_dev, int32_t *scratch_dev,
                                  oec_status_t *status_dev, void *stream) {
    if (!vp(p) || !absorbed_mask_dev || !index_dev || !n_abs_dev || !scratch_dev || index_cap < 0)
        return OEC_ERR_INVALID;
    int64_t nwords = (p->capacity + 31) / 32;
    int nblocks = (int)((nwords + kScanThreads - 1) / kScanThreads);
    if (nblocks > kMaxScanBlocks) return OEC_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    if (nblocks <= kSmallScanBlocks) {
        k_mask_index_small<<<1, kScanThreads, 0, s>>>(absorbed_mask_dev, p->count, index_dev, index_cap, n_abs_dev,
                                                      status_dev ? &status_dev->n_absorbed : nullptr);
        OEC_LAUNCH_CHECK();
        return OEC_OK;
    }
    k_mask_count<<<nblocks, kScanThreads, 0, s>>>(absorbed_mask_dev, p->count, scratch_dev);
    k_partial_scan<<<1, kMaxScanBlocks, 0, s>>>(scratch_dev, nblocks, n_abs_dev,
                                                status_dev ? &status_dev->n_absorbed : nullptr);
    k_mask_scatter<<<nblocks, kScanThreads, 0, s>>>(absorbed_mask_dev, p->count, scratch_dev, index_dev, index_cap);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_save_absorbed(const oec_grid_t *grid, const oec_particles_t *p, const int32_t *index_dev,
                                 const int32_t *n_abs_dev, int32_t cap, double *rows_dev, void *stream) {
    if (!grid || !vp(p) || !index_dev || !n_abs_dev || !rows_dev || cap < 0) return OEC_ERR_INVALID;
    GridConst gc = make_grid_const(*grid);
    k_gather_rows<<<persistent_grid((cap + 255) / 256, 4), 256, 0, as_stream(stream)>>>(
        *p, index_dev, n_abs_dev, cap, gc.nx, 1.0f / (float)gc.nx, gc.dx, gc.dy, gc.lxh, gc.lyh, rows_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_wall_interaction(const oec_grid_t *grid, const oec_boundary_t *boundary, double dt,
                                    double *rows_dev, const int32_t *n_abs_dev, int32_t cap, double *normals_dev,
                                    oec_status_t *status_dev, void *stream) {
    if (!grid || !boundary || !rows_dev || !n_abs_dev || !normals_dev || !status_dev || cap < 0)
        return OEC_ERR_INVALID;
    GridConst gc = make_grid_const(*grid);
    WallConst c{};
    c.kind = boundary->kind;
    // host FP64 constants, computed as particleBoundary.pyx computes them
    const double eps = 1e-6;
    c.dxi = gc.dxi; c.dyi = gc.dyi;
    c.lxh_ext = gc.lxh; c.lyh_ext = gc.lyh; c.dt = dt; c.nx = gc.nx;
    c.rect_hx = gc.lx * 0.5 - gc.dx * eps;
    c.rect_hy = gc.ly * 0.5 - gc.dy * eps;
    c.ell_ax = 4. / pow(gc.lx - eps * gc.dx, 2);
    c.ell_ay = 4. / pow(gc.ly - eps * gc.dy, 2);
    c.ell_nx2 = 4. / (gc.lx * gc.lx);
    c.ell_ny2 = 4. / (gc.ly * gc.ly);
    c.ell_nx4 = c.ell_nx2 * c.ell_nx2;
    c.ell_ny4 = c.ell_ny2 * c.ell_ny2;
    if (c.kind == OEC_BOUNDARY_CUTCELL) {
        if (!boundary->inside_faces_dev || !boundary->boundary_points_dev || !boundary->cut_cell_points_ind_dev ||
            !boundary->cut_cell_normals_dev)
            return OEC_ERR_INVALID;
        c.faces = boundary->inside_faces_dev;
        c.bpts = boundary->boundary_points_dev;
        c.cpi = boundary->cut_cell_points_ind_dev;
        c.cnorm = boundary->cut_cell_normals_dev;
    } else if (c.kind != OEC_BOUNDARY_RECT && c.kind != OEC_BOUNDARY_ELLIPSE) {
        return OEC_ERR_INVALID;
    }
    k_wall<<<persistent_grid((cap + 127) / 128, 4), 128, 0, as_stream(stream)>>>(c, rows_dev, n_abs_dev, cap,
                                                                                  normals_dev, gc.G, status_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_add_remove(const oec_grid_t *grid, oec_particles_t *p, oec_particles_t *tmp,
                              const uint32_t *absorbed_mask_dev, const int32_t *holes_dev, const int32_t *n_holes_dev,
                              int32_t holes_cap, const double *add_rows_dev, const int32_t *n_add_dev, int32_t add_cap,
                              int32_t *array_len_dev, int64_t *rho_fix_dev, const double *wscale_dev,
                              oec_status_t *status_dev, void *stream) {
    if (!grid || !vp(p) || !vstore(tmp) || tmp->capacity < p->capacity || !absorbed_mask_dev || !holes_dev ||
        !n_holes_dev || !n_add_dev || !status_dev || holes_cap < 0 || add_cap < 0 ||
        (add_cap > 0 && !add_rows_dev))
        return OEC_ERR_INVALID;
    if (rho_fix_dev && !wscale_dev) return OEC_ERR_INVALID;
    GridConst gc = make_grid_const(*grid);
    AddArgs a{};
    a.p = *p;
    a.tmp = *tmp;
    a.holes = holes_dev;
    a.n_holes = n_holes_dev;
    a.holes_cap = holes_cap;
    a.add_rows = add_rows_dev;
    a.n_add = n_add_dev;
    a.add_cap = add_cap;
    a.array_len = array_len_dev;
    a.nx = gc.nx; a.ny = gc.ny;
    a.dxi = gc.dxi; a.dyi = gc.dyi; a.lxh = gc.lxh; a.lyh = gc.lyh;
    a.rho = reinterpret_cast<unsigned long long *>(rho_fix_dev);
    a.wscale = wscale_dev;
    a.status = status_dev;
    cudaStream_t s = as_stream(stream);
    const int64_t cap = p->capacity;
    const int64_t span = cap > (int64_t)add_cap ? cap : (int64_t)add_cap;
    k_place_gather<<<persistent_grid((span + kGatherThreads - 1) / kGatherThreads, 2), kGatherThreads, 0, s>>>(
        a, absorbed_mask_dev);
    k_region_scatter<<<persistent_grid((cap + add_cap + 255) / 256, 4), 256, 0, s>>>(a);
    k_set_count<<<1, 1, 0, s>>>(a);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_mask_from_keep(const uint16_t *keep_dev, int64_t n, uint32_t *mask_dev, int64_t mask_words,
                                  void *stream) {
    if (!keep_dev || !mask_dev || n < 0 || mask_words * 32 < n) return OEC_ERR_INVALID;
    k_mask_from_keep<<<persistent_grid((mask_words + 255) / 256, 4), 256, 0, as_stream(stream)>>>(
        keep_dev, (int)n, mask_dev, (int)mask_words);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}
