// particles.cu -- particle store conversions, CIC weights, field gather,
// Boris push and the fused gather+push+inside-test+deposit hot kernel.
//
// Reference: particles.pyx (openECLOUD).  Layout and precision choices:
//  * particles are SoA FP32 with the position held as (cell index, in-cell
//    offset); the offset keeps ~6e-8 cell resolution anywhere on the grid,
//    where an absolute FP32 coordinate would keep only ~2e-5 cell on a
//    512-cell grid;
//  * field tables are cell-centric float4 corner quadruples so one gather is
//    two (E) or three (B) 16-byte loads;
//  * the deposit is an int64 fixed-point sum, so the grid is independent of
//    particle order and the total charge is conserved exactly.
#include <math.h>
#include <stdlib.h>

#include <mutex>

#include "oec_common.cuh"

namespace oec {

int sm_count() {
    static std::atomic<int> cached[kMaxDevices];
    return per_device_cached(cached, [] {
        int dev = 0, n = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) return 148;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 148;
        return n > 0 ? n : 148;
    });
}

bool pdl_enabled() {
    static const bool on = [] {
        const char *v = getenv("OEC_NO_PDL");
        return !(v && v[0] == '1');
    }();
    return on;
}

namespace {

constexpr int kThreads = 256;           // threads per CTA
constexpr int kPer = 4;                 // particles per thread (one float4)
constexpr int kChunk = kThreads * kPer; // particles per CTA iteration
constexpr float kBelowOne = 0x1.fffffep-1f;

// ------------------------------------------------------------------ A1

__global__ void k_from_aos(const double *__restrict__ aos, int64_t n, oec_particles_t p, int nx,
                           int ny, double dxi, double dyi, double lxh, double lyh) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) *p.count = (int32_t)n;
    if (i >= n) return;
    const double *r = aos + 6 * i;
    // particles.pyx:408-413: normalised coordinate, truncating cast, remainder.
    double ux = (r[0] + lxh) * dxi;
    double uy = (r[1] + lyh) * dyi;
    double fx = floor(ux), fy = floor(uy);
    int ix = (int)fmax(fmin(fx, (double)(nx - 2)), 0.0);
    int iy = (int)fmax(fmin(fy, (double)(ny - 2)), 0.0);
    float ox = (float)(ux - (double)ix);
    float oy = (float)(uy - (double)iy);
    ox = fminf(fmaxf(ox, 0.0f), kBelowOne);
    oy = fminf(fmaxf(oy, 0.0f), kBelowOne);
    p.cell[i] = ix + iy * nx;
    p.ox[i] = ox;
    p.oy[i] = oy;
    p.vx[i] = (float)r[2];
    p.vy[i] = (float)r[3];
    p.vz[i] = (float)r[4];
    p.w[i] = (float)r[5];
}

__global__ void k_to_aos(oec_particles_t p, double *__restrict__ aos, int64_t max_rows, int nx,
                         float inv_nx, double dx, double dy, double lxh, double lyh) {
    int64_t n = *p.count;
    if (n > max_rows) n = max_rows;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        int ix, iy;
        split_cell(p.cell[i], nx, inv_nx, ix, iy);
        double *r = aos + 6 * i;
        r[0] = abs_coord(ix, p.ox[i], dx, lxh);
        r[1] = abs_coord(iy, p.oy[i], dy, lyh);
        r[2] = (double)p.vx[i];
        r[3] = (double)p.vy[i];
        r[4] = (double)p.vz[i];
        r[5] = (double)p.w[i];
    }
}

// ------------------------------------------------------------------ A2

__global__ void k_calc_weights(oec_particles_t p, uint32_t *__restrict__ in_cell,
                               double *__restrict__ w00, double *__restrict__ w10,
                               double *__restrict__ w01, double *__restrict__ w11) {
    int64_t n = *p.count;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double fx = (double)p.ox[i], fy = (double)p.oy[i];
        in_cell[i] = (uint32_t)p.cell[i];
        w00[i] = (1.0 - fx) * (1.0 - fy);
        w10[i] = fx * (1.0 - fy);
        w01[i] = (1.0 - fx) * fy;
        w11[i] = fx * fy;
    }
}

// ---------------------------------------------------------- field tables

__global__ void k_field_prepare(const double *__restrict__ f, int ncomp, int nx, int G,
                                float4 *__restrict__ out) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < G; c += gridDim.x * blockDim.x) {
        for (int k = 0; k < ncomp; ++k) {
            const double *fk = f + (int64_t)k * G;
            float4 q;
            q.x = (float)fk[c];
            q.y = (c + 1 < G) ? (float)fk[c + 1] : 0.0f;
            q.z = (c + nx < G) ? (float)fk[c + nx] : 0.0f;
            q.w = (c + nx + 1 < G) ? (float)fk[c + nx + 1] : 0.0f;
            out[(int64_t)c * ncomp + k] = q;
        }
    }
}

__device__ __forceinline__ float corner_sum(float4 q, float w00, float w10, float w01, float w11) {
    // particles.pyx:363-372 accumulation order.
    float s = w00 * q.x;
    s += w10 * q.y;
    s += w01 * q.z;
    s += w11 * q.w;
    return s;
}

__global__ void k_gather(oec_particles_t p, const float4 *__restrict__ tab, int ncomp, int ncell,
                         double *__restrict__ out) {
    int64_t n = *p.count;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        int c = p.cell[i];
        if ((unsigned)c >= (unsigned)ncell) {
            for (int k = 0; k < ncomp; ++k) out[i * ncomp + k] = 0.0;
            continue;
        }
        float fx = p.ox[i], fy = p.oy[i];
        float w00 = (1.0f - fx) * (1.0f - fy), w10 = fx * (1.0f - fy);
        float w01 = (1.0f - fx) * fy, w11 = fx * fy;
        for (int k = 0; k < ncomp; ++k)
            out[i * ncomp + k] = (double)corner_sum(__ldg(&tab[(int64_t)c * ncomp + k]), w00, w10, w01, w11);
    }
}

// ------------------------------------------------------------- A5-A7

struct PushConst {
    int type_b;
    float qm_dt;             // type 0: q/m*dt ; types 1,2: q/(2m)*dt
    float t0, t1, t2;        // type 1 rotation vector
    float s0, s1, s2;        // type 1: 2t/(1+t.t)
    float dtdxi, dtdyi;      // dt/dx, dt/dy (cell units per m/s)
};

// One Boris step on (vx,vy,vz) with E (and B for type 2): particles.pyx:272-333.
template <int TB>
__device__ __forceinline__ void boris(const PushConst &k, float ex, float ey, float bx, float by,
                                      float bz, float &vx, float &vy, float &vz) {
    if (TB == 0) {
        vx += k.qm_dt * ex;
        vy += k.qm_dt * ey;
    } else {
        float t0, t1, t2, s0, s1, s2;
        if (TB == 1) {
            t0 = k.t0; t1 = k.t1; t2 = k.t2;
            s0 = k.s0; s1 = k.s1; s2 = k.s2;
        } else {
            t0 = k.qm_dt * bx; t1 = k.qm_dt * by; t2 = k.qm_dt * bz;
            float f = 2.0f / (1.0f + t0 * t0 + t1 * t1 + t2 * t2);
            s0 = t0 * f; s1 = t1 * f; s2 = t2 * f;
        }
        float hx = k.qm_dt * ex, hy = k.qm_dt * ey;
        vx += hx;
        vy += hy;
        float w0 = vx + vy * t2 - vz * t1;
        float w1 = vy + vz * t0 - vx * t2;
        float w2 = vz + vx * t1 - vy * t0;
        vx += w1 * s2 - w2 * s1 + hx;
        vy += w2 * s0 - w0 * s2 + hy;
        vz += w0 * s1 - w1 * s0;
    }
}

// ----------------------------------------------------- boundary geometry

struct BoundaryConst {
    int kind;
    double rx, ry;           // rect: lx/2, ly/2
    double ex, ey;           // ellipse: 4/lx^2, 4/ly^2
    const uint16_t *faces;   // cut-cell
    const double *bpts;
    const int32_t *cpi;
    float clip_lo;           // cut-cell clip, cell units (1e-6)
    // rect: the cells [sx0, sx1] x [sy0, sy1] lie wholly inside the box with
    // a margin far above the rounding of the f64 coordinate, so every particle
    // in them passes the f64 test; particles in other cells (and all of the
    // other kinds: empty range) take the f64 test.
    int sx0, sx1, sy0, sy1;
};

// Inside predicates of particleBoundary.pyx evaluated in FP64 with explicit
// round-to-nearest operations (no FMA contraction) so that the decision is
// bit-identical to the FP64 reference for the same stored position.
__device__ __forceinline__ bool inside_rect(const BoundaryConst &b, double x, double y) {
    // particleBoundary.pyx:92-97: outside if x<-lx/2 or x>lx/2 or y<-ly/2 or y>ly/2.
    return !(x < -b.rx || x > b.rx || y < -b.ry || y > b.ry);
}

__device__ __forceinline__ bool inside_ellipse(const BoundaryConst &b, double x, double y) {
    // particleBoundary.pyx:238-242: outside if x^2*4/lx^2 + y^2*4/ly^2 >= 1.
    double r = __dadd_rn(__dmul_rn(__dmul_rn(x, x), b.ex), __dmul_rn(__dmul_rn(y, y), b.ey));
    return !(r >= 1.0);
}

__device__ __forceinline__ bool inside_cutcell(const BoundaryConst &b, int cell, double x, double y) {
    // particleBoundary.pyx:358-370.
    unsigned f = b.faces[cell];
    if (f == 8) return true;
    if (f == 0) return false;
    int i0 = b.cpi[2 * cell], i1 = b.cpi[2 * cell + 1];
    if (i0 < 0 || i1 < 0) return false;
    double a = __dmul_rn(__dsub_rn(b.bpts[2 * i0], x), __dsub_rn(b.bpts[2 * i1 + 1], y));
    double c = __dmul_rn(__dsub_rn(b.bpts[2 * i1], x), __dsub_rn(b.bpts[2 * i0 + 1], y));
    return a > c;
}

// ----------------------------------------------------------- deposit

// Quantised corner charges of one particle; the four parts sum exactly to
// llrint(w * wscale) so the deposited total is independent of splitting.
// gx, gy are the in-cell offsets widened to f64.  The parts are integers
// below 2^51 held in doubles: round-to-nearest products and rint_d give the
// same values as llrint of the plain products, and sums of a few parts stay
// exact in f64.
__device__ __forceinline__ double rint_d(double x) {
    const double C = 6755399441055744.0;  // 1.5 * 2^52: x + C rounds x to an integer (|x| < 2^51)
    return __dsub_rn(__dadd_rn(x, C), C);
}

__device__ __forceinline__ void corner_charges(float w, double gx, double gy, double wscale, double v[4]) {
    const double qd = rint_d(__dmul_rn((double)w, wscale));
    const double hx = __dsub_rn(1.0, gx), hy = __dsub_rn(1.0, gy);
    v[0] = rint_d(__dmul_rn(qd, __dmul_rn(hx, hy)));  // LowXLowY  -> node c
    v[1] = rint_d(__dmul_rn(qd, __dmul_rn(gx, hy)));  // UpXLowY   -> node c+1
    v[2] = rint_d(__dmul_rn(qd, __dmul_rn(hx, gy)));  // LowXUpY   -> node c+nx
    v[3] = __dsub_rn(__dsub_rn(__dsub_rn(qd, v[0]), v[1]), v[2]);  // UpXUpY -> node c+nx+1
}

__device__ __forceinline__ void add_node4(unsigned long long *rho, int key, int nx, const double v[4]) {
    atomicAdd(rho + key, (unsigned long long)__double2ll_rn(v[0]));
    atomicAdd(rho + key + 1, (unsigned long long)__double2ll_rn(v[1]));
    atomicAdd(rho + key + nx, (unsigned long long)__double2ll_rn(v[2]));
    atomicAdd(rho + key + nx + 1, (unsigned long long)__double2ll_rn(v[3]));
}

// A CTA's deposit window: kWinRows x kWinCols node sums in shared memory,
// anchored 4 cells left of and 8 cells below the cell of the chunk's first
// particle.  Cell-ordered storage puts a chunk's 1024 particles in a short run
// of one row; pushes move some of them to neighbouring cells and rows, which
// cuts warps into many short key runs but keeps the chunk inside the window.
// The window is tall rather than wide: in a dipole field B_y the electrons
// gyrate on a small radius in x but stream freely along y, so between sorts
// they leave their row far sooner than their column (16 x 24 ran 3 % faster
// than 10 x 40 on the 2^24-electron, B_y = 0.5 T microbench).
// Nodes are summed here and sent to the grid once per chunk; a cell whose
// four nodes fall outside the window is added to the grid directly, so any
// particle order gives the same exact result.
//
// An int64 charge x of magnitude below 2^41 is held as two 32-bit planes,
// x = lo + mid*2^21 with lo = x & (2^21 - 1) (unsigned) and mid = x >> 21
// (signed, |mid| <= 2^20), each summed with fire-and-forget 32-bit shared
// atomics (a 64-bit shared add would need a compare-and-swap loop).  A node
// takes at most one add per particle of the chunk (1024), so the lo sum
// stays below 2^31 and the mid sum inside +-2^30, also when the copies below
// are summed: no plane overflows and the recombined total is exact.  A value
// of 2^41 or more (a run of very heavy particles in a small store) goes to
// the grid directly instead, so the window never needs a third plane.
//
// Dense cells put most lanes of a warp on the same few nodes, and same-address
// shared atomics serialise; each node therefore has kWinCopies copies of its
// planes, lane l adding to copy l % kWinCopies, and the flush sums the copies.
// Layout: word (entry * 2 + plane) * kWinCopies + copy.
constexpr int kWinRows = 16, kWinCols = 24, kWinNodes = kWinRows * kWinCols;
constexpr int kWinCopies = 4;
constexpr int kWinPlanes = 2;
constexpr int kWinWords = kWinNodes * kWinPlanes * kWinCopies;

struct NodeWindow {
    unsigned *v;   // shared, kWinWords
    int ox, oy;    // node (column, row) of entry 0

    // x to window entry e (grid node `node` when x is out of the planes' range)
    __device__ __forceinline__ void add_entry(int e, long long x, unsigned long long *rho, int node) {
        if ((unsigned long long)(x + (1LL << 41)) >= (1ULL << 42)) {
            atomicAdd(rho + node, (unsigned long long)x);
            return;
        }
        unsigned *w = v + e * (kWinPlanes * kWinCopies) + (threadIdx.x & (kWinCopies - 1));
        atomicAdd(w, (unsigned)x & 0x1fffffu);
        atomicAdd(w + kWinCopies, (unsigned)(int)(x >> 21));
    }

    __device__ __forceinline__ void add(int key, const double q[4], unsigned long long *rho, int nx,
                                        unsigned long long nx_magic) {
        int ix, iy;
        split_cell_m(key, nx, nx_magic, ix, iy);
        add_at(key, ix, iy, q, rho, nx);
    }

    // x to window entry e, |x| < 2^41 known
    __device__ __forceinline__ void add_entry_in_range(int e, long long x) {
        unsigned *w = v + e * (kWinPlanes * kWinCopies) + (threadIdx.x & (kWinCopies - 1));
        atomicAdd(w, (unsigned)x & 0x1fffffu);
        atomicAdd(w + kWinCopies, (unsigned)(int)(x >> 21));
    }

    // add_at for the corner charges of a particle whose whole charge is
    // below 2^40 in magnitude, so every corner is below 2^41 and the range
    // test is made once per particle by the caller instead of per corner
    // (3 % of the fused step on the 2^24-electron microbench)
    __device__ __forceinline__ void add_at_in_range(int key, int ix, int iy, const double q[4],
                                                    unsigned long long *rho, int nx) {
        const int rx = ix - ox, ry = iy - oy;
        if ((unsigned)rx < (unsigned)(kWinCols - 1) && (unsigned)ry < (unsigned)(kWinRows - 1)) {
            const int e = ry * kWinCols + rx;
            add_entry_in_range(e, __double2ll_rn(q[0]));
            add_entry_in_range(e + 1, __double2ll_rn(q[1]));
            add_entry_in_range(e + kWinCols, __double2ll_rn(q[2]));
            add_entry_in_range(e + kWinCols + 1, __double2ll_rn(q[3]));
        } else {
            add_node4(rho, key, nx, q);
        }
    }

    // the same for cell key = ix + iy * nx with its column and row known
    __device__ __forceinline__ void add_at(int key, int ix, int iy, const double q[4], unsigned long long *rho,
                                           int nx) {
        const int rx = ix - ox, ry = iy - oy;
        if ((unsigned)rx < (unsigned)(kWinCols - 1) && (unsigned)ry < (unsigned)(kWinRows - 1)) {
            const int e = ry * kWinCols + rx;
            add_entry(e, __double2ll_rn(q[0]), rho, key);
            add_entry(e + 1, __double2ll_rn(q[1]), rho, key + 1);
            add_entry(e + kWinCols, __double2ll_rn(q[2]), rho, key + nx);
            add_entry(e + kWinCols + 1, __double2ll_rn(q[3]), rho, key + nx + 1);
        } else {
            add_node4(rho, key, nx, q);
        }
    }
};

// Window anchor from the chunk's first cell (clamped to a valid cell).
__device__ __forceinline__ void window_anchor(NodeWindow &nw, int first, int ncell, int nx,
                                              unsigned long long nx_magic) {
    first = min(max(first, 0), ncell - 1);
    int bx, by;
    split_cell_m(first, nx, nx_magic, bx, by);
    nw.ox = bx - 4;
    nw.oy = by - 8;
}

__device__ __forceinline__ unsigned sum4(const uint4 &a) { return a.x + a.y + a.z + a.w; }

// Send the window's nonzero nodes to the grid and clear it (all threads of
// the CTA, after a barrier that follows the last add).  Only entries that a
// valid cell wrote are nonzero, so every node sent is on the grid.
__device__ __forceinline__ void window_flush(const NodeWindow &nw, unsigned long long *rho, int nx, int nodes) {
    (void)nodes;
    static_assert(kWinCopies == 4, "flush reads the copies of a plane as one uint4");
    const uint4 z = make_uint4(0u, 0u, 0u, 0u);
    for (int e = threadIdx.x; e < kWinNodes; e += blockDim.x) {
        uint4 *w = reinterpret_cast<uint4 *>(nw.v + e * (kWinPlanes * kWinCopies));
        const unsigned lo = sum4(w[0]), mid = sum4(w[1]);
        if (lo | mid) {
            w[0] = z;
            w[1] = z;
            const long long x = (long long)lo + (long long)(int)mid * (1LL << 21);
            const int node = (nw.oy + e / kWinCols) * nx + nw.ox + e % kWinCols;
            if (x != 0 && OEC_IN_BOUNDS(node, nodes)) atomicAdd(rho + node, (unsigned long long)x);
        }
    }
}

// A thread's deposit accumulator: charges of consecutive particles in the
// same cell are summed in registers (cell-ordered storage puts a thread's
// four consecutive particles in one or two cells; the f64 sums of integer
// parts below 2^50 are exact) and a run goes to the node window when the
// cell changes.  Used by the standalone deposit, whose particles sit in
// their stored order; after a push the runs are short enough that the
// fused kernel adds each particle to the window directly (4 % faster on the
// 2^24-electron microbench).
struct DepAcc {
    int k;
    double a[4];
    __device__ __forceinline__ void reset() {
        k = -1;
#pragma unroll
        for (int t = 0; t < 4; ++t) a[t] = 0.0;
    }
    __device__ __forceinline__ void add(int key, const double v[4], NodeWindow &nw, unsigned long long *rho, int nx,
                                        unsigned long long nx_magic) {
        if (key != k) {
            if (k >= 0) nw.add(k, a, rho, nx, nx_magic);
            k = key;
#pragma unroll
            for (int t = 0; t < 4; ++t) a[t] = v[t];
        } else {
#pragma unroll
            for (int t = 0; t < 4; ++t) a[t] = __dadd_rn(a[t], v[t]);
        }
    }
    __device__ __forceinline__ void deposit(NodeWindow &nw, unsigned long long *rho, int nx,
                                            unsigned long long nx_magic) const {
        if (k >= 0) nw.add(k, a, rho, nx, nx_magic);
    }
};

// ------------------------------------------------------- fused kernel

struct FusedArgs {
    int32_t *cell;
    float *ox, *oy, *vx, *vy, *vz;
    const float *w;
    const int32_t *count;
    const float4 *etab;      // 2 float4 per cell
    const float4 *btab;      // 3 float4 per cell (type 2)
    PushConst k;
    BoundaryConst b;
    int nx, ny;
    int ncell;               // cells with all four corners on the grid: G - nx - 1
    float inv_nx;
    unsigned long long nx_magic;  // split_magic(nx)
    double dx, dy, lxh, lyh;
    uint32_t *mask;
    unsigned long long *rho;
    const double *wscale;
    oec_status_t *status;
    int64_t capacity;
};

struct Tally {
    int absorbed = 0, nonfinite = 0, clipped = 0, outgrid = 0;
};

// One thread's group of kPer consecutive particles (float4 group q), its
// SoA fields already in registers: gather, push, move, wall test, write-back,
// absorbed bits and the deposit of the survivors.
template <int TB, int KIND, bool DEP>
__device__ __forceinline__ void process_group(const FusedArgs &a, int q, int n, double wscale, int4 c4, float4 fx4,
                                              float4 fy4, float4 vx4, float4 vy4, float4 vz4, float4 w4,
                                              Tally &t, NodeWindow &nw) {
    const int lane = threadIdx.x & 31;
    const int base = q * kPer;
    int cc[4] = {c4.x, c4.y, c4.z, c4.w};
    float fx[4] = {fx4.x, fx4.y, fx4.z, fx4.w};
    float fy[4] = {fy4.x, fy4.y, fy4.z, fy4.w};
    float vx[4] = {vx4.x, vx4.y, vx4.z, vx4.w};
    float vy[4] = {vy4.x, vy4.y, vy4.z, vy4.w};
    float vz[4] = {vz4.x, vz4.y, vz4.z, vz4.w};
    float ww[4] = {w4.x, w4.y, w4.z, w4.w};
    unsigned nib = 0;

#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        if (base + j >= n) continue;
        const int c = cc[j];
        if ((unsigned)c >= (unsigned)a.ncell) {  // not a valid interpolation cell
            nib |= 1u << j;
            ++t.outgrid;
            continue;
        }
        // --- gather at the current position (particles.pyx:354-372)
        float gx = fx[j], gy = fy[j];
        float w00 = (1.0f - gx) * (1.0f - gy), w10 = gx * (1.0f - gy);
        float w01 = (1.0f - gx) * gy, w11 = gx * gy;
        float4 qx = __ldg(&a.etab[2 * c]);
        float4 qy = __ldg(&a.etab[2 * c + 1]);
        float ex = corner_sum(qx, w00, w10, w01, w11);
        float ey = corner_sum(qy, w00, w10, w01, w11);
        float bx = 0.f, by = 0.f, bz = 0.f;
        if (TB == 2) {
            bx = corner_sum(__ldg(&a.btab[3 * c]), w00, w10, w01, w11);
            by = corner_sum(__ldg(&a.btab[3 * c + 1]), w00, w10, w01, w11);
            bz = corner_sum(__ldg(&a.btab[3 * c + 2]), w00, w10, w01, w11);
        }
        // --- push
        boris<TB>(a.k, ex, ey, bx, by, bz, vx[j], vy[j], vz[j]);
        // --- move in cell units and carry whole cells into the index
        float nxo = gx + a.k.dtdxi * vx[j];
        float nyo = gy + a.k.dtdyi * vy[j];
        int ix, iy;
        split_cell_m(c, a.nx, a.nx_magic, ix, iy);
        // huge or non-finite moves take the checked path
        bool finite = true;
        float cxo = nxo, cyo = nyo;
        if (!(fabsf(nxo) < 1048576.f && fabsf(nyo) < 1048576.f)) {
            finite = isfinite(nxo) && isfinite(nyo);
            cxo = fminf(fmaxf(nxo, -1048576.f), 1048576.f);
            cyo = fminf(fmaxf(nyo, -1048576.f), 1048576.f);
        }
        bool out = false;
        if (!finite) {
            ++t.nonfinite;
            out = true;
            fx[j] = nxo;
            fy[j] = nyo;
        } else {
            float sx, sy;
            const int isx = floor_small(cxo, sx);
            const int isy = floor_small(cyo, sy);
            nxo -= sx;
            nyo -= sy;
            ix += isx;
            iy += isy;
            if (nxo >= 1.0f) { nxo = 0.0f; ix += 1; }
            if (nyo >= 1.0f) { nyo = 0.0f; iy += 1; }
            if (KIND == OEC_BOUNDARY_CUTCELL) {
                // _clipParticleDataToGrid (particleBoundary.pyx:485-508):
                // keep the point 1e-6 cells inside the extended grid.
                bool clip = false;
                if (ix < 0 || (ix == 0 && nxo < a.b.clip_lo)) { ix = 0; nxo = a.b.clip_lo; clip = true; }
                if (ix > a.nx - 2) { ix = a.nx - 2; nxo = 1.0f - a.b.clip_lo; clip = true; }
                if (ix == a.nx - 2 && nxo > 1.0f - a.b.clip_lo) { nxo = 1.0f - a.b.clip_lo; clip = true; }
                if (iy < 0 || (iy == 0 && nyo < a.b.clip_lo)) { iy = 0; nyo = a.b.clip_lo; clip = true; }
                if (iy > a.ny - 2) { iy = a.ny - 2; nyo = 1.0f - a.b.clip_lo; clip = true; }
                if (iy == a.ny - 2 && nyo > 1.0f - a.b.clip_lo) { nyo = 1.0f - a.b.clip_lo; clip = true; }
                t.clipped += clip ? 1 : 0;
            } else if (ix < 0 || iy < 0 || ix > a.nx - 2 || iy > a.ny - 2) {
                // Left the extended grid: outside any rect/ellipse wall.
                // Keep the old (valid) cell and the unfloored offset so
                // the absolute position stays exact for the wall
                // intersection and no packed index wraps around.
                out = true;
                ++t.outgrid;
                nxo = gx + a.k.dtdxi * vx[j];
                nyo = gy + a.k.dtdyi * vy[j];
                ix = -1;
            }
            fx[j] = nxo;
            fy[j] = nyo;
            if (ix >= 0) cc[j] = ix + iy * a.nx;
            if (!out) {
                const double dox = (double)nxo, doy = (double)nyo;
                bool in;
                if (KIND == OEC_BOUNDARY_RECT && (unsigned)(ix - a.b.sx0) <= (unsigned)(a.b.sx1 - a.b.sx0) &&
                    (unsigned)(iy - a.b.sy0) <= (unsigned)(a.b.sy1 - a.b.sy0)) {
                    in = true;  // interior cell
                } else {
                    const double x = abs_coord_d(ix, dox, a.dx, a.lxh);
                    const double y = abs_coord_d(iy, doy, a.dy, a.lyh);
                    if (KIND == OEC_BOUNDARY_RECT)
                        in = inside_rect(a.b, x, y);
                    else if (KIND == OEC_BOUNDARY_ELLIPSE)
                        in = inside_ellipse(a.b, x, y);
                    else
                        in = inside_cutcell(a.b, cc[j], x, y);
                }
                out = !in;
                // --- charge of the survivor at its new position
                if (DEP && !out && OEC_IN_BOUNDS(cc[j], a.ncell)) {
                    double v[4];
                    corner_charges(ww[j], dox, doy, wscale, v);
                    // |corner| <= |rint(w * wscale)| + 2 (the fourth corner takes the rounding rest)
                    if (fabs((double)ww[j] * wscale) < 0x1p40)
                        nw.add_at_in_range(cc[j], ix, iy, v, a.rho, a.nx);
                    else
                        nw.add_at(cc[j], ix, iy, v, a.rho, a.nx);
                }
            }
        }
        if (out) nib |= 1u << j;
    }

    // --- write back (invalid tail slots are rewritten unchanged)
    reinterpret_cast<int4 *>(a.cell)[q] = make_int4(cc[0], cc[1], cc[2], cc[3]);
    reinterpret_cast<float4 *>(a.ox)[q] = make_float4(fx[0], fx[1], fx[2], fx[3]);
    reinterpret_cast<float4 *>(a.oy)[q] = make_float4(fy[0], fy[1], fy[2], fy[3]);
    reinterpret_cast<float4 *>(a.vx)[q] = make_float4(vx[0], vx[1], vx[2], vx[3]);
    reinterpret_cast<float4 *>(a.vy)[q] = make_float4(vy[0], vy[1], vy[2], vy[3]);
    reinterpret_cast<float4 *>(a.vz)[q] = make_float4(vz[0], vz[1], vz[2], vz[3]);

    // --- absorbed bits: 8 lanes x 4 particles = one 32-bit word
    unsigned word = nib << (4 * (lane & 7));
    word |= __shfl_xor_sync(kFullMask, word, 1);
    word |= __shfl_xor_sync(kFullMask, word, 2);
    word |= __shfl_xor_sync(kFullMask, word, 4);
    if ((lane & 7) == 0) a.mask[q >> 3] = word;
    t.absorbed += __popc(nib);
}

template <int KIND>
__device__ __forceinline__ void publish_tally(const FusedArgs &a, const Tally &t) {
    const int lane = threadIdx.x & 31;
    int s = __reduce_add_sync(kFullMask, t.absorbed);
    if (lane == 0 && s) atomicAdd(&a.status->n_absorbed, s);
    s = __reduce_add_sync(kFullMask, t.nonfinite);
    if (lane == 0 && s) atomicAdd(&a.status->n_nonfinite, s);
    s = __reduce_add_sync(kFullMask, t.outgrid);
    if (lane == 0 && s) atomicAdd(&a.status->n_out_of_grid, s);
    if (KIND == OEC_BOUNDARY_CUTCELL) {
        s = __reduce_add_sync(kFullMask, t.clipped);
        if (lane == 0 && s) atomicAdd(&a.status->n_clipped, s);
    }
}

constexpr int fused_min_blocks(int tb, int kind) { return (tb == 2 || kind == OEC_BOUNDARY_CUTCELL) ? 3 : 4; }

// Persistent loop over chunks of kChunk particles.  With the deposit the CTA
// has two node windows used by alternate chunks, and one barrier per chunk:
// the barrier at the start of chunk k publishes its anchor and ends every add
// of chunk k-1, whose window is then flushed while chunk k adds into the
// other one (that window's last flush, of chunk k-2, ended at the same
// barrier).  A last barrier after the loop ends the final chunk's adds.
template <int TB, int KIND, bool DEP>
__global__ void __launch_bounds__(kThreads, fused_min_blocks(TB, KIND)) k_push_gather(FusedArgs a) {
    __shared__ __align__(16) unsigned win[DEP ? 2 * kWinWords : 4];
    __shared__ int first_cell[2];
    const int n = min(*a.count, (int)a.capacity);
    const int nchunks = (n + kChunk - 1) / kChunk;
    const double wscale = DEP ? *a.wscale : 0.0;
    Tally t;
    NodeWindow nw{win, 0, 0};
    NodeWindow prev{win, 0, 0};  // the previous chunk's window and anchor
    bool have_prev = false;
    int parity = 0;
    if (DEP)
        for (int e = threadIdx.x; e < 2 * kWinWords; e += kThreads) win[e] = 0u;
    for (int chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x) {
        const int q = chunk * kThreads + threadIdx.x;  // float4 group index
        int4 c4 = reinterpret_cast<const int4 *>(a.cell)[q];
        float4 fx4 = reinterpret_cast<const float4 *>(a.ox)[q];
        float4 fy4 = reinterpret_cast<const float4 *>(a.oy)[q];
        float4 vx4 = reinterpret_cast<const float4 *>(a.vx)[q];
        float4 vy4 = reinterpret_cast<const float4 *>(a.vy)[q];
        float4 vz4 = reinterpret_cast<const float4 *>(a.vz)[q];
        float4 w4 = make_float4(0.f, 0.f, 0.f, 0.f);
        if (DEP) {
            w4 = reinterpret_cast<const float4 *>(a.w)[q];
            if (threadIdx.x == 0) first_cell[parity] = c4.x;
            __syncthreads();
            if (have_prev) window_flush(prev, a.rho, a.nx, a.ncell + a.nx + 1);
            nw.v = win + parity * kWinWords;
            window_anchor(nw, first_cell[parity], a.ncell, a.nx, a.nx_magic);
        }
        process_group<TB, KIND, DEP>(a, q, n, wscale, c4, fx4, fy4, vx4, vy4, vz4, w4, t, nw);
        if (DEP) {
            prev.v = nw.v;
            prev.ox = nw.ox;
            prev.oy = nw.oy;
            have_prev = true;
            parity ^= 1;
        }
    }
    if (DEP) {
        __syncthreads();
        if (have_prev) window_flush(prev, a.rho, a.nx, a.ncell + a.nx + 1);
    }
    publish_tally<KIND>(a, t);
}

// ------------------------------------------------------ standalone deposit

__global__ void __launch_bounds__(kThreads)
    k_deposit(const int32_t *__restrict__ cell, const float *__restrict__ ox,
              const float *__restrict__ oy, const float *__restrict__ w, const int32_t *count, int nx,
              int ncell, unsigned long long nx_magic, int capacity, unsigned long long *rho,
              const double *wscale_p) {
    __shared__ __align__(16) unsigned win[kWinWords];
    __shared__ int first_cell;
    const int n = min(*count, capacity);
    const double wscale = *wscale_p;
    const int nchunks = (n + kChunk - 1) / kChunk;
    NodeWindow nw{win, 0, 0};
    for (int e = threadIdx.x; e < kWinWords; e += kThreads) win[e] = 0u;
    for (int chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x) {
        const int q = chunk * kThreads + threadIdx.x;
        const int base = q * kPer;
        int4 c4 = reinterpret_cast<const int4 *>(cell)[q];
        if (threadIdx.x == 0) first_cell = c4.x;
        __syncthreads();
        window_anchor(nw, first_cell, ncell, nx, nx_magic);
        float4 fx4 = reinterpret_cast<const float4 *>(ox)[q];
        float4 fy4 = reinterpret_cast<const float4 *>(oy)[q];
        float4 w4 = reinterpret_cast<const float4 *>(w)[q];
        int cc[4] = {c4.x, c4.y, c4.z, c4.w};
        float fx[4] = {fx4.x, fx4.y, fx4.z, fx4.w};
        float fy[4] = {fy4.x, fy4.y, fy4.z, fy4.w};
        float ww[4] = {w4.x, w4.y, w4.z, w4.w};
        DepAcc acc;
        acc.reset();
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            if (base + j < n && (unsigned)cc[j] < (unsigned)ncell) {
                double v[4];
                corner_charges(ww[j], (double)fx[j], (double)fy[j], wscale, v);
                acc.add(cc[j], v, nw, rho, nx, nx_magic);
            }
        }
        acc.deposit(nw, rho, nx, nx_magic);
        __syncthreads();
        window_flush(nw, rho, nx, ncell + nx + 1);
    }
}

__global__ void k_deposit_finalize(const long long *__restrict__ fix, int G, const double *wscale_p,
                                   double charge, double *__restrict__ out) {
    double f = charge / *wscale_p;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < G; i += gridDim.x * blockDim.x)
        out[i] = (double)fix[i] * f;
}

// wscale = 2^(bits - ceil(log2 max|w|)): integer charge units of a particle
// stay below 2^bits.  `bits` is fixed by the host from the capacity so that
// no node can leave the int64 range even if every particle met in one node.
// Pass 1: grid-wide max of |w| as float bits (monotone for |w| >= 0) into the
// first word of the output; pass 2: the scale, in place.
__global__ void k_wmax(const float *__restrict__ w, const int32_t *count, int *maxbits) {
    int n = *count;
    float m = 0.0f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(w[i]));
    for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(kFullMask, m, off));
    if ((threadIdx.x & 31) == 0 && m > 0.0f) atomicMax(maxbits, __float_as_int(m));
}

__global__ void k_wscale(double *out, int bits) {
    float m = __int_as_float(*reinterpret_cast<const int *>(out));
    int e = 0;
    if (m > 0.0f && isfinite(m)) frexp((double)m, &e);  // m = f*2^e, f in [0.5,1): ceil(log2 m) <= e
    *out = ldexp(1.0, bits - e);
}

// ------------------------------------------------------- inside test only

template <int KIND>
__global__ void __launch_bounds__(kThreads) k_index_inside(FusedArgs a) {
    const int n = *a.count;
    const int lane = threadIdx.x & 31;
    const int nchunks = (n + kChunk - 1) / kChunk;
    int absorbed_local = 0, clipped_local = 0;
    for (int chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x) {
        const int q = chunk * kThreads + threadIdx.x;
        const int base = q * kPer;
        int4 c4 = reinterpret_cast<const int4 *>(a.cell)[q];
        float4 fx4 = reinterpret_cast<const float4 *>(a.ox)[q];
        float4 fy4 = reinterpret_cast<const float4 *>(a.oy)[q];
        int cc[4] = {c4.x, c4.y, c4.z, c4.w};
        float fx[4] = {fx4.x, fx4.y, fx4.z, fx4.w};
        float fy[4] = {fy4.x, fy4.y, fy4.z, fy4.w};
        unsigned nib = 0;
        bool changed = false;
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            if (base + j >= n) continue;
            if ((unsigned)cc[j] >= (unsigned)a.ncell) {
                nib |= 1u << j;
                continue;
            }
            int ix, iy;
            split_cell(cc[j], a.nx, a.inv_nx, ix, iy);
            if (KIND == OEC_BOUNDARY_CUTCELL) {
                float lo = a.b.clip_lo, hi = 1.0f - a.b.clip_lo;
                bool clip = false;
                if (ix == 0 && fx[j] < lo) { fx[j] = lo; clip = true; }
                if (ix == a.nx - 2 && fx[j] > hi) { fx[j] = hi; clip = true; }
                if (iy == 0 && fy[j] < lo) { fy[j] = lo; clip = true; }
                if (iy == a.ny - 2 && fy[j] > hi) { fy[j] = hi; clip = true; }
                clipped_local += clip ? 1 : 0;
                changed |= clip;
            }
            double x = abs_coord(ix, fx[j], a.dx, a.lxh);
            double y = abs_coord(iy, fy[j], a.dy, a.lyh);
            bool in;
            if (KIND == OEC_BOUNDARY_RECT)
                in = inside_rect(a.b, x, y);
            else if (KIND == OEC_BOUNDARY_ELLIPSE)
                in = inside_ellipse(a.b, x, y);
            else
                in = inside_cutcell(a.b, cc[j], x, y);
            if (!in) nib |= 1u << j;
        }
        if (KIND == OEC_BOUNDARY_CUTCELL && changed) {
            reinterpret_cast<float4 *>(a.ox)[q] = make_float4(fx[0], fx[1], fx[2], fx[3]);
            reinterpret_cast<float4 *>(a.oy)[q] = make_float4(fy[0], fy[1], fy[2], fy[3]);
        }
        unsigned word = nib << (4 * (lane & 7));
        word |= __shfl_xor_sync(kFullMask, word, 1);
        word |= __shfl_xor_sync(kFullMask, word, 2);
        word |= __shfl_xor_sync(kFullMask, word, 4);
        if ((lane & 7) == 0) a.mask[q >> 3] = word;
        absorbed_local += __popc(nib);
    }
    int s = __reduce_add_sync(kFullMask, absorbed_local);
    if (lane == 0 && s) atomicAdd(&a.status->n_absorbed, s);
    if (KIND == OEC_BOUNDARY_CUTCELL) {
        s = __reduce_add_sync(kFullMask, clipped_local);
        if (lane == 0 && s) atomicAdd(&a.status->n_clipped, s);
    }
}

}  // namespace
}  // namespace oec

using namespace oec;

namespace oec {
OEC_BOUND_QUERY(bound_violations_particles)
}  // namespace oec

// =================================================================== C ABI

extern "C" int oec_bound_violations(int64_t *out, int32_t reset) {
    if (!out) return OEC_ERR_INVALID;
#ifdef OEC_BOUNDS_CHECK
    unsigned long long a = 0, b = 0;
    OEC_TRY(bound_violations_particles(&a, reset != 0));
    OEC_TRY(bound_violations_boundary(&b, reset != 0));
    *out = (int64_t)(a + b);
#else
    (void)reset;
    *out = -1;  // the normal build does not count
#endif
    return OEC_OK;
}

static bool aligned16(const void *ptr) { return (reinterpret_cast<uintptr_t>(ptr) & 15u) == 0; }

// The kernels read and write whole float4 groups and whole chunks: every
// field array 16-byte aligned, capacity a multiple of kChunk.
static bool valid_particles(const oec_particles_t *p) {
    return p && p->cell && p->ox && p->oy && p->vx && p->vy && p->vz && p->w && p->count &&
           p->capacity > 0 && p->capacity <= INT32_MAX && (p->capacity % kChunk) == 0 && aligned16(p->cell) &&
           aligned16(p->ox) && aligned16(p->oy) && aligned16(p->vx) && aligned16(p->vy) && aligned16(p->vz) &&
           aligned16(p->w);
}

static bool valid_grid(const oec_grid_t *g) {
    return g && g->nx >= 3 && g->ny >= 3 && g->dx > 0 && g->dy > 0 &&
           (int64_t)g->nx * g->ny < (1 << 23);
}

static int64_t cap_chunks(const oec_particles_t *p) { return p->capacity / kChunk; }

static PushConst make_push_const(const GridConst &gc, const double bconst[3], double dt, double qm,
                                 int type_b) {
    PushConst k{};
    k.type_b = type_b;
    if (type_b == 0) {
        k.qm_dt = (float)(qm * dt);
    } else {
        double h = 0.5 * qm * dt;
        k.qm_dt = (float)h;
        if (type_b == 1) {
            double t0 = h * bconst[0], t1 = h * bconst[1], t2 = h * bconst[2];
            double f = 2.0 / (1.0 + t0 * t0 + t1 * t1 + t2 * t2);
            k.t0 = (float)t0; k.t1 = (float)t1; k.t2 = (float)t2;
            k.s0 = (float)(t0 * f); k.s1 = (float)(t1 * f); k.s2 = (float)(t2 * f);
        }
    }
    k.dtdxi = (float)(dt * gc.dxi);
    k.dtdyi = (float)(dt * gc.dyi);
    return k;
}

static int make_boundary_const(const oec_boundary_t *bd, const GridConst &gc, BoundaryConst &b) {
    b = BoundaryConst{};
    b.kind = bd ? bd->kind : OEC_BOUNDARY_RECT;
    b.rx = gc.lx * 0.5;
    b.ry = gc.ly * 0.5;
    b.ex = 4.0 / (gc.lx * gc.lx);
    b.ey = 4.0 / (gc.ly * gc.ly);
    b.clip_lo = 1e-6f;
    b.sx0 = b.sy0 = 1;
    b.sx1 = b.sy1 = 0;
    if (b.kind == OEC_BOUNDARY_RECT) {
        // x = ((ix + o) dx) - lxExt/2 with o in [0, 1) is rounded twice in f64
        // (below 1e-17 m here); the margin is 1e-12 of the box size
        const double mx = 1e-12 * (gc.lx > gc.ly ? gc.lx : gc.ly);
        int x0 = (int)ceil((-b.rx + mx + gc.lxh) / gc.dx), x1 = (int)floor((b.rx - mx + gc.lxh) / gc.dx) - 1;
        int y0 = (int)ceil((-b.ry + mx + gc.lyh) / gc.dy), y1 = (int)floor((b.ry - mx + gc.lyh) / gc.dy) - 1;
        while (x0 * gc.dx - gc.lxh < -b.rx + mx) ++x0;
        while ((x1 + 1) * gc.dx - gc.lxh > b.rx - mx) --x1;
        while (y0 * gc.dy - gc.lyh < -b.ry + mx) ++y0;
        while ((y1 + 1) * gc.dy - gc.lyh > b.ry - mx) --y1;
        if (x0 <= x1 && y0 <= y1) {
            b.sx0 = x0;
            b.sx1 = x1;
            b.sy0 = y0;
            b.sy1 = y1;
        }
    }
    if (b.kind == OEC_BOUNDARY_CUTCELL) {
        if (!bd->inside_faces_dev || !bd->boundary_points_dev || !bd->cut_cell_points_ind_dev)
            return OEC_ERR_INVALID;
        b.faces = bd->inside_faces_dev;
        b.bpts = bd->boundary_points_dev;
        b.cpi = bd->cut_cell_points_ind_dev;
    } else if (b.kind != OEC_BOUNDARY_RECT && b.kind != OEC_BOUNDARY_ELLIPSE) {
        return OEC_ERR_INVALID;
    }
    return OEC_OK;
}

extern "C" int oec_particles_from_aos(const oec_grid_t *grid, const double *aos_dev, int64_t n,
                                      oec_particles_t *p, void *stream) {
    if (!valid_grid(grid) || !valid_particles(p) || n < 0 || (n > 0 && !aos_dev)) return OEC_ERR_INVALID;
    if (n > p->capacity) return OEC_ERR_CAPACITY;
    GridConst gc = make_grid_const(*grid);
    int64_t blocks = (n + 255) / 256;
    if (blocks < 1) blocks = 1;
    k_from_aos<<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(aos_dev, n, *p, gc.nx, gc.ny, gc.dxi,
                                                                gc.dyi, gc.lxh, gc.lyh);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_particles_to_aos(const oec_grid_t *grid, const oec_particles_t *p, double *aos_dev,
                                    int64_t max_rows, void *stream) {
    if (!valid_grid(grid) || !valid_particles(p) || !aos_dev || max_rows < 0) return OEC_ERR_INVALID;
    GridConst gc = make_grid_const(*grid);
    k_to_aos<<<persistent_grid((max_rows + 255) / 256, 8), 256, 0, as_stream(stream)>>>(
        *p, aos_dev, max_rows, gc.nx, 1.0f / (float)gc.nx, gc.dx, gc.dy, gc.lxh, gc.lyh);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_calc_grid_weights(const oec_grid_t *grid, const oec_particles_t *p,
                                     uint32_t *in_cell_dev, double *w00_dev, double *w10_dev,
                                     double *w01_dev, double *w11_dev, void *stream) {
    if (!valid_grid(grid) || !valid_particles(p) || !in_cell_dev || !w00_dev || !w10_dev || !w01_dev ||
        !w11_dev)
        return OEC_ERR_INVALID;
    k_calc_weights<<<persistent_grid(cap_chunks(p) * 4, 8), 256, 0, as_stream(stream)>>>(
        *p, in_cell_dev, w00_dev, w10_dev, w01_dev, w11_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_field_prepare(const oec_grid_t *grid, const double *node_field_dev, int32_t ncomp,
                                 float *cell_field_dev, void *stream) {
    if (!valid_grid(grid) || !node_field_dev || !cell_field_dev || (ncomp != 2 && ncomp != 3))
        return OEC_ERR_INVALID;
    if (((uintptr_t)cell_field_dev & 15u) != 0) return OEC_ERR_INVALID;
    int G = grid->nx * grid->ny;
    k_field_prepare<<<persistent_grid((G + 255) / 256, 8), 256, 0, as_stream(stream)>>>(
        node_field_dev, ncomp, grid->nx, G, reinterpret_cast<float4 *>(cell_field_dev));
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_gather(const oec_grid_t *grid, const oec_particles_t *p, const float *cell_field_dev,
                          int32_t ncomp, double *out_dev, void *stream) {
    if (!valid_grid(grid) || !valid_particles(p) || !cell_field_dev || !out_dev ||
        (ncomp != 2 && ncomp != 3))
        return OEC_ERR_INVALID;
    k_gather<<<persistent_grid(cap_chunks(p) * 4, 8), 256, 0, as_stream(stream)>>>(
        *p, reinterpret_cast<const float4 *>(cell_field_dev), ncomp, grid->nx * grid->ny - grid->nx - 1,
        out_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

namespace oec {
namespace {
// Standalone push (API path): velocity update then move with carry.
__global__ void k_boris_push_move(oec_particles_t p, const double *__restrict__ e_at,
                                  const double *__restrict__ b_at, PushConst k, int nx, int ny, float inv_nx) {
    int64_t n = *p.count;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        float vx = p.vx[i], vy = p.vy[i], vz = p.vz[i];
        float ex = (float)e_at[2 * i], ey = (float)e_at[2 * i + 1];
        if (k.type_b == 0)
            boris<0>(k, ex, ey, 0.f, 0.f, 0.f, vx, vy, vz);
        else if (k.type_b == 1)
            boris<1>(k, ex, ey, 0.f, 0.f, 0.f, vx, vy, vz);
        else
            boris<2>(k, ex, ey, (float)b_at[3 * i], (float)b_at[3 * i + 1], (float)b_at[3 * i + 2], vx,
                     vy, vz);
        p.vx[i] = vx;
        p.vy[i] = vy;
        p.vz[i] = vz;
        float ox = p.ox[i] + k.dtdxi * vx;
        float oy = p.oy[i] + k.dtdyi * vy;
        if (!(isfinite(ox) && isfinite(oy))) continue;  // left for the inside test to absorb
        float fx = floorf(fminf(fmaxf(ox, -1048576.f), 1048576.f));
        float fy = floorf(fminf(fmaxf(oy, -1048576.f), 1048576.f));
        int cx = (int)fx, cy = (int)fy;
        int ix, iy;
        split_cell(p.cell[i], nx, inv_nx, ix, iy);
        if (ix + cx < 0 || iy + cy < 0 || ix + cx > nx - 2 || iy + cy > ny - 2) {
            // left the extended grid: keep the valid cell, unfloored offset
            p.ox[i] = ox;
            p.oy[i] = oy;
            continue;
        }
        ox -= fx;
        oy -= fy;
        if (ox >= 1.0f) { ox = 0.0f; cx += 1; }
        if (oy >= 1.0f) { oy = 0.0f; cy += 1; }
        p.ox[i] = ox;
        p.oy[i] = oy;
        p.cell[i] += cx + cy * nx;
    }
}
}  // namespace
}  // namespace oec

extern "C" int oec_boris_push(const oec_grid_t *grid, oec_particles_t *p, const double *e_at_particles_dev,
                              const double *b_at_particles_dev, const double bconst[3], double dt,
                              double charge_over_mass, int32_t type_b_field, void *stream) {
    if (!valid_grid(grid) || !valid_particles(p) || !e_at_particles_dev) return OEC_ERR_INVALID;
    if (type_b_field < 0 || type_b_field > 2) return OEC_ERR_INVALID;
    if (type_b_field == 1 && !bconst) return OEC_ERR_INVALID;
    if (type_b_field == 2 && !b_at_particles_dev) return OEC_ERR_INVALID;
    GridConst gc = make_grid_const(*grid);
    double zero[3] = {0, 0, 0};
    PushConst k = make_push_const(gc, bconst ? bconst : zero, dt, charge_over_mass, type_b_field);
    k_boris_push_move<<<persistent_grid(cap_chunks(p) * 4, 8), 256, 0, as_stream(stream)>>>(
        *p, e_at_particles_dev, b_at_particles_dev, k, gc.nx, gc.ny, 1.0f / (float)gc.nx);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

static int deposit_bits(int64_t capacity) {
    // A node sums at most `capacity` particles, each below 2^bits units (w
    // is an FP32 below 2^e, so w * 2^(bits - e) stays at least 2^(bits - 24)
    // below 2^bits and its rounding cannot reach 2^bits): with capacity <=
    // 2^(63 - bits) every node stays strictly inside int64.  At most 50 bits
    // so that the f64 corner products stay exact to well below a unit.
    int lc = 0;
    while ((int64_t(1) << lc) < capacity) ++lc;
    int bits = 63 - lc;
    return bits > 50 ? 50 : bits;
}

extern "C" int oec_deposit_scale_capacity(const oec_particles_t *p, int64_t total_capacity, double *wscale_dev,
                                          void *stream) {
    if (!valid_particles(p) || !wscale_dev || total_capacity < p->capacity || total_capacity > (int64_t(1) << 40))
        return OEC_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    OEC_CUDA_TRY(cudaMemsetAsync(wscale_dev, 0, sizeof(double), s));
    k_wmax<<<persistent_grid(cap_chunks(p), 4), kThreads, 0, s>>>(p->w, p->count,
                                                                   reinterpret_cast<int *>(wscale_dev));
    OEC_LAUNCH_CHECK();
    k_wscale<<<1, 1, 0, s>>>(wscale_dev, deposit_bits(total_capacity));
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_deposit_scale(const oec_particles_t *p, double *wscale_dev, void *stream) {
    if (!valid_particles(p)) return OEC_ERR_INVALID;
    return oec_deposit_scale_capacity(p, p->capacity, wscale_dev, stream);
}

template <int TB, int KIND, bool DEP>
static void launch_fused(const FusedArgs &a, int grid_unused, cudaStream_t s) {
    (void)grid_unused;
    // resident CTAs per SM for this instantiation, per device
    static std::atomic<int> cached[kMaxDevices];
    const int per_sm = per_device_cached(cached, [] {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_push_gather<TB, KIND, DEP>, kThreads, 0) !=
                cudaSuccess ||
            b < 1)
            b = 1;
        return b;
    });
    int64_t chunks = ((int64_t)a.capacity + kChunk - 1) / kChunk;
    k_push_gather<TB, KIND, DEP><<<persistent_grid(chunks, per_sm), kThreads, 0, s>>>(a);
}

template <int TB, int KIND>
static void launch_fused_dep(const FusedArgs &a, bool dep, int grid, cudaStream_t s) {
    if (dep)
        launch_fused<TB, KIND, true>(a, grid, s);
    else
        launch_fused<TB, KIND, false>(a, grid, s);
}

template <int TB>
static void launch_fused_kind(const FusedArgs &a, int kind, bool dep, int grid, cudaStream_t s) {
    if (kind == OEC_BOUNDARY_RECT)
        launch_fused_dep<TB, OEC_BOUNDARY_RECT>(a, dep, grid, s);
    else if (kind == OEC_BOUNDARY_ELLIPSE)
        launch_fused_dep<TB, OEC_BOUNDARY_ELLIPSE>(a, dep, grid, s);
    else
        launch_fused_dep<TB, OEC_BOUNDARY_CUTCELL>(a, dep, grid, s);
}

static FusedArgs make_fused_args(const GridConst &gc, oec_particles_t *p) {
    FusedArgs a{};
    a.cell = p->cell;
    a.ox = p->ox;
    a.oy = p->oy;
    a.vx = p->vx;
    a.vy = p->vy;
    a.vz = p->vz;
    a.w = p->w;
    a.count = p->count;
    a.capacity = p->capacity;
    a.nx = gc.nx;
    a.ny = gc.ny;
    a.ncell = gc.G - gc.nx - 1;
    a.inv_nx = 1.0f / (float)gc.nx;
    a.nx_magic = split_magic(gc.nx);
    a.dx = gc.dx;
    a.dy = gc.dy;
    a.lxh = gc.lxh;
    a.lyh = gc.lyh;
    return a;
}

namespace oec {
namespace {

// Arguments of the fused kernel for the store (or store view) p.
int push_args(const oec_grid_t *grid, oec_particles_t *p, const float *e_cell_dev, const float *b_cell_dev,
              const double bconst[3], double dt, double charge_over_mass, int32_t type_b_field,
              const oec_boundary_t *boundary, uint32_t *absorbed_mask_dev, int64_t *rho_fix_dev,
              const double *wscale_dev, oec_status_t *status_dev, FusedArgs &a) {
    if (!valid_grid(grid) || !valid_particles(p) || !e_cell_dev || !absorbed_mask_dev || !status_dev)
        return OEC_ERR_INVALID;
    if (type_b_field < 0 || type_b_field > 2) return OEC_ERR_INVALID;
    if (type_b_field == 1 && !bconst) return OEC_ERR_INVALID;
    if (type_b_field == 2 && !b_cell_dev) return OEC_ERR_INVALID;
    if (rho_fix_dev && !wscale_dev) return OEC_ERR_INVALID;
    GridConst gc = make_grid_const(*grid);
    double zero[3] = {0, 0, 0};
    a = make_fused_args(gc, p);
    a.k = make_push_const(gc, bconst ? bconst : zero, dt, charge_over_mass, type_b_field);
    int rc = make_boundary_const(boundary, gc, a.b);
    if (rc != OEC_OK) return rc;
    a.etab = reinterpret_cast<const float4 *>(e_cell_dev);
    a.btab = reinterpret_cast<const float4 *>(b_cell_dev);
    a.mask = absorbed_mask_dev;
    a.rho = reinterpret_cast<unsigned long long *>(rho_fix_dev);
    a.wscale = wscale_dev;
    a.status = status_dev;
    return OEC_OK;
}

void launch_push(const FusedArgs &a, int32_t type_b_field, const oec_particles_t *p, cudaStream_t s) {
    const int g = persistent_grid(cap_chunks(p), 8);
    const bool dep = a.rho != nullptr;
    if (type_b_field == 0)
        launch_fused_kind<0>(a, a.b.kind, dep, g, s);
    else if (type_b_field == 1)
        launch_fused_kind<1>(a, a.b.kind, dep, g, s);
    else
        launch_fused_kind<2>(a, a.b.kind, dep, g, s);
}

}  // namespace
}  // namespace oec

extern "C" int oec_push_gather(const oec_grid_t *grid, oec_particles_t *p, const float *e_cell_dev,
                               const float *b_cell_dev, const double bconst[3], double dt,
                               double charge_over_mass, int32_t type_b_field,
                               const oec_boundary_t *boundary, uint32_t *absorbed_mask_dev,
                               int64_t *rho_fix_dev, const double *wscale_dev,
                               oec_status_t *status_dev, void *stream) {
    FusedArgs a;
    int rc = push_args(grid, p, e_cell_dev, b_cell_dev, bconst, dt, charge_over_mass, type_b_field, boundary,
                       absorbed_mask_dev, rho_fix_dev, wscale_dev, status_dev, a);
    if (rc != OEC_OK) return rc;
    cudaStream_t s = as_stream(stream);
    OEC_CUDA_TRY(cudaMemsetAsync(&status_dev->n_absorbed, 0, sizeof(int32_t), s));
    if (rho_fix_dev)
        OEC_CUDA_TRY(cudaMemsetAsync(rho_fix_dev, 0, sizeof(int64_t) * (size_t)grid->nx * grid->ny, s));
    launch_push(a, type_b_field, p, s);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_deposit(const oec_grid_t *grid, const oec_particles_t *p, int64_t *rho_fix_dev,
                           const double *wscale_dev, int32_t zero_first, oec_status_t *status_dev,
                           void *stream) {
    (void)status_dev;
    if (!valid_grid(grid) || !valid_particles(p) || !rho_fix_dev || !wscale_dev) return OEC_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    int G = grid->nx * grid->ny;
    if (zero_first) OEC_CUDA_TRY(cudaMemsetAsync(rho_fix_dev, 0, sizeof(int64_t) * (size_t)G, s));
    k_deposit<<<persistent_grid(cap_chunks(p), 8), kThreads, 0, s>>>(
        p->cell, p->ox, p->oy, p->w, p->count, grid->nx, G - grid->nx - 1, split_magic(grid->nx),
        (int)p->capacity, reinterpret_cast<unsigned long long *>(rho_fix_dev),
        wscale_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_deposit_finalize(const oec_grid_t *grid, const int64_t *rho_fix_dev,
                                    const double *wscale_dev, double particle_charge, double *rho_dev,
                                    void *stream) {
    if (!valid_grid(grid) || !rho_fix_dev || !wscale_dev || !rho_dev) return OEC_ERR_INVALID;
    int G = grid->nx * grid->ny;
    k_deposit_finalize<<<persistent_grid((G + 255) / 256, 8), 256, 0, as_stream(stream)>>>(
        reinterpret_cast<const long long *>(rho_fix_dev), G, wscale_dev, particle_charge, rho_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_index_inside(const oec_grid_t *grid, oec_particles_t *p, const oec_boundary_t *boundary,
                                uint32_t *absorbed_mask_dev, oec_status_t *status_dev, void *stream) {
    if (!valid_grid(grid) || !valid_particles(p) || !absorbed_mask_dev || !status_dev || !boundary)
        return OEC_ERR_INVALID;
    GridConst gc = make_grid_const(*grid);
    FusedArgs a = make_fused_args(gc, p);
    int rc = make_boundary_const(boundary, gc, a.b);
    if (rc != OEC_OK) return rc;
    a.mask = absorbed_mask_dev;
    a.status = status_dev;
    cudaStream_t s = as_stream(stream);
    OEC_CUDA_TRY(cudaMemsetAsync(&status_dev->n_absorbed, 0, sizeof(int32_t), s));
    int g = persistent_grid(cap_chunks(p), 8);
    if (a.b.kind == OEC_BOUNDARY_RECT)
        k_index_inside<OEC_BOUNDARY_RECT><<<g, kThreads, 0, s>>>(a);
    else if (a.b.kind == OEC_BOUNDARY_ELLIPSE)
        k_index_inside<OEC_BOUNDARY_ELLIPSE><<<g, kThreads, 0, s>>>(a);
    else
        k_index_inside<OEC_BOUNDARY_CUTCELL><<<g, kThreads, 0, s>>>(a);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

// ============================================ host round trip (end-to-end)

namespace oec {
namespace {

__global__ void k_from_aos_rows(const double *__restrict__ aos, int64_t row0, int64_t rows, oec_particles_t p,
                                int nx, int ny, double dxi, double dyi, double lxh, double lyh) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= rows) return;
    int64_t i = row0 + k;
    const double *r = aos + 6 * k;
    double ux = (r[0] + lxh) * dxi;
    double uy = (r[1] + lyh) * dyi;
    int ix = (int)fmax(fmin(floor(ux), (double)(nx - 2)), 0.0);
    int iy = (int)fmax(fmin(floor(uy), (double)(ny - 2)), 0.0);
    float ox = fminf(fmaxf((float)(ux - (double)ix), 0.0f), kBelowOne);
    float oy = fminf(fmaxf((float)(uy - (double)iy), 0.0f), kBelowOne);
    p.cell[i] = ix + iy * nx;
    p.ox[i] = ox;
    p.oy[i] = oy;
    p.vx[i] = (float)r[2];
    p.vy[i] = (float)r[3];
    p.vz[i] = (float)r[4];
    p.w[i] = (float)r[5];
}

__global__ void k_to_aos_rows(oec_particles_t p, int64_t row0, int64_t rows, double *__restrict__ aos, int nx,
                              float inv_nx, double dx, double dy, double lxh, double lyh) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= rows) return;
    int64_t i = row0 + k;
    int ix, iy;
    split_cell(p.cell[i], nx, inv_nx, ix, iy);
    double *r = aos + 6 * k;
    r[0] = abs_coord(ix, p.ox[i], dx, lxh);
    r[1] = abs_coord(iy, p.oy[i], dy, lyh);
    r[2] = (double)p.vx[i];
    r[3] = (double)p.vy[i];
    r[4] = (double)p.vz[i];
    r[5] = (double)p.w[i];
}

// Two-slot pipeline: the copy of chunk k+1 overlaps the conversion of chunk k.
struct Pipe {
    cudaStream_t copy = nullptr;
    cudaEvent_t copied[2] = {nullptr, nullptr};
    cudaEvent_t used[2] = {nullptr, nullptr};
    bool ready = false;
    int init() {
        if (ready) return OEC_OK;
        OEC_CUDA_TRY(cudaStreamCreateWithFlags(&copy, cudaStreamNonBlocking));
        for (int s = 0; s < 2; ++s) {
            OEC_CUDA_TRY(cudaEventCreateWithFlags(&copied[s], cudaEventDisableTiming));
            OEC_CUDA_TRY(cudaEventCreateWithFlags(&used[s], cudaEventDisableTiming));
        }
        ready = true;
        return OEC_OK;
    }
};

// One pipeline per device; g_pipe_mu is held while a call enqueues its
// copies, so two host threads never interleave their use of the slots.
std::mutex g_pipe_mu;

Pipe *pipe() {
    static Pipe p[kMaxDevices];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    return &p[dev];
}

// Ring of staging slots for a whole host-to-host step: uploads on one
// stream, the kernels on the caller's stream, downloads on a third, so the
// two copy directions overlap each other and the kernels.
constexpr int kRing = 4;

struct StepPipe {
    cudaStream_t h2d = nullptr, d2h = nullptr;
    cudaEvent_t in[kRing], out[kRing], freed[kRing], start = nullptr, done = nullptr;
    bool ready = false;
    int init() {
        if (ready) return OEC_OK;
        OEC_CUDA_TRY(cudaStreamCreateWithFlags(&h2d, cudaStreamNonBlocking));
        OEC_CUDA_TRY(cudaStreamCreateWithFlags(&d2h, cudaStreamNonBlocking));
        for (int k = 0; k < kRing; ++k) {
            OEC_CUDA_TRY(cudaEventCreateWithFlags(&in[k], cudaEventDisableTiming));
            OEC_CUDA_TRY(cudaEventCreateWithFlags(&out[k], cudaEventDisableTiming));
            OEC_CUDA_TRY(cudaEventCreateWithFlags(&freed[k], cudaEventDisableTiming));
        }
        OEC_CUDA_TRY(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
        OEC_CUDA_TRY(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
        ready = true;
        return OEC_OK;
    }
};

StepPipe *step_pipe() {
    static StepPipe p[kMaxDevices];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    return &p[dev];
}

__global__ void k_set_count(int32_t *count, int32_t value) { *count = value; }

}  // namespace
}  // namespace oec

extern "C" int oec_particles_upload_host(const oec_grid_t *grid, const double *aos_host, int64_t n,
                                         oec_particles_t *p, double *staging_dev, int64_t staging_rows,
                                         void *stream) {
    if (!valid_grid(grid) || !valid_particles(p) || n < 0 || (n > 0 && (!aos_host || !staging_dev)) ||
        staging_rows < 2)
        return OEC_ERR_INVALID;
    if (n > p->capacity) return OEC_ERR_CAPACITY;
    std::lock_guard<std::mutex> lock(g_pipe_mu);
    Pipe *ppp = pipe();
    if (!ppp) return OEC_ERR_CUDA;
    Pipe &pp = *ppp;
    int rc = pp.init();
    if (rc != OEC_OK) return rc;
    cudaStream_t s = as_stream(stream);
    GridConst gc = make_grid_const(*grid);
    int64_t half = staging_rows / 2;
    // the copy stream must not run ahead of work already queued on `s`
    OEC_CUDA_TRY(cudaEventRecord(pp.used[0], s));
    OEC_CUDA_TRY(cudaEventRecord(pp.used[1], s));
    int k = 0;
    for (int64_t row0 = 0; row0 < n; row0 += half, ++k) {
        int slot = k & 1;
        int64_t rows = (n - row0 < half) ? (n - row0) : half;
        double *buf = staging_dev + 6 * half * slot;
        OEC_CUDA_TRY(cudaStreamWaitEvent(pp.copy, pp.used[slot], 0));
        OEC_CUDA_TRY(cudaMemcpyAsync(buf, aos_host + 6 * row0, sizeof(double) * 6 * rows, cudaMemcpyHostToDevice,
                                     pp.copy));
        OEC_CUDA_TRY(cudaEventRecord(pp.copied[slot], pp.copy));
        OEC_CUDA_TRY(cudaStreamWaitEvent(s, pp.copied[slot], 0));
        k_from_aos_rows<<<(unsigned)((rows + 255) / 256), 256, 0, s>>>(buf, row0, rows, *p, gc.nx, gc.ny, gc.dxi,
                                                                       gc.dyi, gc.lxh, gc.lyh);
        OEC_LAUNCH_CHECK();
        OEC_CUDA_TRY(cudaEventRecord(pp.used[slot], s));
    }
    int32_t cnt = (int32_t)n;
    OEC_CUDA_TRY(cudaMemcpyAsync(p->count, &cnt, sizeof(int32_t), cudaMemcpyHostToDevice, s));
    OEC_CUDA_TRY(cudaStreamSynchronize(s));  // `cnt` lives on this stack frame
    return OEC_OK;
}

extern "C" int oec_particles_download_host(const oec_grid_t *grid, const oec_particles_t *p, double *aos_host,
                                           int64_t n, double *staging_dev, int64_t staging_rows, void *stream) {
    if (!valid_grid(grid) || !valid_particles(p) || n < 0 || (n > 0 && (!aos_host || !staging_dev)) ||
        staging_rows < 2 || n > p->capacity)
        return OEC_ERR_INVALID;
    std::lock_guard<std::mutex> lock(g_pipe_mu);
    Pipe *ppp = pipe();
    if (!ppp) return OEC_ERR_CUDA;
    Pipe &pp = *ppp;
    int rc = pp.init();
    if (rc != OEC_OK) return rc;
    cudaStream_t s = as_stream(stream);
    GridConst gc = make_grid_const(*grid);
    int64_t half = staging_rows / 2;
    OEC_CUDA_TRY(cudaEventRecord(pp.used[0], pp.copy));
    OEC_CUDA_TRY(cudaEventRecord(pp.used[1], pp.copy));
    int k = 0;
    for (int64_t row0 = 0; row0 < n; row0 += half, ++k) {
        int slot = k & 1;
        int64_t rows = (n - row0 < half) ? (n - row0) : half;
        double *buf = staging_dev + 6 * half * slot;
        OEC_CUDA_TRY(cudaStreamWaitEvent(s, pp.used[slot], 0));  // previous copy out of this slot finished
        k_to_aos_rows<<<(unsigned)((rows + 255) / 256), 256, 0, s>>>(*p, row0, rows, buf, gc.nx,
                                                                     1.0f / (float)gc.nx, gc.dx, gc.dy, gc.lxh,
                                                                     gc.lyh);
        OEC_LAUNCH_CHECK();
        OEC_CUDA_TRY(cudaEventRecord(pp.copied[slot], s));
        OEC_CUDA_TRY(cudaStreamWaitEvent(pp.copy, pp.copied[slot], 0));
        OEC_CUDA_TRY(cudaMemcpyAsync(aos_host + 6 * row0, buf, sizeof(double) * 6 * rows, cudaMemcpyDeviceToHost,
                                     pp.copy));
        OEC_CUDA_TRY(cudaEventRecord(pp.used[slot], pp.copy));
    }
    // make `stream` wait for the last host copies so its users see the data
    OEC_CUDA_TRY(cudaEventRecord(pp.copied[0], pp.copy));
    OEC_CUDA_TRY(cudaStreamWaitEvent(s, pp.copied[0], 0));
    return OEC_OK;
}

extern "C" int oec_push_gather_host(const oec_grid_t *grid, oec_particles_t *p, const double *rows_in_host,
                                    double *rows_out_host, int64_t n, double *staging_dev, int64_t staging_rows,
                                    const float *e_cell_dev, const float *b_cell_dev, const double bconst[3],
                                    double dt, double charge_over_mass, int32_t type_b_field,
                                    const oec_boundary_t *boundary, uint32_t *absorbed_mask_dev,
                                    int64_t *rho_fix_dev, const double *wscale_dev, oec_status_t *status_dev,
                                    void *stream) {
    if (!valid_grid(grid) || !valid_particles(p) || n < 0 || (n > 0 && (!rows_in_host || !rows_out_host)) ||
        !staging_dev || !absorbed_mask_dev || !status_dev)
        return OEC_ERR_INVALID;
    if (n > p->capacity) return OEC_ERR_CAPACITY;
    // slots of C rows (a multiple of kChunk, so every view keeps the float4
    // groups and the absorbed words aligned) and, after them, a count per slot
    const int64_t C = ((staging_rows - 1) / kRing) / kChunk * kChunk;
    if (C < kChunk) return OEC_ERR_INVALID;
    int32_t *counts = reinterpret_cast<int32_t *>(staging_dev + 6 * kRing * C);
    {
        FusedArgs probe;  // argument checks on the whole store
        int rc = push_args(grid, p, e_cell_dev, b_cell_dev, bconst, dt, charge_over_mass, type_b_field, boundary,
                           absorbed_mask_dev, rho_fix_dev, wscale_dev, status_dev, probe);
        if (rc != OEC_OK) return rc;
    }
    std::lock_guard<std::mutex> lock(g_pipe_mu);
    StepPipe *ppp = step_pipe();
    if (!ppp) return OEC_ERR_CUDA;
    StepPipe &pp = *ppp;
    int rc = pp.init();
    if (rc != OEC_OK) return rc;
    cudaStream_t s = as_stream(stream);
    GridConst gc = make_grid_const(*grid);
    OEC_CUDA_TRY(cudaMemsetAsync(&status_dev->n_absorbed, 0, sizeof(int32_t), s));
    if (rho_fix_dev) OEC_CUDA_TRY(cudaMemsetAsync(rho_fix_dev, 0, sizeof(int64_t) * (size_t)gc.G, s));
    k_set_count<<<1, 1, 0, s>>>(p->count, (int32_t)n);
    // neither copy stream may run ahead of the work already queued on s
    OEC_CUDA_TRY(cudaEventRecord(pp.start, s));
    OEC_CUDA_TRY(cudaStreamWaitEvent(pp.h2d, pp.start, 0));
    OEC_CUDA_TRY(cudaStreamWaitEvent(pp.d2h, pp.start, 0));
    int k = 0;
    for (int64_t off = 0; off < n; off += C, ++k) {
        const int slot = k % kRing;
        const int64_t rows = n - off < C ? n - off : C;
        double *buf = staging_dev + 6 * C * slot;
        if (k >= kRing) OEC_CUDA_TRY(cudaStreamWaitEvent(pp.h2d, pp.freed[slot], 0));
        OEC_CUDA_TRY(cudaMemcpyAsync(buf, rows_in_host + 6 * off, sizeof(double) * 6 * rows, cudaMemcpyHostToDevice,
                                     pp.h2d));
        OEC_CUDA_TRY(cudaEventRecord(pp.in[slot], pp.h2d));
        OEC_CUDA_TRY(cudaStreamWaitEvent(s, pp.in[slot], 0));
        k_from_aos_rows<<<(unsigned)((rows + 255) / 256), 256, 0, s>>>(buf, off, rows, *p, gc.nx, gc.ny, gc.dxi, gc.dyi,
                                                                       gc.lxh, gc.lyh);
        k_set_count<<<1, 1, 0, s>>>(counts + slot, (int32_t)rows);
        const int64_t view_cap = p->capacity - off < C ? p->capacity - off : C;
        oec_particles_t view{p->cell + off, p->ox + off, p->oy + off, p->vx + off, p->vy + off, p->vz + off,
                             p->w + off, counts + slot, view_cap};
        FusedArgs a;
        rc = push_args(grid, &view, e_cell_dev, b_cell_dev, bconst, dt, charge_over_mass, type_b_field, boundary,
                       absorbed_mask_dev + off / 32, rho_fix_dev, wscale_dev, status_dev, a);
        if (rc != OEC_OK) return rc;
        launch_push(a, type_b_field, &view, s);
        k_to_aos_rows<<<(unsigned)((rows + 255) / 256), 256, 0, s>>>(*p, off, rows, buf, gc.nx, 1.0f / (float)gc.nx,
                                                                     gc.dx, gc.dy, gc.lxh, gc.lyh);
        OEC_LAUNCH_CHECK();
        OEC_CUDA_TRY(cudaEventRecord(pp.out[slot], s));
        OEC_CUDA_TRY(cudaStreamWaitEvent(pp.d2h, pp.out[slot], 0));
        OEC_CUDA_TRY(cudaMemcpyAsync(rows_out_host + 6 * off, buf, sizeof(double) * 6 * rows, cudaMemcpyDeviceToHost,
                                     pp.d2h));
        OEC_CUDA_TRY(cudaEventRecord(pp.freed[slot], pp.d2h));
    }
    // the caller's stream covers the last download
    OEC_CUDA_TRY(cudaEventRecord(pp.done, pp.d2h));
    OEC_CUDA_TRY(cudaStreamWaitEvent(s, pp.done, 0));
    return OEC_OK;
}
