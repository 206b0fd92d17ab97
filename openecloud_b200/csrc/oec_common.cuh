// oec_common.cuh -- helpers shared by the liboec CUDA translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <utility>

#include "oec.h"

#define OEC_CUDA_TRY(expr)                         \
    do {                                           \
        cudaError_t oec_err_ = (expr);             \
        if (oec_err_ != cudaSuccess) return OEC_ERR_CUDA; \
    } while (0)

#define OEC_LAUNCH_CHECK() OEC_CUDA_TRY(cudaGetLastError())

// Returns the status of an entry point or helper that did not succeed.
#ifndef OEC_TRY
#define OEC_TRY(expr)                    \
    do {                                 \
        const int oec_rc_ = (expr);      \
        if (oec_rc_ != OEC_OK) return oec_rc_; \
    } while (0)
#endif

namespace oec {

constexpr unsigned kFullMask = 0xffffffffu;

// Index checks of the bounds-checked build (-DOEC_BOUNDS_CHECK, built as
// liboec_checked.so by `python -m openecloud_b200.build --bounds-check`):
// OEC_IN_BOUNDS(i, n) is true when 0 <= i < n; otherwise it adds one to the
// library's violation counter (read with oec_bound_violations) and is false,
// so the guarded access is skipped instead of faulting.  In the normal build
// it is the constant true and costs nothing.
// Each translation unit counts its own violations (device variables are not
// shared between units of this non-relocatable build);
// bound_violations_{particles,boundary} read and reset them on the host.
#ifdef OEC_BOUNDS_CHECK
namespace {
__device__ unsigned long long g_bound_violations = 0;
}
__device__ __forceinline__ bool in_bounds_checked(long long i, long long n) {
    if (i >= 0 && i < n) return true;
    atomicAdd(&g_bound_violations, 1ULL);
    return false;
}
#define OEC_IN_BOUNDS(i, n) (::oec::in_bounds_checked((long long)(i), (long long)(n)))
#define OEC_BOUND_QUERY(name)                                                                 \
    int name(unsigned long long *out, bool reset) {                                           \
        OEC_CUDA_TRY(cudaMemcpyFromSymbol(out, g_bound_violations, sizeof(*out)));            \
        if (reset) {                                                                          \
            const unsigned long long z = 0;                                                   \
            OEC_CUDA_TRY(cudaMemcpyToSymbol(g_bound_violations, &z, sizeof(z)));              \
        }                                                                                     \
        return OEC_OK;                                                                        \
    }
#else
#define OEC_IN_BOUNDS(i, n) true
#define OEC_BOUND_QUERY(name)                               \
    int name(unsigned long long *out, bool) {              \
        *out = 0;                                          \
        return OEC_OK;                                     \
    }
#endif
int bound_violations_particles(unsigned long long *out, bool reset);
int bound_violations_boundary(unsigned long long *out, bool reset);

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Devices a process may drive; per-device caches below are indexed by the
// CUDA device ordinal.
constexpr int kMaxDevices = 64;

// A figure that is fixed for a device (an attribute, an occupancy limit),
// computed by `compute` on the first call made with that device current and
// kept per device.  Slots hold value + 1 (0 = not computed yet); two threads
// that race on a first call compute and store the same value.
template <class F>
int per_device_cached(std::atomic<int> *slots, F compute) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return compute();
    int v = slots[dev].load(std::memory_order_relaxed);
    if (v == 0) {
        v = compute() + 1;
        slots[dev].store(v, std::memory_order_relaxed);
    }
    return v - 1;
}

// Number of SMs of the current device (cached per device).
int sm_count();

// Programmatic dependent launch.  A kernel launched by launch_overlapped may
// be scheduled while the kernel before it on the stream (or before it in a
// captured graph) still runs; its first statement is pdl_wait(), which
// returns once that kernel has finished and its writes are visible, and
// pdl_launch() then lets the next kernel be scheduled early in turn.  Both
// are no-ops in a kernel launched the ordinary way.  Setting the environment
// variable OEC_NO_PDL=1 before the first launch turns the overlap off (for
// timing comparisons).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

bool pdl_enabled();

template <typename... P, typename... A>
cudaError_t launch_overlapped(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              A &&...args) {
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

// Persistent grid: enough CTAs to cover `work_items` CTA-sized chunks, at
// most `per_sm` resident CTAs per SM.
inline int persistent_grid(int64_t chunks, int per_sm) {
    int64_t cap = (int64_t)sm_count() * per_sm;
    int64_t g = chunks < cap ? chunks : cap;
    return g < 1 ? 1 : (int)g;
}

// Host-side constants of the extended grid, computed exactly as the
// reference does (grid.pyx:57-68, particles.pyx:52-56).
struct GridConst {
    int nx, ny, G;
    double dx, dy, dxi, dyi;
    double lxh, lyh;        // lxExt/2, lyExt/2 (extended half widths)
    double lx, ly;          // inner domain
};

inline GridConst make_grid_const(const oec_grid_t &g) {
    GridConst c;
    c.nx = g.nx;
    c.ny = g.ny;
    c.G = g.nx * g.ny;
    c.dx = g.dx;
    c.dy = g.dy;
    c.dxi = 1.0 / g.dx;
    c.dyi = 1.0 / g.dy;
    c.lxh = (g.lx + 2.0 * g.dx) * 0.5;
    c.lyh = (g.ly + 2.0 * g.dy) * 0.5;
    c.lx = g.lx;
    c.ly = g.ly;
    return c;
}

// Exact row/column split of a linear cell index with a float reciprocal and
// one correction step (valid for cell < 2^23).
__device__ __forceinline__ void split_cell(int cell, int nx, float inv_nx, int &ix, int &iy) {
    iy = __float2int_rz(((float)cell + 0.5f) * inv_nx);
    ix = cell - iy * nx;
    if (ix < 0) {
        iy -= 1;
        ix += nx;
    } else if (ix >= nx) {
        iy += 1;
        ix -= nx;
    }
}

// Absolute coordinate of (cell index, offset) with round-to-nearest f64
// operations and no contraction, matching the host conversion bit for bit.
__device__ __forceinline__ double abs_coord(int i, float o, double d, double half) {
    return __dsub_rn(__dmul_rn(__dadd_rn((double)i, (double)o), d), half);
}

// ---- conversions without the conversion unit -----------------------------
// Int <-> float conversion instructions issue at a quarter of the FP32 rate
// or less; the hot kernel needs about twenty per particle written the plain
// way, enough to saturate that unit.  The helpers below give bit-identical
// results with FP32/FP64 adds and integer operations only.

// cell -> (ix, iy) with m = ceil(2^64 / nx): floor(cell * m / 2^64) equals
// cell / nx for every 0 <= cell < 2^32 and 2 <= nx < 2^31 (the error term
// cell * (m - 2^64/nx) / 2^64 stays below 1/nx).
inline unsigned long long split_magic(int nx) { return ~0ULL / (unsigned long long)nx + 1ULL; }

__device__ __forceinline__ void split_cell_m(int cell, int nx, unsigned long long m, int &ix, int &iy) {
    iy = (int)__umul64hi((unsigned long long)(unsigned)cell, m);
    ix = cell - iy * nx;
}

// floorf(v) as (float, int) for |v| <= 2^22: adding 1.5*2^23 rounds v to an
// integer held in the low mantissa bits; one compare turns round into floor.
__device__ __forceinline__ int floor_small(float v, float &fl) {
    const float C = 12582912.0f;  // 1.5 * 2^23, bits 0x4b400000
    float t = __fadd_rn(v, C);
    int r = __float_as_int(t) - 0x4b400000;
    float rf = __fsub_rn(t, C);
    if (rf > v) {
        r -= 1;
        rf = __fsub_rn(rf, 1.0f);
    }
    fl = rf;
    return r;
}

// (double)i for any int32: 1.5*2^52 + 2^31 + i carries i in the low word.
__device__ __forceinline__ double int_to_double(int i) {
    return __dsub_rn(__hiloint2double(0x43380000, (int)((unsigned)i ^ 0x80000000u)), 6755401588539392.0);
}

// llrint(x) (round to nearest, ties to even) for |x| < 2^51, also returned
// as a double in xr.
__device__ __forceinline__ long long rint_i64(double x, double &xr) {
    const double C = 6755399441055744.0;  // 1.5 * 2^52, bits 0x4338000000000000
    double t = __dadd_rn(x, C);
    xr = __dsub_rn(t, C);
    return __double_as_longlong(t) - 0x4338000000000000LL;
}

// The same with the offset already widened and the index added without a
// conversion instruction (identical result).
__device__ __forceinline__ double abs_coord_d(int i, double o, double d, double half) {
    return __dsub_rn(__dmul_rn(__dadd_rn(int_to_double(i), o), d), half);
}

}  // namespace oec
