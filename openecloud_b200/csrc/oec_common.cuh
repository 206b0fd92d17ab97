// oec_common.cuh -- helpers shared by the liboec CUDA translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "oec.h"

#define OEC_CUDA_TRY(expr)                         \
    do {                                           \
        cudaError_t oec_err_ = (expr);             \
        if (oec_err_ != cudaSuccess) return OEC_ERR_CUDA; \
    } while (0)

#define OEC_LAUNCH_CHECK() OEC_CUDA_TRY(cudaGetLastError())

namespace oec {

constexpr unsigned kFullMask = 0xffffffffu;

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Number of SMs of the current device (cached per process; the library is
// used with one device per process).
int sm_count();

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

// Warp-segmented suffix sum of four int64 lanes grouped by equal, adjacent
// keys.  On return the first lane of every segment ("head") holds the
// segment's totals.  Keys need not be sorted: a key that reappears after a
// different key starts a new segment.
__device__ __forceinline__ bool warp_segment_sum4(int key, long long v[4]) {
    const int lane = threadIdx.x & 31;
    int prev = __shfl_up_sync(kFullMask, key, 1);
    bool head = (lane == 0) || (prev != key);
    unsigned heads = __ballot_sync(kFullMask, head);
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        long long o0 = __shfl_down_sync(kFullMask, v[0], off);
        long long o1 = __shfl_down_sync(kFullMask, v[1], off);
        long long o2 = __shfl_down_sync(kFullMask, v[2], off);
        long long o3 = __shfl_down_sync(kFullMask, v[3], off);
        if (lane + off < 32) {
            unsigned between = ((1u << off) - 1u) << (lane + 1);
            if ((heads & between) == 0u) {
                v[0] += o0;
                v[1] += o1;
                v[2] += o2;
                v[3] += o3;
            }
        }
    }
    return head;
}

}  // namespace oec
