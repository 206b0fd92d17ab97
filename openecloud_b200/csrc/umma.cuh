// umma.cuh -- 5th-generation tensor-core (tcgen05) building blocks for
// sm_100a and the 3x3 convolution of the learned Poisson network on them.
//
// One CTA of 128 threads computes a tile of 128 pixels of one image row for
// all CO output channels as an implicit GEMM D[128 x CO] = A[128 x 9 CI] *
// B[9 CI x CO]: the K dimension runs over the 9 taps and the CI input
// channels in steps of 16 (one tcgen05.mma of kind::f16 per step, bf16
// operands, f32 accumulation in tensor memory).  Operands sit in shared
// memory in the canonical K-major layout without swizzle: 16-byte rows
// (8 bf16 of one pixel or one output channel), 8 rows per core matrix, the
// two 8-element halves of a 16-wide K step LBO bytes apart and successive
// 8-row groups SBO = 128 bytes apart.  With the rows of a K half stored
// contiguously, the A operand of tap (ty, tx) is the halo row ty shifted by
// tx rows: the same staged input serves all nine taps.  One elected thread
// issues the MMAs and commits them to an mbarrier; every warp then reads its
// 32 accumulator lanes (pixels) with tcgen05.ld and writes bf16 NHWC output.
// Every wait is bounded: a wait that gives up sets *err and the CTA stops
// after freeing its tensor memory.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace oec {
namespace umma {

constexpr int kM = 128;         // pixels per tile (accumulator lanes)
constexpr int kThreads = 128;   // 4 warps: warp w owns accumulator lanes 32w..32w+31
constexpr int kHalo = kM + 2;   // staged pixels per halo row
constexpr int kSpin = 1 << 22;  // bound of an mbarrier wait (try_wait iterations)

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: K-major, no swizzle (layout type 0),
// descriptor version 1 (bits 46-47), start / LBO / SBO in 16-byte units.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr & 0x3FFFFu) >> 4);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of kind::f16: D f32, A and B bf16, both K-major,
// shape M x N.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Bounded wait for the mbarrier phase `parity`; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (int i = 0; i < kSpin; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t"
            ".reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t"
            "}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Tensor-memory allocation (one full warp).
__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive f32 columns of this thread's accumulator lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared-memory layout of the convolution (bytes from the dynamic base,
// which is 1024-byte aligned by the kernel): weights [9][CI/8][CO] rows of
// 16 bytes, two halo buffers [3][CI/8][kHalo] rows (tile k stages into one
// while the tensor cores read the other), the two mbarriers and the tensor
// memory address.  Tensor memory holds two accumulators of CO columns.
template <int CI, int CO>
struct ConvSmem {
    static constexpr int kW = 9 * (CI / 8) * CO * 16;
    static constexpr int kA = 3 * (CI / 8) * kHalo * 16;
    static constexpr int kBar = kW + 2 * kA;
    static constexpr int kBytes = kBar + 32 + 1024;  // + barriers, tmem address, alignment slack
    static constexpr int kCols = 2 * CO <= 32 ? 32 : (2 * CO <= 64 ? 64 : 128);
};

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

// out[y][x][co] = sum_{ty,tx,ci} in[y+ty-1][x+tx-1][ci] * w[co][(ty*3+tx)*CI + ci]
// (zero outside the image), bf16 in and out, f32 accumulation.  Each CTA
// walks its tiles (blockIdx.x, + gridDim.x, ...) as a two-stage pipeline:
// it starts the asynchronous copies of tile k's halo into buffer k % 2,
// writes tile k-1 out of the other accumulator while they fly, then issues
// tile k's MMAs into accumulator k % 2.  Several CTAs share an SM (as many
// as its shared memory holds), so one CTA's copies overlap another's MMAs
// and epilogue.
template <int CI, int CO>
__global__ void __launch_bounds__(kThreads, 1)
    k_conv3(int H, int W, const __nv_bfloat16 *__restrict__ in, const __nv_bfloat16 *__restrict__ wgt,
            __nv_bfloat16 *__restrict__ out, int *err) {
    static_assert(CI % 16 == 0 && CO % 16 == 0 && CO <= 64, "16..64 channels in steps of 16");
    using L = ConvSmem<CI, CO>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                                            ~uintptr_t(1023));
    unsigned char *sW = base;
    unsigned char *sA = base + L::kW;
    uint64_t *bar = reinterpret_cast<uint64_t *>(base + L::kBar);  // bar[0], bar[1]
    uint32_t *tslot = reinterpret_cast<uint32_t *>(base + L::kBar + 16);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int C8 = CI / 8;

    // weights: row (tap, c8, co) = w[co][tap*CI + c8*8 .. +8]
    for (int i = tid; i < 9 * C8 * CO; i += kThreads) {
        const int co = i % CO, c8 = (i / CO) % C8, tap = i / (CO * C8);
        *reinterpret_cast<uint4 *>(sW + (size_t)i * 16) =
            *reinterpret_cast<const uint4 *>(wgt + (size_t)co * 9 * CI + tap * CI + c8 * 8);
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
    }
    if (warp == 0) tmem_alloc(tslot, L::kCols);
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t idesc = idesc_bf16_f32(kM, CO);
    const uint32_t sW0 = smem_u32(sW), sA0 = smem_u32(sA);
    const int tiles_x = (W + kM - 1) / kM;
    const int ntiles = H * tiles_x;
    const int mine = blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    uint32_t phase0 = 0u, phase1 = 0u;  // parity of the next completion of bar[0], bar[1]
    bool ok = true;

    // halo rows y-1..y+1, pixels x0-1..x0+kM of tile `tile` into buffer b: row (r, c8, px),
    // by asynchronous 16-byte copies (zeros stored directly outside the image)
    auto stage = [&](int tile, int b) {
        const int y = tile / tiles_x, x0 = (tile % tiles_x) * kM;
        unsigned char *dst = sA + b * L::kA;
        for (int i = tid; i < 3 * C8 * kHalo; i += kThreads) {
            const int px = i % kHalo, c8 = (i / kHalo) % C8, r = i / (kHalo * C8);
            const int yy = y + r - 1, xx = x0 + px - 1;
            if (yy >= 0 && yy < H && xx >= 0 && xx < W)
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst + (size_t)i * 16)),
                             "l"(in + ((size_t)yy * W + xx) * CI + c8 * 8)
                             : "memory");
            else
                *reinterpret_cast<uint4 *>(dst + (size_t)i * 16) = make_uint4(0u, 0u, 0u, 0u);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    auto staged = [&]() { asm volatile("cp.async.wait_group 0;" ::: "memory"); };
    // MMAs of the tile staged in buffer b into accumulator b, committed to bar[b]
    auto issue = [&](int b) {
        if (tid == 0) {
            const uint32_t a0 = sA0 + (uint32_t)(b * L::kA);
            const uint32_t d = tmem + (uint32_t)(b * CO);
#pragma unroll 1
            for (int tap = 0; tap < 9; ++tap) {
                const int ty = tap / 3, tx = tap % 3;
#pragma unroll
                for (int kc = 0; kc < CI / 16; ++kc) {
                    const uint32_t a = a0 + (uint32_t)(((ty * C8 + 2 * kc) * kHalo + tx) * 16);
                    const uint32_t bw = sW0 + (uint32_t)((tap * C8 + 2 * kc) * CO * 16);
                    mma_bf16(d, smem_desc(a, kHalo * 16, 128), smem_desc(bw, CO * 16, 128), idesc, (tap | kc) != 0);
                }
            }
            commit(bar + b);
        }
        __syncwarp();
    };
    // waits for accumulator b and writes the tile out
    auto epilogue = [&](int tile, int b) {
        if (mbar_wait(bar + b, b ? phase1 : phase0)) {
            if (b) phase1 ^= 1u;
            else phase0 ^= 1u;
        } else {
            atomicExch(err, 1);
            ok = false;
            return;
        }
        fence_after_sync();
        const int y = tile / tiles_x, x = (tile % tiles_x) * kM + warp * 32 + lane;
#pragma unroll
        for (int c0 = 0; c0 < CO; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(b * CO + c0), v);
            if (x < W) {
                uint4 *dst = reinterpret_cast<uint4 *>(out + ((size_t)y * W + x) * CO + c0);
                dst[0] = make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
                dst[1] = make_uint4(pack2(v[8], v[9]), pack2(v[10], v[11]), pack2(v[12], v[13]),
                                    pack2(v[14], v[15]));
            }
        }
    };

    if (mine > 0) {
        stage(blockIdx.x, 0);
        staged();
        fence_async_smem();
        __syncthreads();
        fence_after_sync();
        issue(0);
    }
    for (int k = 1; k < mine; ++k) {  // the same trip count in every thread
        const int b = k & 1;
        // buffer and accumulator b last served tile k-2, whose MMAs this
        // thread saw complete and whose accumulator every warp has read;
        // tile k's copies fly while tile k-1 is written out
        stage(blockIdx.x + k * gridDim.x, b);
        epilogue(blockIdx.x + (k - 1) * gridDim.x, b ^ 1);
        staged();
        fence_async_smem();
        fence_before_sync();
        ok = __syncthreads_and(ok);
        fence_after_sync();
        if (!ok) break;
        issue(b);
    }
    if (mine > 0 && ok) epilogue(blockIdx.x + (mine - 1) * gridDim.x, (mine - 1) & 1);
    fence_before_sync();
    ok = __syncthreads_and(ok);
    if (!ok) {
        // committed MMAs get a bounded time to end before their tensor
        // memory is freed
        mbar_wait(bar, phase0);
        mbar_wait(bar + 1, phase1);
    }
    __syncthreads();
    fence_after_sync();
    if (warp == 0) tmem_free(tmem, L::kCols);
}

}  // namespace umma
}  // namespace oec
