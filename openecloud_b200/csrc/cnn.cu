// cnn.cu -- the learned Poisson preconditioner: a small convolutional network
// (4-level U-Net, 16-32-64-64 channels, 3x3 convolutions) applied as
// z = M r inside the flexible PCG solve (pcg.cu), with the forward pass,
// the backward pass and an Adam step as hand-written kernels.
//
// No counterpart in the reference (it solves with SuperLU only,
// poissonSolver.pyx:59, :85).
//
// Network (all levels on the extended grid, level l has ceil(n/2^l) nodes per
// side; "pool" averages the 2x2 children of a coarse node, "up" copies a
// coarse node to its children):
//   e0 = conv(x, 1->16)          L0      u2 = up(e3) + e2        L2
//   e1 = conv(pool e0, 16->32)   L1      d2 = conv(u2, 64->32)   L2
//   e2 = conv(pool e1, 32->64)   L2      u1 = up(d2) + e1        L1
//   e3 = conv(pool e2, 64->64)   L3      d1 = conv(u1, 32->16)   L1
//                                        u0 = up(d1) + e0        L0
//                                        d0 = conv(u0, 16->16)   L0
//   z = inside * (d0 . w_out)    (1x1 convolution, 16->1)
// The network is linear (no activation, no bias): its target, the inverse of
// the FIT operator, is linear and odd, which a rectifier network is not.
//
// Storage: activations and weights in bf16 (NHWC, channels innermost),
// accumulation in f32.  3x3 convolutions with 16..64 input channels run as
// implicit GEMMs on the tensor cores, in one of two kernels chosen by
// oec_cnn_t.conv_kernel: tcgen05.mma with the accumulators in tensor memory
// (umma.cuh), or the warp-level mma.sync m16n8k16 bf16 -> f32 with operands
// fetched by ldmatrix (below); the single-channel input convolution and the
// 1x1 output use the f32 pipes.  The
// data gradient of a 3x3 convolution is the same kernel with the weights
// flipped and transposed; the weight gradients (training only) are f32
// reductions over the pixels.
#include <cuda_bf16.h>
#include <math.h>
#include <stdint.h>

#include "oec_common.cuh"
#include "umma.cuh"

typedef __nv_bfloat16 bf16;

namespace oec {
namespace {

// ------------------------------------------------------------ network spec
constexpr int kNConv = 7;  // 3x3 convolutions: e0 e1 e2 e3 d2 d1 d0
struct ConvSpec {
    int ci, co, level;
};
__host__ __device__ constexpr ConvSpec conv_spec(int i) {
    return i == 0   ? ConvSpec{1, 16, 0}
           : i == 1 ? ConvSpec{16, 32, 1}
           : i == 2 ? ConvSpec{32, 64, 2}
           : i == 3 ? ConvSpec{64, 64, 3}
           : i == 4 ? ConvSpec{64, 32, 2}
           : i == 5 ? ConvSpec{32, 16, 1}
                    : ConvSpec{16, 16, 0};
}
constexpr int conv_params(int i) { return conv_spec(i).co * 9 * conv_spec(i).ci; }
constexpr int conv_offset(int i) { return i == 0 ? 0 : conv_offset(i - 1) + conv_params(i - 1); }
constexpr int kOutOffset = conv_offset(kNConv);  // 1x1 output weights (16)
constexpr int kNParams = kOutOffset + 16;

struct Level {
    int h, w;
};

// ------------------------------------------------------------------ PTX
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void ldsm_x4(uint32_t r[4], const void *p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_addr(p)));
}

__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

// ------------------------------------------------- 3x3 conv, tensor cores
// out[y][x][co] = sum_{ty,tx,ci} in[y+ty-1][x+tx-1][ci] * w[co][(ty*3+tx)*CI + ci]
// (zero outside the image).  CTA: 4 warps, a tile of 64 pixels of one row;
// warp w computes pixels 16w..16w+15 for all CO channels.  Weights stay in
// shared memory for the CTA's whole persistent loop.
constexpr int kTX = 64;

template <int CI, int CO>
constexpr int conv_smem_bytes() {
    return (CO * (9 * CI + 8) + 3 * (kTX + 2) * (CI + 8)) * 2;
}

template <int CI, int CO>
__global__ void __launch_bounds__(128) k_conv3_mma(int H, int W, const bf16 *__restrict__ in,
                                                   const bf16 *__restrict__ wgt, bf16 *__restrict__ out) {
    static_assert(CI % 16 == 0 && CO % 16 == 0, "tensor-core path needs multiples of 16 channels");
    constexpr int KW = 9 * CI, WS = KW + 8, IS = CI + 8, C8 = CI / 8;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    bf16 *sW = reinterpret_cast<bf16 *>(smem_raw);
    bf16 *sIn = sW + CO * WS;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < CO * (KW / 8); i += 128) {
        const int co = i / (KW / 8), c8 = i % (KW / 8);
        *reinterpret_cast<uint4 *>(sW + co * WS + c8 * 8) = *reinterpret_cast<const uint4 *>(wgt + co * KW + c8 * 8);
    }
    const int tiles_x = (W + kTX - 1) / kTX;
    const int ntiles = H * tiles_x;
    // ldmatrix lane roles
    const int a_m = lane & 15, a_k = (lane >> 4) * 8;
    const int b_n = (lane & 7) + ((lane >> 4) << 3), b_k = ((lane >> 3) & 1) * 8;
    const int g = lane >> 2, t = lane & 3;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int y = tile / tiles_x, x0 = (tile % tiles_x) * kTX;
        __syncthreads();  // the previous tile's reads of sIn are done; weights visible
        for (int i = tid; i < 3 * (kTX + 2) * C8; i += 128) {
            const int c8 = i % C8, px = (i / C8) % (kTX + 2), r = i / (C8 * (kTX + 2));
            const int yy = y + r - 1, xx = x0 + px - 1;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (yy >= 0 && yy < H && xx >= 0 && xx < W)
                v = *reinterpret_cast<const uint4 *>(in + ((size_t)yy * W + xx) * CI + c8 * 8);
            *reinterpret_cast<uint4 *>(sIn + (r * (kTX + 2) + px) * IS + c8 * 8) = v;
        }
        __syncthreads();
        float acc[CO / 8][4];
#pragma unroll
        for (int n = 0; n < CO / 8; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
        const int pbase = warp * 16;
#pragma unroll
        for (int tap = 0; tap < 9; ++tap) {
            const int ty = tap / 3, tx = tap % 3;
            const bf16 *rowA = sIn + (ty * (kTX + 2) + pbase + tx) * IS;
#pragma unroll
            for (int kc = 0; kc < CI / 16; ++kc) {
                uint32_t a[4];
                ldsm_x4(a, rowA + a_m * IS + kc * 16 + a_k);
#pragma unroll
                for (int np = 0; np < CO / 16; ++np) {
                    uint32_t b[4];
                    ldsm_x4(b, sW + (np * 16 + b_n) * WS + tap * CI + kc * 16 + b_k);
                    mma_bf16(acc[2 * np], a, b[0], b[1]);
                    mma_bf16(acc[2 * np + 1], a, b[2], b[3]);
                }
            }
        }
        const int xa = x0 + pbase + g, xb = xa + 8;
#pragma unroll
        for (int n = 0; n < CO / 8; ++n) {
            const int co = n * 8 + 2 * t;
            if (xa < W) *reinterpret_cast<uint32_t *>(out + ((size_t)y * W + xa) * CO + co) = pack_bf16(acc[n][0], acc[n][1]);
            if (xb < W) *reinterpret_cast<uint32_t *>(out + ((size_t)y * W + xb) * CO + co) = pack_bf16(acc[n][2], acc[n][3]);
        }
    }
}

// Input convolution, one channel in (f32), 16 out (bf16); inside mask on x.
// A CTA computes a 32 x 8 pixel tile from a 34 x 10 halo tile of the masked,
// bf16-rounded input staged once in shared memory (each input pixel is read
// from memory once per tile instead of once per tap).
constexpr int kIn1TX = 32, kIn1TY = 8;
__global__ void __launch_bounds__(kIn1TX *kIn1TY)
    k_conv3_in1(int H, int W, const float *__restrict__ x, const uint8_t *__restrict__ inside,
                const bf16 *__restrict__ wgt, bf16 *__restrict__ out, bf16 *__restrict__ x16) {
    __shared__ float sw[16 * 9];
    __shared__ float tile[kIn1TY + 2][kIn1TX + 2];
    const int tid = threadIdx.x;
    for (int i = tid; i < 16 * 9; i += blockDim.x) sw[i] = __bfloat162float(wgt[i]);
    const int x0 = blockIdx.x * kIn1TX, y0 = blockIdx.y * kIn1TY;
    for (int e = tid; e < (kIn1TY + 2) * (kIn1TX + 2); e += blockDim.x) {
        const int ty = e / (kIn1TX + 2), tx = e - ty * (kIn1TX + 2);
        const int yy = y0 + ty - 1, xs = x0 + tx - 1;
        float v = 0.f;
        if (yy >= 0 && yy < H && xs >= 0 && xs < W) {
            const int q = yy * W + xs;
            if (inside[q]) v = __bfloat162float(__float2bfloat16_rn(x[q]));
        }
        tile[ty][tx] = v;
    }
    __syncthreads();
    const int lx = tid % kIn1TX, ly = tid / kIn1TX;
    const int xx = x0 + lx, y = y0 + ly;
    if (xx >= W || y >= H) return;
    const int p = y * W + xx;
    float v[9];
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) v[tap] = tile[ly + tap / 3][lx + tap % 3];
    x16[p] = __float2bfloat16_rn(inside[p] ? x[p] : 0.f);
    uint32_t o[8];
#pragma unroll
    for (int c = 0; c < 16; c += 2) {
        float s0 = 0.f, s1 = 0.f;
#pragma unroll
        for (int tap = 0; tap < 9; ++tap) {
            s0 = fmaf(v[tap], sw[c * 9 + tap], s0);
            s1 = fmaf(v[tap], sw[(c + 1) * 9 + tap], s1);
        }
        o[c / 2] = pack_bf16(s0, s1);
    }
    uint4 *dst = reinterpret_cast<uint4 *>(out + (size_t)p * 16);
    dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
    dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
}

// 2x2 average of the children (out-of-range children count as zero).
template <int C>
__global__ void k_pool(Level fine, Level coarse, const bf16 *__restrict__ in, bf16 *__restrict__ out) {
    const int n = coarse.h * coarse.w * (C / 8);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c8 = i % (C / 8), P = i / (C / 8), Y = P / coarse.w, X = P % coarse.w;
        float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const int y = 2 * Y + (d >> 1), x = 2 * X + (d & 1);
            if (y < fine.h && x < fine.w) {
                uint4 v = *reinterpret_cast<const uint4 *>(in + ((size_t)y * fine.w + x) * C + c8 * 8);
                const bf16 *h = reinterpret_cast<const bf16 *>(&v);
#pragma unroll
                for (int k = 0; k < 8; ++k) s[k] += __bfloat162float(h[k]);
            }
        }
        uint4 o;
        uint32_t *ow = reinterpret_cast<uint32_t *>(&o);
#pragma unroll
        for (int k = 0; k < 4; ++k) ow[k] = pack_bf16(0.25f * s[2 * k], 0.25f * s[2 * k + 1]);
        *reinterpret_cast<uint4 *>(out + (size_t)P * C + c8 * 8) = o;
    }
}

// out[y][x] = a * coarse[y/2][x/2] + skip[y][x]
template <int C>
__global__ void k_up_add(Level fine, Level coarse, float a, const bf16 *__restrict__ crs, const bf16 *__restrict__ skip,
                         bf16 *__restrict__ out) {
    const int n = fine.h * fine.w * (C / 8);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c8 = i % (C / 8), p = i / (C / 8), y = p / fine.w, x = p % fine.w;
        uint4 u = *reinterpret_cast<const uint4 *>(crs + ((size_t)(y >> 1) * coarse.w + (x >> 1)) * C + c8 * 8);
        uint4 v = *reinterpret_cast<const uint4 *>(skip + (size_t)p * C + c8 * 8);
        const bf16 *hu = reinterpret_cast<const bf16 *>(&u);
        const bf16 *hv = reinterpret_cast<const bf16 *>(&v);
        uint4 o;
        uint32_t *ow = reinterpret_cast<uint32_t *>(&o);
#pragma unroll
        for (int k = 0; k < 4; ++k)
            ow[k] = pack_bf16(fmaf(a, __bfloat162float(hu[2 * k]), __bfloat162float(hv[2 * k])),
                              fmaf(a, __bfloat162float(hu[2 * k + 1]), __bfloat162float(hv[2 * k + 1])));
        *reinterpret_cast<uint4 *>(out + (size_t)p * C + c8 * 8) = o;
    }
}

// coarse[Y][X] = sum of the in-range children of fine (gradient of "up").
template <int C>
__global__ void k_down_sum(Level fine, Level coarse, const bf16 *__restrict__ in, bf16 *__restrict__ out) {
    const int n = coarse.h * coarse.w * (C / 8);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c8 = i % (C / 8), P = i / (C / 8), Y = P / coarse.w, X = P % coarse.w;
        float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const int y = 2 * Y + (d >> 1), x = 2 * X + (d & 1);
            if (y < fine.h && x < fine.w) {
                uint4 v = *reinterpret_cast<const uint4 *>(in + ((size_t)y * fine.w + x) * C + c8 * 8);
                const bf16 *h = reinterpret_cast<const bf16 *>(&v);
#pragma unroll
                for (int k = 0; k < 8; ++k) s[k] += __bfloat162float(h[k]);
            }
        }
        uint4 o;
        uint32_t *ow = reinterpret_cast<uint32_t *>(&o);
#pragma unroll
        for (int k = 0; k < 4; ++k) ow[k] = pack_bf16(s[2 * k], s[2 * k + 1]);
        *reinterpret_cast<uint4 *>(out + (size_t)P * C + c8 * 8) = o;
    }
}

// z = inside * sum_c d0[c] w[c]   (f32 out)
__global__ void k_conv_out(int n, const bf16 *__restrict__ d0, const bf16 *__restrict__ w,
                           const uint8_t *__restrict__ inside, float *__restrict__ z) {
    float wf[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) wf[c] = __bfloat162float(w[c]);
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const uint4 *src = reinterpret_cast<const uint4 *>(d0 + (size_t)p * 16);
        uint4 v0 = src[0], v1 = src[1];
        const bf16 *h0 = reinterpret_cast<const bf16 *>(&v0);
        const bf16 *h1 = reinterpret_cast<const bf16 *>(&v1);
        float s = 0.f;
#pragma unroll
        for (int c = 0; c < 8; ++c) s = fmaf(__bfloat162float(h0[c]), wf[c], s);
#pragma unroll
        for (int c = 0; c < 8; ++c) s = fmaf(__bfloat162float(h1[c]), wf[8 + c], s);
        z[p] = inside[p] ? s : 0.f;
    }
}

// ------------------------------------------------------------- backward
// g_d0[p][c] = inside[p] * gz[p] * w[c];  gw[c] += sum_p inside * gz * d0[p][c]
__global__ void k_conv_out_bwd(int n, const float *__restrict__ gz, const bf16 *__restrict__ d0,
                               const bf16 *__restrict__ w, const uint8_t *__restrict__ inside, bf16 *__restrict__ gd0,
                               float *__restrict__ gw) {
    float wf[16], acc[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) {
        wf[c] = __bfloat162float(w[c]);
        acc[c] = 0.f;
    }
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const float gp = inside[p] ? gz[p] : 0.f;
        const uint4 *src = reinterpret_cast<const uint4 *>(d0 + (size_t)p * 16);
        uint4 v0 = src[0], v1 = src[1];
        const bf16 *h0 = reinterpret_cast<const bf16 *>(&v0);
        const bf16 *h1 = reinterpret_cast<const bf16 *>(&v1);
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[c] = fmaf(gp, __bfloat162float(h0[c]), acc[c]);
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[8 + c] = fmaf(gp, __bfloat162float(h1[c]), acc[8 + c]);
        uint32_t o[8];
#pragma unroll
        for (int c = 0; c < 16; c += 2) o[c / 2] = pack_bf16(gp * wf[c], gp * wf[c + 1]);
        uint4 *dst = reinterpret_cast<uint4 *>(gd0 + (size_t)p * 16);
        dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
        dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
    }
#pragma unroll
    for (int c = 0; c < 16; ++c) {
        float v = acc[c];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(kFullMask, v, off);
        if ((threadIdx.x & 31) == 0 && v != 0.f) atomicAdd(gw + c, v);
    }
}

// wt[ci][(8 - tap)*CO + co] = w[co][tap*CI + ci]: the weights of the data
// gradient (a 3x3 convolution from CO to CI channels).
__global__ void k_flip_transpose(int ci, int co, const bf16 *__restrict__ w, bf16 *__restrict__ wt) {
    const int n = 9 * ci * co;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int o = i / (9 * ci), r = i % (9 * ci), tap = r / ci, c = r % ci;
        wt[(size_t)c * 9 * co + (8 - tap) * co + o] = w[i];
    }
}

// gW[co][tap*CI + ci] += sum_p X[p + tap][ci] * G[p][co].  CTA: a slice of 64
// weight columns k (blockIdx.y) for all CO rows, over its range of pixels in
// chunks of 32; each thread a 4 x 4 block of (co, k).
constexpr int kDwPix = 32;

__global__ void __launch_bounds__(256) k_conv3_dw(int H, int W, int CI, int CO, const bf16 *__restrict__ X,
                                                  const bf16 *__restrict__ Gy, float *__restrict__ gW) {
    __shared__ float sX[kDwPix][65];
    __shared__ float sG[kDwPix][65];
    const int KW = 9 * CI, k0 = blockIdx.y * 64;
    const int npix = H * W;
    const int per = (npix + gridDim.x - 1) / gridDim.x;
    const int p0 = blockIdx.x * per, p1 = min(npix, p0 + per);
    const int tid = threadIdx.x;
    const int cob = tid / 16, kb = tid % 16;  // co = 4*cob.., k = 4*kb..
    float acc[4][4] = {};
    for (int pc = p0; pc < p1; pc += kDwPix) {
        __syncthreads();
        for (int i = tid; i < kDwPix * 64; i += 256) {
            const int pp = i / 64, kk = i % 64, p = pc + pp, k = k0 + kk;
            float v = 0.f;
            if (p < p1 && k < KW) {
                const int tap = k / CI, c = k % CI;
                const int y = p / W + tap / 3 - 1, x = p % W + tap % 3 - 1;
                if (y >= 0 && y < H && x >= 0 && x < W) v = __bfloat162float(X[((size_t)y * W + x) * CI + c]);
            }
            sX[pp][kk] = v;
        }
        for (int i = tid; i < kDwPix * 64; i += 256) {
            const int pp = i / 64, o = i % 64, p = pc + pp;
            sG[pp][o] = (p < p1 && o < CO) ? __bfloat162float(Gy[(size_t)p * CO + o]) : 0.f;
        }
        __syncthreads();
        if (4 * cob < CO) {
#pragma unroll 4
            for (int pp = 0; pp < kDwPix; ++pp) {
                float gx[4], xk[4];
#pragma unroll
                for (int a = 0; a < 4; ++a) gx[a] = sG[pp][4 * cob + a];
#pragma unroll
                for (int b = 0; b < 4; ++b) xk[b] = sX[pp][4 * kb + b];
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) acc[a][b] = fmaf(gx[a], xk[b], acc[a][b]);
            }
        }
    }
    if (4 * cob < CO) {
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int k = k0 + 4 * kb + b;
                if (k < KW && acc[a][b] != 0.f) atomicAdd(gW + (size_t)(4 * cob + a) * KW + k, acc[a][b]);
            }
    }
}

// loss = sum_inside (z - t)^2 / sum_inside t^2 ; first pass: the two sums.
__global__ void k_loss_sums(int n, const float *__restrict__ z, const float *__restrict__ tgt,
                            const uint8_t *__restrict__ inside, double *sums) {
    double a = 0.0, b = 0.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        if (inside[p]) {
            const double d = (double)z[p] - (double)tgt[p];
            a += d * d;
            b += (double)tgt[p] * (double)tgt[p];
        }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        a += __shfl_xor_sync(kFullMask, a, off);
        b += __shfl_xor_sync(kFullMask, b, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(sums, a);
        atomicAdd(sums + 1, b);
    }
}

// gz = 2 (z - t) / sum t^2 on the inside nodes
__global__ void k_loss_grad(int n, const float *__restrict__ z, const float *__restrict__ tgt,
                            const uint8_t *__restrict__ inside, const double *sums, float *__restrict__ gz) {
    const double s = sums[1] > 0.0 ? 2.0 / sums[1] : 0.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        gz[p] = inside[p] ? (float)(s * ((double)z[p] - (double)tgt[p])) : 0.f;
}

// Residual loss with the scaled FIT operator A (edge weights ex, ey; see
// oec_stencil_t), invariant to the scale of z (the flexible PCG is):
//   L = |s A z - x|^2 / |x|^2 at the best scalar s = (Az.x) / |Az|^2
//     = 1 - (Az.x)^2 / (|Az|^2 |x|^2),
//   dL/dz = (2 s / |x|^2) A (s A z - x)   (A symmetric).
// First pass: y = A z on the inside nodes, sums = (|Az|^2, |x|^2, Az.x).
__device__ __forceinline__ float stencil_at(int i, int nx, const float *__restrict__ ex, const float *__restrict__ ey,
                                            const float *__restrict__ v) {
    const float vi = v[i];
    return ex[i] * (vi - v[i + 1]) + ex[i - 1] * (vi - v[i - 1]) + ey[i] * (vi - v[i + nx]) +
           ey[i - nx] * (vi - v[i - nx]);
}

__global__ void k_res_loss(int n, int nx, const float *__restrict__ ex, const float *__restrict__ ey,
                           const uint8_t *__restrict__ inside, const float *__restrict__ z, const float *__restrict__ x,
                           float *__restrict__ y, double *sums) {
    double a = 0.0, b = 0.0, c = 0.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        float v = 0.f;
        if (inside[p]) {
            const float xp = x[p];
            v = stencil_at(p, nx, ex, ey, z);
            b += (double)xp * (double)xp;
            c += (double)v * (double)xp;
        }
        y[p] = v;
        a += (double)v * (double)v;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        a += __shfl_xor_sync(kFullMask, a, off);
        b += __shfl_xor_sync(kFullMask, b, off);
        c += __shfl_xor_sync(kFullMask, c, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(sums, a);
        atomicAdd(sums + 1, b);
        atomicAdd(sums + 2, c);
    }
}

// y <- s y - x (inside), s = sums[2] / sums[0]
__global__ void k_res_combine(int n, const uint8_t *__restrict__ inside, const float *__restrict__ x,
                              const double *sums, float *__restrict__ y) {
    const float s = sums[0] > 0.0 ? (float)(sums[2] / sums[0]) : 0.f;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        y[p] = inside[p] ? s * y[p] - x[p] : 0.f;
}

// gz = (2 s / |x|^2) A y on the inside nodes; the loss written as
// sums[0] <- |x|^2 - (Az.x)^2 / |Az|^2 (so loss = sums[0] / sums[1]).
__global__ void k_res_grad(int n, int nx, const float *__restrict__ ex, const float *__restrict__ ey,
                           const uint8_t *__restrict__ inside, const float *__restrict__ y, const double *sums,
                           float *__restrict__ gz) {
    const double sc = sums[0] > 0.0 ? sums[2] / sums[0] : 0.0;
    const float f = sums[1] > 0.0 ? (float)(2.0 * sc / sums[1]) : 0.f;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        gz[p] = inside[p] ? f * stencil_at(p, nx, ex, ey, y) : 0.f;
}

__global__ void k_res_report(double *sums, double *loss_out) {
    const double a = sums[0], b = sums[1], c = sums[2];
    loss_out[0] = a > 0.0 ? b - c * c / a : b;
    loss_out[1] = b;
}

// Warm start phi0 = |b| N(b / |b|), b = scale32 * q on the inside nodes
// (A phi = q  <=>  (scale32 A) phi = b).
__global__ void k_ws_norm(int n, const double *__restrict__ q, const uint8_t *__restrict__ inside, double s,
                          double *sum) {
    double a = 0.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        if (inside[p]) {
            const double b = s * q[p];
            a += b * b;
        }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) a += __shfl_xor_sync(kFullMask, a, off);
    if ((threadIdx.x & 31) == 0 && a != 0.0) atomicAdd(sum, a);
}

__global__ void k_ws_scale(int n, const double *__restrict__ q, const uint8_t *__restrict__ inside, double s,
                           const double *sum, float *__restrict__ x) {
    const double f = sum[0] > 0.0 ? s / sqrt(sum[0]) : 0.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        x[p] = inside[p] ? (float)(f * q[p]) : 0.f;
}

__global__ void k_ws_out(int n, const float *__restrict__ z, const uint8_t *__restrict__ inside, const double *sum,
                         double *__restrict__ phi) {
    const double f = sqrt(sum[0]);
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        phi[p] = inside[p] ? f * (double)z[p] : 0.0;
}

// d = q - 2 q1 + q2 (the second difference in time of the charge, 0 while
// fewer than two earlier charges exist: *count < 2), then q2 <- q1, q1 <- q;
// the sum of |s d|^2 over the inside nodes goes to sum.
__global__ void k_corr_diff(int n, const double *__restrict__ q, double *__restrict__ q1, double *__restrict__ q2,
                            const int32_t *count, const uint8_t *__restrict__ inside, double s, double *__restrict__ d,
                            double *sum) {
    const bool have = *count >= 2;
    double a = 0.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const double qn = q[p], a1 = q1[p];
        const double v = (have && inside[p]) ? qn - 2.0 * a1 + q2[p] : 0.0;
        d[p] = v;
        q2[p] = a1;
        q1[p] = qn;
        a += (s * v) * (s * v);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) a += __shfl_xor_sync(kFullMask, a, off);
    if ((threadIdx.x & 31) == 0 && a != 0.0) atomicAdd(sum, a);
}

__global__ void k_corr_count(int32_t *count) { *count = min(*count + 1, 2); }

// phi += |s d| z on the inside nodes.
__global__ void k_corr_add(int n, const float *__restrict__ z, const uint8_t *__restrict__ inside, const double *sum,
                           double *__restrict__ phi) {
    const double f = sqrt(sum[0]);
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        if (inside[p]) phi[p] += f * (double)z[p];
}

// Adam on the f32 master weights; writes the bf16 copy.
__global__ void k_adam(int n, float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, bf16 *__restrict__ w16, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
        w[i] = wi;
        w16[i] = __float2bfloat16_rn(wi);
    }
}

__global__ void k_to_bf16(int n, const float *__restrict__ a, bf16 *__restrict__ b) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = __float2bfloat16_rn(a[i]);
}

}  // namespace
}  // namespace oec

using namespace oec;

// ======================================================== host side
namespace {

struct Buffers {  // activation workspace (bf16 unless noted)
    bf16 *x16, *e0, *p1, *e1, *p2, *e2, *p3, *e3, *u2, *d2, *u1, *d1, *u0, *d0;
    bf16 *gd0, *gu0, *gd1, *gu1, *gd2, *gu2, *ge3, *gp3, *ge2, *gp2, *ge1, *gp1, *ge0;
    float *gz, *res;
    double *sums;
    int *err;  // set by a tensor-core convolution whose bounded wait gave up
};

size_t al(size_t b) { return (b + 255) & ~size_t(255); }

void levels_of(int nx, int ny, Level L[4]) {
    int h = ny, w = nx;
    for (int l = 0; l < 4; ++l) {
        L[l] = Level{h, w};
        h = (h + 1) / 2;
        w = (w + 1) / 2;
    }
}

size_t carve_buffers(void *base, int nx, int ny, bool training, Buffers *b) {
    Level L[4];
    levels_of(nx, ny, L);
    auto sz = [&](int l, int c) { return al(sizeof(bf16) * (size_t)L[l].h * L[l].w * c); };
    char *c = static_cast<char *>(base);
    size_t off = 0;
    auto take = [&](size_t bytes) -> void * {
        void *p = c ? c + off : nullptr;
        off += bytes;
        return p;
    };
    Buffers t{};
    t.err = (int *)take(256);
    t.x16 = (bf16 *)take(sz(0, 1));
    t.e0 = (bf16 *)take(sz(0, 16));
    t.p1 = (bf16 *)take(sz(1, 16));
    t.e1 = (bf16 *)take(sz(1, 32));
    t.p2 = (bf16 *)take(sz(2, 32));
    t.e2 = (bf16 *)take(sz(2, 64));
    t.p3 = (bf16 *)take(sz(3, 64));
    t.e3 = (bf16 *)take(sz(3, 64));
    t.u2 = (bf16 *)take(sz(2, 64));
    t.d2 = (bf16 *)take(sz(2, 32));
    t.u1 = (bf16 *)take(sz(1, 32));
    t.d1 = (bf16 *)take(sz(1, 16));
    t.u0 = (bf16 *)take(sz(0, 16));
    t.d0 = (bf16 *)take(sz(0, 16));
    if (training) {
        t.gd0 = (bf16 *)take(sz(0, 16));
        t.gu0 = (bf16 *)take(sz(0, 16));
        t.gd1 = (bf16 *)take(sz(1, 16));
        t.gu1 = (bf16 *)take(sz(1, 32));
        t.gd2 = (bf16 *)take(sz(2, 32));
        t.gu2 = (bf16 *)take(sz(2, 64));
        t.ge3 = (bf16 *)take(sz(3, 64));
        t.gp3 = (bf16 *)take(sz(3, 64));
        t.ge2 = (bf16 *)take(sz(2, 64));
        t.gp2 = (bf16 *)take(sz(2, 32));
        t.ge1 = (bf16 *)take(sz(1, 32));
        t.gp1 = (bf16 *)take(sz(1, 16));
        t.ge0 = (bf16 *)take(sz(0, 16));
        t.gz = (float *)take(al(sizeof(float) * (size_t)nx * ny));
        t.res = (float *)take(al(sizeof(float) * (size_t)nx * ny));
        t.sums = (double *)take(al(4 * sizeof(double)));
    }
    if (b) *b = t;
    return off;
}

int grid_for(size_t n, int per_sm = 8) { return persistent_grid((int64_t)((n + 255) / 256), per_sm); }

template <int CI, int CO>
int conv3_mma_sync(const Level &L, const bf16 *in, const bf16 *w, bf16 *out, cudaStream_t s) {
    constexpr int smem = conv_smem_bytes<CI, CO>();
    static std::atomic<int> attr[kMaxDevices];
    if (per_device_cached(attr, [] {
            return cudaFuncSetAttribute(k_conv3_mma<CI, CO>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) ==
                           cudaSuccess
                       ? 1
                       : 0;
        }) != 1)
        return OEC_ERR_CUDA;
    const int tiles = L.h * ((L.w + kTX - 1) / kTX);
    k_conv3_mma<CI, CO><<<persistent_grid(tiles, 2), 128, smem, s>>>(L.h, L.w, in, w, out);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

template <int CI, int CO>
int conv3_tcgen05(const Level &L, const bf16 *in, const bf16 *w, bf16 *out, int *err, cudaStream_t s) {
    using S = umma::ConvSmem<CI, CO>;
    // Resident CTAs per SM, per device: what the SM's shared memory holds,
    // capped by its 512 tensor-memory columns.  (The occupancy calculator
    // reports one CTA per SM for these kernels; the SM runs as many as its
    // shared memory allows -- 0.53 -> 0.31 ms per forward pass at 1026^2 --
    // and the cap keeps every CTA's column allocation satisfiable.)
    static std::atomic<int> per_sm_cache[kMaxDevices];
    const int per_sm = per_device_cached(per_sm_cache, [] {
        int dev = 0, sm_smem = 0, reserved = 0;
        if (cudaFuncSetAttribute(umma::k_conv3<CI, CO>, cudaFuncAttributeMaxDynamicSharedMemorySize, S::kBytes) !=
                cudaSuccess ||
            cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sm_smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess)
            return -1;
        const int by_smem = sm_smem / (S::kBytes + reserved);
        const int by_tmem = 512 / S::kCols;
        return by_smem < by_tmem ? by_smem : by_tmem;
    });
    if (per_sm < 1) return OEC_ERR_CUDA;
    const int tiles = L.h * ((L.w + umma::kM - 1) / umma::kM);
    umma::k_conv3<CI, CO><<<persistent_grid(tiles, per_sm), umma::kThreads, S::kBytes, s>>>(L.h, L.w, in, w, out,
                                                                                             err);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

// One 3x3 convolution by the kernel the network selects.
template <int CI, int CO>
int conv3(int kernel, const Level &L, const bf16 *in, const bf16 *w, bf16 *out, int *err, cudaStream_t s) {
    if (kernel == OEC_CNN_CONV_TCGEN05) return conv3_tcgen05<CI, CO>(L, in, w, out, err, s);
    return conv3_mma_sync<CI, CO>(L, in, w, out, s);
}

template <int C>
void pool(const Level &f, const Level &c, const bf16 *in, bf16 *out, cudaStream_t s) {
    k_pool<C><<<grid_for((size_t)c.h * c.w * C / 8), 256, 0, s>>>(f, c, in, out);
}

template <int C>
void up_add(const Level &f, const Level &c, float a, const bf16 *crs, const bf16 *skip, bf16 *out, cudaStream_t s) {
    k_up_add<C><<<grid_for((size_t)f.h * f.w * C / 8), 256, 0, s>>>(f, c, a, crs, skip, out);
}

template <int C>
void down_sum(const Level &f, const Level &c, const bf16 *in, bf16 *out, cudaStream_t s) {
    k_down_sum<C><<<grid_for((size_t)c.h * c.w * C / 8), 256, 0, s>>>(f, c, in, out);
}

void conv3_dw(const Level &L, int ci, int co, const bf16 *X, const bf16 *G, float *gW, cudaStream_t s) {
    const int kslices = (9 * ci + 63) / 64;
    int px = persistent_grid(((int64_t)L.h * L.w + 4095) / 4096, 2) / kslices;
    if (px < 1) px = 1;
    k_conv3_dw<<<dim3(px, kslices), 256, 0, s>>>(L.h, L.w, ci, co, X, G, gW);
}

bool valid_cnn(const oec_cnn_t *c) {
    return c && c->nx >= 3 && c->ny >= 3 && c->inside && c->w16 && c->act &&
           (c->conv_kernel == OEC_CNN_CONV_MMA_SYNC || c->conv_kernel == OEC_CNN_CONV_TCGEN05);
}

int forward(const oec_cnn_t *c, const float *x, Buffers &b, cudaStream_t s) {
    Level L[4];
    levels_of(c->nx, c->ny, L);
    const bf16 *w = reinterpret_cast<const bf16 *>(c->w16);
    const size_t n0 = (size_t)c->nx * c->ny;
    OEC_CUDA_TRY(cudaMemsetAsync(b.err, 0, sizeof(int), s));
    k_conv3_in1<<<dim3((L[0].w + kIn1TX - 1) / kIn1TX, (L[0].h + kIn1TY - 1) / kIn1TY), kIn1TX * kIn1TY, 0, s>>>(
        L[0].h, L[0].w, x, c->inside, w + conv_offset(0), b.e0, b.x16);
    OEC_LAUNCH_CHECK();
    pool<16>(L[0], L[1], b.e0, b.p1, s);
    int rc = conv3<16, 32>(c->conv_kernel, L[1], b.p1, w + conv_offset(1), b.e1, b.err, s);
    if (rc) return rc;
    pool<32>(L[1], L[2], b.e1, b.p2, s);
    if ((rc = conv3<32, 64>(c->conv_kernel, L[2], b.p2, w + conv_offset(2), b.e2, b.err, s))) return rc;
    pool<64>(L[2], L[3], b.e2, b.p3, s);
    if ((rc = conv3<64, 64>(c->conv_kernel, L[3], b.p3, w + conv_offset(3), b.e3, b.err, s))) return rc;
    up_add<64>(L[2], L[3], 1.f, b.e3, b.e2, b.u2, s);
    if ((rc = conv3<64, 32>(c->conv_kernel, L[2], b.u2, w + conv_offset(4), b.d2, b.err, s))) return rc;
    up_add<32>(L[1], L[2], 1.f, b.d2, b.e1, b.u1, s);
    if ((rc = conv3<32, 16>(c->conv_kernel, L[1], b.u1, w + conv_offset(5), b.d1, b.err, s))) return rc;
    up_add<16>(L[0], L[1], 1.f, b.d1, b.e0, b.u0, s);
    if ((rc = conv3<16, 16>(c->conv_kernel, L[0], b.u0, w + conv_offset(6), b.d0, b.err, s))) return rc;
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

}  // namespace

namespace oec {
int cnn_precond_apply(const void *ctx, const float *r_dev, float *z_dev, cudaStream_t s) {
    return oec_cnn_forward(static_cast<const oec_cnn_t *>(ctx), r_dev, z_dev, s);
}
}  // namespace oec

extern "C" int32_t oec_cnn_num_params(void) { return kNParams; }

extern "C" int oec_cnn_param_layout(int32_t *offsets, int32_t *shapes) {
    if (!offsets || !shapes) return OEC_ERR_INVALID;
    for (int i = 0; i < kNConv; ++i) {
        offsets[i] = conv_offset(i);
        shapes[3 * i] = conv_spec(i).co;
        shapes[3 * i + 1] = 9;
        shapes[3 * i + 2] = conv_spec(i).ci;
    }
    offsets[kNConv] = kOutOffset;
    shapes[3 * kNConv] = 1;
    shapes[3 * kNConv + 1] = 1;
    shapes[3 * kNConv + 2] = 16;
    offsets[kNConv + 1] = kNParams;
    return OEC_OK;
}

extern "C" int64_t oec_cnn_act_bytes(int32_t nx, int32_t ny, int32_t training) {
    if (nx < 3 || ny < 3) return -1;
    return (int64_t)carve_buffers(nullptr, nx, ny, training != 0, nullptr);
}

extern "C" int oec_cnn_forward(const oec_cnn_t *c, const float *x_dev, float *z_dev, void *stream) {
    if (!valid_cnn(c) || !x_dev || !z_dev) return OEC_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    Buffers b;
    carve_buffers(c->act, c->nx, c->ny, false, &b);
    int rc = forward(c, x_dev, b, s);
    if (rc) return rc;
    const bf16 *w = reinterpret_cast<const bf16 *>(c->w16);
    const size_t n0 = (size_t)c->nx * c->ny;
    k_conv_out<<<grid_for(n0), 256, 0, s>>>((int)n0, b.d0, w + kOutOffset, c->inside, z_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_cnn_status(const oec_cnn_t *c, int32_t *wait_timeouts_host, void *stream) {
    if (!valid_cnn(c) || !wait_timeouts_host) return OEC_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    Buffers b;
    carve_buffers(c->act, c->nx, c->ny, false, &b);
    OEC_CUDA_TRY(cudaMemcpyAsync(wait_timeouts_host, b.err, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    OEC_CUDA_TRY(cudaStreamSynchronize(s));
    return OEC_OK;
}

extern "C" int oec_cnn_train_step(const oec_cnn_t *c, const oec_stencil_t *op, const float *x_dev,
                                  const float *target_dev, float *z_dev, float *w32_dev, float *grad_dev,
                                  float *adam_m_dev, float *adam_v_dev, void *wt16_dev, float lr, int32_t step,
                                  int32_t update, double *loss_dev, void *stream) {
    if (!valid_cnn(c) || !x_dev || !z_dev || !grad_dev || !wt16_dev || !loss_dev) return OEC_ERR_INVALID;
    if (!op && !target_dev) return OEC_ERR_INVALID;
    if (op && (op->nx != c->nx || op->ny != c->ny || !op->ex32 || !op->ey32)) return OEC_ERR_INVALID;
    if (update && (!w32_dev || !adam_m_dev || !adam_v_dev || step < 1)) return OEC_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    Buffers b;
    carve_buffers(c->act, c->nx, c->ny, true, &b);
    Level L[4];
    levels_of(c->nx, c->ny, L);
    const size_t n0 = (size_t)c->nx * c->ny;
    bf16 *w = reinterpret_cast<bf16 *>(c->w16);
    bf16 *wt = reinterpret_cast<bf16 *>(wt16_dev);
    // flipped / transposed weights of the data gradients
    for (int i = 1; i < kNConv; ++i) {
        const ConvSpec sp = conv_spec(i);
        k_flip_transpose<<<grid_for((size_t)conv_params(i)), 256, 0, s>>>(sp.ci, sp.co, w + conv_offset(i),
                                                                          wt + conv_offset(i));
    }
    int rc = forward(c, x_dev, b, s);
    if (rc) return rc;
    k_conv_out<<<grid_for(n0), 256, 0, s>>>((int)n0, b.d0, w + kOutOffset, c->inside, z_dev);
    OEC_CUDA_TRY(cudaMemsetAsync(b.sums, 0, 4 * sizeof(double), s));
    if (op) {  // scale-free residual loss
        k_res_loss<<<grid_for(n0), 256, 0, s>>>((int)n0, c->nx, op->ex32, op->ey32, c->inside, z_dev, x_dev, b.res,
                                                 b.sums);
        k_res_combine<<<grid_for(n0), 256, 0, s>>>((int)n0, c->inside, x_dev, b.sums, b.res);
        k_res_grad<<<grid_for(n0), 256, 0, s>>>((int)n0, c->nx, op->ex32, op->ey32, c->inside, b.res, b.sums, b.gz);
        k_res_report<<<1, 1, 0, s>>>(b.sums, loss_dev);
    } else {   // supervised loss |z - t|^2 / |t|^2
        k_loss_sums<<<grid_for(n0), 256, 0, s>>>((int)n0, z_dev, target_dev, c->inside, b.sums);
        k_loss_grad<<<grid_for(n0), 256, 0, s>>>((int)n0, z_dev, target_dev, c->inside, b.sums, b.gz);
        OEC_CUDA_TRY(cudaMemcpyAsync(loss_dev, b.sums, 2 * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    // ---- backward
    OEC_CUDA_TRY(cudaMemsetAsync(grad_dev, 0, sizeof(float) * kNParams, s));
    k_conv_out_bwd<<<grid_for(n0), 256, 0, s>>>((int)n0, b.gz, b.d0, w + kOutOffset, c->inside, b.gd0,
                                                grad_dev + kOutOffset);
    // d0 = conv(u0)
    conv3_dw(L[0], 16, 16, b.u0, b.gd0, grad_dev + conv_offset(6), s);
    if ((rc = conv3<16, 16>(c->conv_kernel, L[0], b.gd0, wt + conv_offset(6), b.gu0, b.err, s))) return rc;
    // u0 = up(d1) + e0
    down_sum<16>(L[0], L[1], b.gu0, b.gd1, s);
    // d1 = conv(u1)
    conv3_dw(L[1], 32, 16, b.u1, b.gd1, grad_dev + conv_offset(5), s);
    if ((rc = conv3<16, 32>(c->conv_kernel, L[1], b.gd1, wt + conv_offset(5), b.gu1, b.err, s))) return rc;
    // u1 = up(d2) + e1
    down_sum<32>(L[1], L[2], b.gu1, b.gd2, s);
    // d2 = conv(u2)
    conv3_dw(L[2], 64, 32, b.u2, b.gd2, grad_dev + conv_offset(4), s);
    if ((rc = conv3<32, 64>(c->conv_kernel, L[2], b.gd2, wt + conv_offset(4), b.gu2, b.err, s))) return rc;
    // u2 = up(e3) + e2
    down_sum<64>(L[2], L[3], b.gu2, b.ge3, s);
    // e3 = conv(p3)
    conv3_dw(L[3], 64, 64, b.p3, b.ge3, grad_dev + conv_offset(3), s);
    if ((rc = conv3<64, 64>(c->conv_kernel, L[3], b.ge3, wt + conv_offset(3), b.gp3, b.err, s))) return rc;
    // p3 = pool(e2); e2 also feeds u2
    up_add<64>(L[2], L[3], 0.25f, b.gp3, b.gu2, b.ge2, s);
    conv3_dw(L[2], 32, 64, b.p2, b.ge2, grad_dev + conv_offset(2), s);
    if ((rc = conv3<64, 32>(c->conv_kernel, L[2], b.ge2, wt + conv_offset(2), b.gp2, b.err, s))) return rc;
    up_add<32>(L[1], L[2], 0.25f, b.gp2, b.gu1, b.ge1, s);
    conv3_dw(L[1], 16, 32, b.p1, b.ge1, grad_dev + conv_offset(1), s);
    if ((rc = conv3<32, 16>(c->conv_kernel, L[1], b.ge1, wt + conv_offset(1), b.gp1, b.err, s))) return rc;
    up_add<16>(L[0], L[1], 0.25f, b.gp1, b.gu0, b.ge0, s);
    conv3_dw(L[0], 1, 16, b.x16, b.ge0, grad_dev + conv_offset(0), s);
    OEC_LAUNCH_CHECK();
    if (update) {
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f / (1.f - powf(b1, (float)step)), c2 = 1.f / (1.f - powf(b2, (float)step));
        k_adam<<<grid_for(kNParams), 256, 0, s>>>(kNParams, w32_dev, grad_dev, adam_m_dev, adam_v_dev, w, lr, b1, b2,
                                                  1e-8f, c1, c2);
        OEC_LAUNCH_CHECK();
    }
    return OEC_OK;
}

extern "C" int oec_cnn_set_weights(const oec_cnn_t *c, const float *w32_dev, void *stream) {
    if (!c || !c->w16 || !w32_dev) return OEC_ERR_INVALID;
    k_to_bf16<<<grid_for(kNParams), 256, 0, as_stream(stream)>>>(kNParams, w32_dev, reinterpret_cast<bf16 *>(c->w16));
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int64_t oec_cnn_correct_work_bytes(int32_t nx, int32_t ny) {
    if (nx < 3 || ny < 3) return -1;
    return (int64_t)(al(sizeof(double) * (size_t)nx * ny) + 2 * al(sizeof(float) * (size_t)nx * ny) + 256);
}

extern "C" int oec_cnn_correct(const oec_cnn_t *c, double scale32, const double *q_dev, double *q_hist_dev,
                               int32_t *count_dev, double *phi_dev, void *work_dev, void *stream) {
    if (!valid_cnn(c) || !q_dev || !q_hist_dev || !count_dev || !phi_dev || !work_dev || !(scale32 > 0.0))
        return OEC_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    const size_t n0 = (size_t)c->nx * c->ny;
    char *w = static_cast<char *>(work_dev);
    double *d = reinterpret_cast<double *>(w);
    float *x = reinterpret_cast<float *>(w + al(sizeof(double) * n0));
    float *z = reinterpret_cast<float *>(w + al(sizeof(double) * n0) + al(sizeof(float) * n0));
    double *sum = reinterpret_cast<double *>(w + al(sizeof(double) * n0) + 2 * al(sizeof(float) * n0));
    OEC_CUDA_TRY(cudaMemsetAsync(sum, 0, sizeof(double), s));
    k_corr_diff<<<grid_for(n0), 256, 0, s>>>((int)n0, q_dev, q_hist_dev, q_hist_dev + n0, count_dev, c->inside,
                                             scale32, d, sum);
    k_corr_count<<<1, 1, 0, s>>>(count_dev);
    k_ws_scale<<<grid_for(n0), 256, 0, s>>>((int)n0, d, c->inside, scale32, sum, x);
    OEC_LAUNCH_CHECK();
    int rc = oec_cnn_forward(c, x, z, stream);
    if (rc) return rc;
    k_corr_add<<<grid_for(n0), 256, 0, s>>>((int)n0, z, c->inside, sum, phi_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int64_t oec_cnn_warm_start_work_bytes(int32_t nx, int32_t ny) {
    if (nx < 3 || ny < 3) return -1;
    return (int64_t)(2 * al(sizeof(float) * (size_t)nx * ny) + 256);
}

extern "C" int oec_cnn_warm_start(const oec_cnn_t *c, double scale32, const double *q_dev, double *phi_dev,
                                  void *work_dev, void *stream) {
    if (!valid_cnn(c) || !q_dev || !phi_dev || !work_dev || !(scale32 > 0.0)) return OEC_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    const size_t n0 = (size_t)c->nx * c->ny;
    char *w = static_cast<char *>(work_dev);
    float *x = reinterpret_cast<float *>(w);
    float *z = reinterpret_cast<float *>(w + al(sizeof(float) * n0));
    double *sum = reinterpret_cast<double *>(w + 2 * al(sizeof(float) * n0));
    OEC_CUDA_TRY(cudaMemsetAsync(sum, 0, sizeof(double), s));
    k_ws_norm<<<grid_for(n0), 256, 0, s>>>((int)n0, q_dev, c->inside, scale32, sum);
    k_ws_scale<<<grid_for(n0), 256, 0, s>>>((int)n0, q_dev, c->inside, scale32, sum, x);
    OEC_LAUNCH_CHECK();
    int rc = oec_cnn_forward(c, x, z, stream);
    if (rc) return rc;
    k_ws_out<<<grid_for(n0), 256, 0, s>>>((int)n0, z, c->inside, sum, phi_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}
