// diag.cu -- field and diagnostic kernels outside the per-step loop:
// the multipole magnetic field on the grid nodes and the mean kinetic energy
// of the particle store.
//
// Reference: magneticField.pyx:23-59 (multipoleExpansion), util.pyx:8-20
// (averageEnergy).
#include <math.h>
#include <stdint.h>

#include "oec_common.cuh"

namespace oec {
namespace {

constexpr int kMaxMultipoleOrder = 32;

struct Multipoles {
    int n;
    double normal[kMaxMultipoleOrder], skew[kMaxMultipoleOrder];
};

// B at node (i, j): in polar coordinates r, phi of the node (phi in
// [0, 2 pi)), B_r = sum_k r^k (-skew_k cos((k+1) phi) + normal_k sin((k+1) phi)),
// B_phi = sum_k r^k (skew_k sin((k+1) phi) + normal_k cos((k+1) phi)); stored
// as [Bx | By | Bz = 0] (magneticField.pyx:44-58).
__global__ void k_multipole(int nx, int ny, const double *__restrict__ xm, const double *__restrict__ ym,
                            Multipoles m, double *__restrict__ b) {
    const int np = nx * ny;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < np; idx += gridDim.x * blockDim.x) {
        const int jj = idx / nx, ii = idx - jj * nx;
        const double x = xm[ii], y = ym[jj];
        const double r = sqrt(x * x + y * y);
        double phi = atan2(y, x);
        if (phi < 0) phi += 2.0 * M_PI;
        double br = 0.0, bphi = 0.0, rk = 1.0;
        for (int k = 0; k < m.n; ++k) {
            double sk, ck;
            sincos((k + 1) * phi, &sk, &ck);
            br += rk * (-m.skew[k] * ck + m.normal[k] * sk);
            bphi += rk * (m.skew[k] * sk + m.normal[k] * ck);
            rk *= r;
        }
        double sp, cp;
        sincos(phi, &sp, &cp);
        b[idx] = br * cp - bphi * sp;
        b[idx + np] = br * sp + bphi * cp;
        b[idx + 2 * np] = 0.0;
    }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
    return v;
}

// out[0] += sum |v|^2 w, out[1] += sum w over the store (util.pyx:15-17).
__global__ void __launch_bounds__(256) k_energy_sums(const float *__restrict__ vx, const float *__restrict__ vy,
                                                     const float *__restrict__ vz, const float *__restrict__ w,
                                                     const int32_t *count, int64_t capacity, double *out) {
    __shared__ double red[2][8];
    const int n = (int)min((int64_t)*count, capacity);
    double e = 0.0, s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double a = vx[i], b = vy[i], c = vz[i], ww = w[i];
        e += (a * a + b * b + c * c) * ww;
        s += ww;
    }
    e = warp_sum(e);
    s = warp_sum(s);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][wid] = e;
        red[1][wid] = s;
    }
    __syncthreads();
    if (wid == 0) {
        e = lane < 8 ? red[0][lane] : 0.0;
        s = lane < 8 ? red[1][lane] : 0.0;
        e = warp_sum(e);
        s = warp_sum(s);
        if (lane == 0) {
            atomicAdd(out, e);
            atomicAdd(out + 1, s);
        }
    }
}

}  // namespace
}  // namespace oec

using namespace oec;

extern "C" int oec_multipole_field(int32_t nx, int32_t ny, const double *xmesh_dev, const double *ymesh_dev,
                                   const double *normal, int32_t n_normal, const double *skew, int32_t n_skew,
                                   double *b_dev, void *stream) {
    if (nx < 1 || ny < 1 || !xmesh_dev || !ymesh_dev || !b_dev || n_normal < 0 ||
        n_normal > kMaxMultipoleOrder || n_skew < 0 || (n_normal && !normal) || (n_skew && !skew))
        return OEC_ERR_INVALID;
    Multipoles m{};
    m.n = n_normal;
    for (int k = 0; k < n_normal; ++k) {
        m.normal[k] = normal[k];
        // a shorter skew list is padded with zeros, a longer one cut to the
        // order of the normal list (magneticField.pyx:38-42, :50)
        m.skew[k] = k < n_skew ? skew[k] : 0.0;
    }
    const int64_t np = (int64_t)nx * ny;
    k_multipole<<<persistent_grid((np + 255) / 256, 4), 256, 0, as_stream(stream)>>>(nx, ny, xmesh_dev, ymesh_dev, m,
                                                                                      b_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_average_energy_sums(const oec_particles_t *p, double *sums_dev, void *stream) {
    if (!p || !p->vx || !p->vy || !p->vz || !p->w || !p->count || p->capacity < 0 || !sums_dev)
        return OEC_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    OEC_CUDA_TRY(cudaMemsetAsync(sums_dev, 0, 2 * sizeof(double), s));
    k_energy_sums<<<persistent_grid((p->capacity + 255) / 256, 4), 256, 0, s>>>(p->vx, p->vy, p->vz, p->w, p->count,
                                                                                p->capacity, sums_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}
