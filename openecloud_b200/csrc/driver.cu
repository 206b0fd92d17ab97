// driver.cu -- small per-step kernels of the device-resident time loop:
// the Poisson right-hand side (fixed-point electron charge + beam imprint),
// the step counter and the per-step history (macro count and line density).
//
// Reference: example01_basic.py:56-57 (histories) and :81 (q = chargeOnGrid +
// beam.getCharge(ii*dt)); beam.py:68-78 / :129-136 for the beam factor.
#include <stdint.h>

#include "oec_common.cuh"

namespace oec {
namespace {

// rho = q_e * fix / wscale + table[step] * profile
__global__ void k_rhs(const long long *__restrict__ fix, int G, const double *wscale_p, double charge,
                      const double *__restrict__ profile, const double *__restrict__ table, const int32_t *step,
                      int table_len, double *__restrict__ rho) {
    double f = charge / *wscale_p;
    int s = *step;
    double b = (table && profile && s >= 0 && s < table_len) ? table[s] : 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < G; i += gridDim.x * blockDim.x)
        rho[i] = (double)fix[i] * f + (b != 0.0 ? b * profile[i] : 0.0);
}

// history[step] = (count, sum w); then ++step
// Per-CTA partial sums of w (first level of the history reduction).
constexpr int kHistCtas = 256;

__global__ void k_history_partial(const int32_t *count, const float *__restrict__ w, double *__restrict__ partial) {
    __shared__ double red[32];
    const int n = *count;
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += (double)w[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFullMask, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFullMask, s, o);
        if (threadIdx.x == 0) partial[blockIdx.x] = s;
    }
}

// Second level: one warp sums the partials in a fixed order (deterministic).
__global__ void k_history(const int32_t *count, const double *__restrict__ partial, int nparts, int32_t *step,
                          int hist_len, double *__restrict__ hist_w, int32_t *__restrict__ hist_n) {
    double s = 0.0;
    for (int i = threadIdx.x; i < nparts; i += 32) s += partial[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFullMask, s, o);
    if (threadIdx.x == 0) {
        const int k = *step;
        if (k >= 0 && k < hist_len) {
            hist_w[k] = s;
            hist_n[k] = *count;
        }
    }
}

__global__ void k_step_advance(int32_t *step) { *step += 1; }

}  // namespace
}  // namespace oec

using namespace oec;

extern "C" int oec_rhs_with_beam(const oec_grid_t *grid, const int64_t *rho_fix_dev, const double *wscale_dev,
                                 double particle_charge, const double *profile_dev, const double *table_dev,
                                 const int32_t *step_dev, int32_t table_len, double *rho_dev, void *stream) {
    if (!grid || !rho_fix_dev || !wscale_dev || !step_dev || !rho_dev) return OEC_ERR_INVALID;
    int G = grid->nx * grid->ny;
    k_rhs<<<persistent_grid((G + 255) / 256, 8), 256, 0, as_stream(stream)>>>(
        reinterpret_cast<const long long *>(rho_fix_dev), G, wscale_dev, particle_charge, profile_dev, table_dev,
        step_dev, table_len, rho_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_history(const oec_particles_t *p, int32_t *step_dev, int32_t hist_len, double *hist_w_dev,
                           int32_t *hist_n_dev, double *scratch_dev, void *stream) {
    if (!p || !step_dev || !hist_w_dev || !hist_n_dev || !scratch_dev) return OEC_ERR_INVALID;
    const int g = persistent_grid((p->capacity + 255) / 256, 2) < kHistCtas ? persistent_grid((p->capacity + 255) / 256, 2)
                                                                            : kHistCtas;
    k_history_partial<<<g, 256, 0, as_stream(stream)>>>(p->count, p->w, scratch_dev);
    k_history<<<1, 32, 0, as_stream(stream)>>>(p->count, scratch_dev, g, step_dev, hist_len, hist_w_dev, hist_n_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_step_advance(int32_t *step_dev, void *stream) {
    if (!step_dev) return OEC_ERR_INVALID;
    k_step_advance<<<1, 1, 0, as_stream(stream)>>>(step_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}
