// cnn.cu -- the learned Poisson preconditioner (placeholder until the network
// kernels land): cnn_precond_apply reports that no network is available.
#include "oec_common.cuh"

namespace oec {
int cnn_precond_apply(const void *ctx, const float *r_dev, float *z_dev, cudaStream_t s) {
    (void)ctx;
    (void)r_dev;
    (void)z_dev;
    (void)s;
    return OEC_ERR_INVALID;
}
}  // namespace oec
