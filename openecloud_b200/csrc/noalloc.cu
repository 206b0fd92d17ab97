// noalloc.cu -- charge deposit for callers that cannot allocate device memory.
//
// Some hosts of this library cannot call cudaMalloc: an application that owns
// the whole device memory budget through its own pool and forbids libraries
// from allocating, or an embedding that runs with a fixed memory plan decided
// before the simulation starts.  For them this file offers one entry point,
// oec_deposit_charge_noalloc, that computes the same float64 charge per node
// as oec_deposit_scale + oec_deposit + oec_deposit_finalize but keeps its
// scratch -- the int64 fixed-point node grid and the fixed-point scale -- in
// file-scope device arrays instead of caller-provided buffers.  The caller
// still passes the particles (input) and the charge array (output).
//
// Limits and sharing:
//  * the scratch grid holds at most kNoAllocMaxNodes nodes (extended grid
//    nxExt*nyExt); larger grids are rejected with OEC_ERR_CAPACITY;
//  * every GPU that loads the library holds the arrays (about 8.8 MB) until
//    the process exits;
//  * all calls share the arrays: calls whose work overlaps on the GPU (on
//    different streams, or from different threads) race on the scratch and
//    corrupt each other's result; serialise them.  Each call clears the part
//    of the grid it uses before depositing, so the contents left by an
//    earlier call never leak into a result;
//  * the device address of the arrays is looked up once per device, with
//    that device current, by the first call made on it
//    (cudaGetSymbolAddress); make that first call before any stream capture.
#include <stdint.h>

#include <mutex>

#include "oec_common.cuh"

namespace {

constexpr int kNoAllocMaxNodes = 1100000;  // covers a 1024x1024 grid (1026^2 extended nodes)
constexpr int kMaxDevices = 64;

__device__ __align__(256) long long g_noalloc_rho_fix[kNoAllocMaxNodes];
__device__ __align__(256) double g_noalloc_wscale[4];

// Per-device addresses of the two arrays (host code only sees their device
// addresses through cudaGetSymbolAddress; the symbols themselves are host
// stand-ins).
struct NoAllocAddr {
    int64_t *rho_fix;
    double *wscale;
    bool ready;
};
NoAllocAddr g_addr[kMaxDevices];
std::mutex g_addr_mu;  // guards g_addr: first calls may come from several threads

// Copies the device's scratch addresses into *out, looking them up on the
// first call made with that device current.
int noalloc_setup(int dev, NoAllocAddr *out) {
    if (dev < 0 || dev >= kMaxDevices) return OEC_ERR_INVALID;
    std::lock_guard<std::mutex> lock(g_addr_mu);
    if (!g_addr[dev].ready) {
        void *rho = nullptr, *scale = nullptr;
        if (cudaGetSymbolAddress(&rho, g_noalloc_rho_fix) != cudaSuccess) return OEC_ERR_CUDA;
        if (cudaGetSymbolAddress(&scale, g_noalloc_wscale) != cudaSuccess) return OEC_ERR_CUDA;
        g_addr[dev].rho_fix = static_cast<int64_t *>(rho);
        g_addr[dev].wscale = static_cast<double *>(scale);
        g_addr[dev].ready = true;
    }
    *out = g_addr[dev];
    return OEC_OK;
}

}  // namespace

extern "C" int oec_deposit_charge_noalloc(const oec_grid_t *grid, const oec_particles_t *p, double particle_charge,
                                          double *rho_dev, void *stream) {
    if (!grid || !p || !rho_dev || grid->nx < 3 || grid->ny < 3) return OEC_ERR_INVALID;
    if ((int64_t)grid->nx * grid->ny > kNoAllocMaxNodes) return OEC_ERR_CAPACITY;
    int dev = 0;
    OEC_CUDA_TRY(cudaGetDevice(&dev));
    NoAllocAddr a;
    int rc = noalloc_setup(dev, &a);
    if (rc != OEC_OK) return rc;
    // the scale is recomputed and the grid cleared (zero_first = 1) on every
    // call, so nothing of an earlier call's scratch reaches this result
    rc = oec_deposit_scale(p, a.wscale, stream);
    if (rc != OEC_OK) return rc;
    rc = oec_deposit(grid, p, a.rho_fix, a.wscale, 1, nullptr, stream);
    if (rc != OEC_OK) return rc;
    return oec_deposit_finalize(grid, a.rho_fix, a.wscale, particle_charge, rho_dev, stream);
}
