// session.cu -- a context and a buildup run that own their device memory,
// streams and graph, for hosts that drive the library without any other
// GPU framework (a Cython or C host that binds only this ABI).
//
// The reference's objects own their arrays (numpy, particles.pyx:14-197,
// poissonSolver.pyx:33-67) and its example loop calls them once per step
// (example01_basic.py:52-97).  Here:
//  * oec_ctx_t is one device, one CUDA stream, one device status block and a
//    list of device allocations freed with the context;
//  * oec_run_t is one buildup run -- the particle store, the grid and its
//    boundary, the LU factors and the field operator, the beam tables, the
//    Furman emitter and every work area of the step -- allocated in its
//    context from host arrays the caller prepares (geometry, factors: the
//    host-side setup of the reference); oec_run_steps advances it by the
//    launch sequence of one time step (rhs + beam, LU solve, E, field table,
//    fused push/deposit, absorbed set, wall rows, emission, refill,
//    history), replayed from a CUDA graph the run captures once, with the
//    reference's globalRandom (particleManagement.pyx:35-67) at its cadence.
// Every entry point returns an OEC status; nothing aborts.  A run and its
// context are used from one host thread at a time.
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "oec_common.cuh"

struct oec_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    oec_status_t *status = nullptr;  // device
    std::vector<void *> allocs;
    std::mutex mu;
};

namespace {

// Allocates `bytes` of zeroed device memory owned by the context.
int ctx_alloc(oec_ctx *c, size_t bytes, void **out) {
    *out = nullptr;
    if (bytes == 0) bytes = 16;
    void *p = nullptr;
    OEC_CUDA_TRY(cudaSetDevice(c->device));
    OEC_CUDA_TRY(cudaMalloc(&p, bytes));
    if (cudaMemsetAsync(p, 0, bytes, c->stream) != cudaSuccess) {
        cudaFree(p);
        return OEC_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lock(c->mu);
    c->allocs.push_back(p);
    *out = p;
    return OEC_OK;
}

template <class T>
int ctx_array(oec_ctx *c, size_t n, T **out) {
    void *p = nullptr;
    int rc = ctx_alloc(c, n * sizeof(T), &p);
    *out = static_cast<T *>(p);
    return rc;
}

// A device copy of a host array (n elements), owned by the context.
template <class T>
int ctx_upload(oec_ctx *c, const T *host, size_t n, T **out) {
    *out = nullptr;
    if (n == 0) return ctx_array(c, 1, out);
    if (!host) return OEC_ERR_INVALID;
    OEC_TRY(ctx_array(c, n, out));
    OEC_CUDA_TRY(cudaMemcpyAsync(*out, host, n * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    return OEC_OK;
}

size_t round_up(size_t n, size_t m) { return (n + m - 1) / m * m; }

}  // namespace

struct oec_run {
    oec_ctx *ctx = nullptr;
    oec_run_desc_t d{};
    oec_boundary_t bnd{};
    oec_particles_t p{};
    oec_particles_t tmp{};      // scratch store of the shifting add/remove rules
    int32_t *array_len = nullptr;  // row count of the reference's particle array
    uint32_t *mask = nullptr;
    int64_t mask_words = 0;
    int64_t *rho_fix = nullptr;
    double *wscale = nullptr, *rho = nullptr, *phi = nullptr, *efield = nullptr, *lu_work = nullptr;
    float *etab = nullptr;
    oec_lu_t lu{};
    std::vector<int32_t> l_level_ptr, u_level_ptr;
    std::vector<int8_t> l_lanes, u_lanes;
    int32_t *e_ptr = nullptr, *e_idx = nullptr;
    double *e_val = nullptr;
    int32_t *index = nullptr, *n_abs = nullptr, *abs_scratch = nullptr;
    double *rows = nullptr, *normals = nullptr;
    void *em_work = nullptr;
    double *em_out = nullptr;
    int32_t em_out_cap = 0, *n_out = nullptr;
    double *profile = nullptr, *table = nullptr;
    int32_t *step = nullptr, *hist_n = nullptr, *n_add = nullptr, *fails = nullptr;
    double *hist_w = nullptr, *hist_scratch = nullptr, *clone_rows = nullptr;
    double *stage = nullptr;  // rows for oec_run_get_rows (allocated on first use)
    int64_t steps_done = 0;
    uint32_t manage_calls = 0;
    cudaGraphExec_t graph = nullptr;
};

namespace {

// The launches of one time step (Buildup._launch_step of the Python driver;
// example01_basic.py:66-97).
int launch_step(oec_run *r) {
    cudaStream_t s = r->ctx->stream;
    const oec_run_desc_t &d = r->d;
    oec_status_t *st = r->ctx->status;
    const int32_t G = d.grid.nx * d.grid.ny;
    OEC_TRY(oec_rhs_with_beam(&d.grid, r->rho_fix, r->wscale, d.charge, r->profile, r->table, r->step, d.table_len,
                              r->rho, s));
    OEC_TRY(oec_lu_solve(&r->lu, r->rho, r->phi, r->lu_work, s));
    OEC_TRY(oec_spmv_csr(2 * G, r->e_ptr, r->e_idx, r->e_val, r->phi, r->efield, s));
    OEC_TRY(oec_field_prepare(&d.grid, r->efield, 2, r->etab, s));
    OEC_TRY(oec_push_gather(&d.grid, &r->p, r->etab, nullptr, d.bconst, d.dt, d.charge / d.mass, d.type_b, &r->bnd,
                            r->mask, r->rho_fix, r->wscale, st, s));
    OEC_TRY(oec_absorbed_index(&r->p, r->mask, r->index, (int32_t)d.capacity, r->n_abs, r->abs_scratch, st, s));
    OEC_TRY(oec_save_absorbed(&d.grid, &r->p, r->index, r->n_abs, d.abs_cap, r->rows, s));
    OEC_TRY(oec_wall_interaction(&d.grid, &r->bnd, d.dt, r->rows, r->n_abs, d.abs_cap, r->normals, st, s));
    OEC_TRY(oec_furman_emit(&d.furman, r->rows, r->normals, r->n_abs, d.abs_cap, r->index, d.emit_seed, 0, r->step,
                            nullptr, r->em_work, r->em_out, r->em_out_cap, r->n_out, st, s));
    OEC_TRY(oec_add_remove(&d.grid, &r->p, &r->tmp, r->mask, r->index, r->n_abs, (int32_t)d.capacity, r->em_out,
                           r->n_out, r->em_out_cap, r->array_len, r->rho_fix, r->wscale, st, s));
    OEC_TRY(oec_step_advance(r->step, s));
    OEC_TRY(oec_history(&r->p, r->step, d.table_len, r->hist_w, r->hist_n, r->hist_scratch, s));
    return OEC_OK;
}

// Fixed-point scale from the current weights and a full deposit.
int prepare_deposit(oec_run *r) {
    cudaStream_t s = r->ctx->stream;
    OEC_TRY(oec_deposit_scale(&r->p, r->wscale, s));
    return oec_deposit(&r->d.grid, &r->p, r->rho_fix, r->wscale, 1, r->ctx->status, s);
}

int read_count(oec_run *r, int32_t *n) {
    OEC_CUDA_TRY(cudaMemcpyAsync(n, r->p.count, sizeof(int32_t), cudaMemcpyDeviceToHost, r->ctx->stream));
    OEC_CUDA_TRY(cudaStreamSynchronize(r->ctx->stream));
    return OEC_OK;
}

// globalRandom (particleManagement.pyx:35-67) toward the run's target when
// the count left the +-5 % band (example01_basic.py:62-64), then a fresh
// deposit scale and deposit.
int manage(oec_run *r) {
    const oec_run_desc_t &d = r->d;
    cudaStream_t s = r->ctx->stream;
    int32_t n = 0;
    OEC_TRY(read_count(r, &n));
    if (!(n > 1.05 * d.target || n < 0.95 * d.target) || n == 0) return OEC_OK;
    const uint32_t call = ++r->manage_calls;
    const uint64_t seed = d.manage_seed + (uint64_t)r->steps_done;
    const double factor = (double)n / (double)d.target;
    OEC_TRY(oec_scale_weights(&r->p, factor, s));
    int32_t n_add = 0;
    OEC_CUDA_TRY(cudaMemsetAsync(r->fails, 0, sizeof(int32_t), s));
    if (n > d.target) {
        OEC_TRY(oec_roulette_select(n, n - d.target, r->mask, r->mask_words, seed, call, r->fails, s));
        int32_t fails = 0;
        OEC_CUDA_TRY(cudaMemcpyAsync(&fails, r->fails, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        OEC_CUDA_TRY(cudaStreamSynchronize(s));
        if (fails) return OEC_ERR_NOT_CONVERGED;
    } else {
        n_add = d.target - n;
        OEC_TRY(oec_clone_rows(&d.grid, &r->p, n, n_add, seed, call, r->clone_rows, s));
        OEC_TRY(oec_roulette_select(0, 0, r->mask, r->mask_words, 0, 0, r->fails, s));  // clears the bits
    }
    OEC_CUDA_TRY(cudaMemcpyAsync(r->n_add, &n_add, sizeof(int32_t), cudaMemcpyHostToDevice, s));
    OEC_TRY(oec_absorbed_index(&r->p, r->mask, r->index, (int32_t)d.capacity, r->n_abs, r->abs_scratch, nullptr, s));
    OEC_TRY(oec_add_remove(&d.grid, &r->p, &r->tmp, r->mask, r->index, r->n_abs, (int32_t)d.capacity,
                           r->clone_rows, r->n_add, d.target, r->array_len, nullptr, nullptr, r->ctx->status, s));
    OEC_CUDA_TRY(cudaStreamSynchronize(s));  // n_add lives on this stack frame
    return prepare_deposit(r);
}

// Replays n steps from the run's step graph (captured on first use).
int replay(oec_run *r, int n, bool use_graph) {
    cudaStream_t s = r->ctx->stream;
    if (!use_graph) {
        for (int k = 0; k < n; ++k) OEC_TRY(launch_step(r));
        return OEC_OK;
    }
    if (!r->graph) {
        OEC_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        const int rc = launch_step(r);
        cudaGraph_t g = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(s, &g);
        if (rc != OEC_OK || ec != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return rc != OEC_OK ? rc : OEC_ERR_CUDA;
        }
        const cudaError_t ei = cudaGraphInstantiate(&r->graph, g, 0);
        cudaGraphDestroy(g);
        OEC_CUDA_TRY(ei);
    }
    for (int k = 0; k < n; ++k) OEC_CUDA_TRY(cudaGraphLaunch(r->graph, s));
    return OEC_OK;
}

bool valid_desc(const oec_run_desc_t *d) {
    const oec_lu_host_t &L = d->lu;
    return d && d->grid.nx >= 3 && d->grid.ny >= 3 && (int64_t)d->grid.nx * d->grid.ny < (1 << 23) &&
           d->capacity >= 1024 && d->capacity <= INT32_MAX && d->abs_cap >= 1 && d->abs_cap <= d->capacity &&
           d->n_rows >= 0 && d->n_rows <= d->capacity && (d->n_rows == 0 || d->rows) && d->table_len >= 1 &&
           d->beam_table && d->beam_profile && d->target >= 1 && d->management_every >= 1 &&
           (d->boundary_kind == OEC_BOUNDARY_RECT || d->boundary_kind == OEC_BOUNDARY_ELLIPSE) &&
           (d->type_b == 0 || d->type_b == 1) && d->mass > 0 && L.n >= 1 && L.head >= 0 && L.head <= L.n &&
           L.n_nodes == d->grid.nx * d->grid.ny && L.l_level_ptr && L.u_level_ptr && d->e_ptr && d->e_idx &&
           d->e_val && L.rhs_node && L.sol_src && L.sol_node;
}

int create_run(oec_ctx *c, const oec_run_desc_t *d, oec_run *r) {
    r->ctx = c;
    r->d = *d;
    const int64_t cap = round_up((size_t)d->capacity, 1024);
    r->d.capacity = cap;
    const int32_t G = d->grid.nx * d->grid.ny;
    // particle store (16-byte aligned SoA: cudaMalloc gives 256 bytes)
    OEC_TRY(ctx_array(c, cap, &r->p.cell));
    float **f[] = {&r->p.ox, &r->p.oy, &r->p.vx, &r->p.vy, &r->p.vz, &r->p.w};
    for (float **a : f) OEC_TRY(ctx_array(c, cap, a));
    OEC_TRY(ctx_array(c, 1, &r->p.count));
    r->p.capacity = cap;
    OEC_TRY(ctx_array(c, cap, &r->tmp.cell));
    float **ft[] = {&r->tmp.ox, &r->tmp.oy, &r->tmp.vx, &r->tmp.vy, &r->tmp.vz, &r->tmp.w};
    for (float **a : ft) OEC_TRY(ctx_array(c, cap, a));
    r->tmp.count = r->p.count;
    r->tmp.capacity = cap;
    OEC_TRY(ctx_array(c, 1, &r->array_len));
    r->mask_words = cap / 32;
    OEC_TRY(ctx_array(c, r->mask_words, &r->mask));
    OEC_TRY(ctx_array(c, G, &r->rho_fix));
    OEC_TRY(ctx_array(c, 1, &r->wscale));
    OEC_TRY(ctx_array(c, G, &r->rho));
    OEC_TRY(ctx_array(c, G, &r->phi));
    OEC_TRY(ctx_array(c, 2 * (size_t)G, &r->efield));
    OEC_TRY(ctx_array(c, 8 * (size_t)G, &r->etab));
    // boundary (rect / ellipse: no arrays)
    r->bnd.kind = d->boundary_kind;
    // LU factors (host arrays of the host-side setup) and the field operator
    const oec_lu_host_t &L = d->lu;
    const int32_t m = L.n - L.head;
    r->lu.n = L.n;
    r->lu.head = L.head;
    r->lu.n_nodes = L.n_nodes;
    r->lu.head_path = L.head_path;
    int32_t *i32;
    double *f64;
    OEC_TRY(ctx_upload(c, L.rhs_node, L.n, &i32)); r->lu.rhs_node = i32;
    OEC_TRY(ctx_upload(c, L.sol_src, L.n, &i32)); r->lu.sol_src = i32;
    OEC_TRY(ctx_upload(c, L.sol_node, L.n, &i32)); r->lu.sol_node = i32;
    r->lu.l_nlevels = L.l_nlevels;
    r->lu.u_nlevels = L.u_nlevels;
    r->l_level_ptr.assign(L.l_level_ptr, L.l_level_ptr + L.l_nlevels + 1);
    r->u_level_ptr.assign(L.u_level_ptr, L.u_level_ptr + L.u_nlevels + 1);
    r->lu.l_level_ptr = r->l_level_ptr.data();
    r->lu.u_level_ptr = r->u_level_ptr.data();
    if (L.l_level_lanes) {
        r->l_lanes.assign(L.l_level_lanes, L.l_level_lanes + L.l_nlevels);
        r->lu.l_level_lanes = r->l_lanes.data();
    }
    if (L.u_level_lanes) {
        r->u_lanes.assign(L.u_level_lanes, L.u_level_lanes + L.u_nlevels);
        r->lu.u_level_lanes = r->u_lanes.data();
    }
    const int32_t h = L.head;
    OEC_TRY(ctx_upload(c, L.l_rows, h, &i32)); r->lu.l_rows = i32;
    OEC_TRY(ctx_upload(c, L.l_ptr, (size_t)h + 1, &i32)); r->lu.l_ptr = i32;
    const int32_t lnnz = L.l_ptr ? L.l_ptr[h] : 0, unnz = L.u_ptr ? L.u_ptr[h] : 0;
    OEC_TRY(ctx_upload(c, L.l_idx, lnnz, &i32)); r->lu.l_idx = i32;
    OEC_TRY(ctx_upload(c, L.l_val, lnnz, &f64)); r->lu.l_val = f64;
    OEC_TRY(ctx_upload(c, L.u_rows, h, &i32)); r->lu.u_rows = i32;
    OEC_TRY(ctx_upload(c, L.u_ptr, (size_t)h + 1, &i32)); r->lu.u_ptr = i32;
    OEC_TRY(ctx_upload(c, L.u_idx, unnz, &i32)); r->lu.u_idx = i32;
    OEC_TRY(ctx_upload(c, L.u_val, unnz, &f64)); r->lu.u_val = f64;
    OEC_TRY(ctx_upload(c, L.u_diag, h, &f64)); r->lu.u_diag = f64;
    if (m > 0) {
        const int32_t cnnz = L.lc_ptr[m];
        OEC_TRY(ctx_upload(c, L.lc_ptr, (size_t)m + 1, &i32)); r->lu.lc_ptr = i32;
        OEC_TRY(ctx_upload(c, L.lc_idx, cnnz, &i32)); r->lu.lc_idx = i32;
        OEC_TRY(ctx_upload(c, L.lc_val, cnnz, &f64)); r->lu.lc_val = f64;
        OEC_TRY(ctx_upload(c, L.tl_inv, (size_t)m * m, &f64)); r->lu.tl_inv = f64;
        OEC_TRY(ctx_upload(c, L.tu_inv, (size_t)m * m, &f64)); r->lu.tu_inv = f64;
    }
    OEC_TRY(ctx_array(c, (size_t)L.n + m + 1, &r->lu_work));
    const int32_t enz = d->e_ptr[2 * G];
    OEC_TRY(ctx_upload(c, d->e_ptr, 2 * (size_t)G + 1, &r->e_ptr));
    OEC_TRY(ctx_upload(c, d->e_idx, enz, &r->e_idx));
    OEC_TRY(ctx_upload(c, d->e_val, enz, &r->e_val));
    // absorbed set, wall rows, emission
    OEC_TRY(ctx_array(c, cap, &r->index));
    OEC_TRY(ctx_array(c, 1, &r->n_abs));
    OEC_TRY(ctx_array(c, 1024, &r->abs_scratch));
    OEC_TRY(ctx_array(c, 6 * (size_t)d->abs_cap, &r->rows));
    OEC_TRY(ctx_array(c, 2 * (size_t)d->abs_cap, &r->normals));
    const int64_t wb = oec_furman_work_bytes(d->abs_cap);
    if (wb < 0) return OEC_ERR_INVALID;
    OEC_TRY(ctx_alloc(c, (size_t)wb, &r->em_work));
    r->em_out_cap = d->furman.m * d->abs_cap + 1;
    OEC_TRY(ctx_array(c, 6 * (size_t)r->em_out_cap, &r->em_out));
    OEC_TRY(ctx_array(c, 1, &r->n_out));
    // beam, step counter, histories, management buffers
    OEC_TRY(ctx_upload(c, d->beam_profile, G, &r->profile));
    OEC_TRY(ctx_upload(c, d->beam_table, d->table_len, &r->table));
    OEC_TRY(ctx_array(c, 1, &r->step));
    OEC_TRY(ctx_array(c, d->table_len, &r->hist_n));
    OEC_TRY(ctx_array(c, d->table_len, &r->hist_w));
    OEC_TRY(ctx_array(c, 256, &r->hist_scratch));
    OEC_TRY(ctx_array(c, 1, &r->n_add));
    OEC_TRY(ctx_array(c, 1, &r->fails));
    OEC_TRY(ctx_array(c, 6 * (size_t)d->target, &r->clone_rows));
    // the initial particles (setParticleData), their deposit, the first history entry
    const int32_t n_rows = (int32_t)d->n_rows;  // read by the copy below before the synchronize
    if (d->n_rows > 0) {
        double *aos;
        OEC_TRY(ctx_upload(c, d->rows, 6 * (size_t)d->n_rows, &aos));
        OEC_TRY(oec_particles_from_aos(&d->grid, aos, d->n_rows, &r->p, c->stream));
    }
    OEC_CUDA_TRY(cudaMemcpyAsync(r->array_len, &n_rows, sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
    OEC_TRY(prepare_deposit(r));
    OEC_TRY(oec_history(&r->p, r->step, d->table_len, r->hist_w, r->hist_n, r->hist_scratch, c->stream));
    OEC_CUDA_TRY(cudaStreamSynchronize(c->stream));  // the host arrays may go once this returns
    // the host pointers of the description are not kept
    r->d.rows = nullptr;
    r->d.beam_profile = r->d.beam_table = nullptr;
    r->d.e_ptr = r->d.e_idx = nullptr;
    r->d.e_val = nullptr;
    memset(&r->d.lu, 0, sizeof(r->d.lu));
    return OEC_OK;
}

}  // namespace

extern "C" int oec_ctx_create(int32_t device, oec_ctx_t **out) {
    if (!out) return OEC_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    OEC_CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return OEC_ERR_INVALID;
    OEC_CUDA_TRY(cudaSetDevice(device));
    oec_ctx *c = new oec_ctx();
    c->device = device;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return OEC_ERR_CUDA;
    }
    void *st = nullptr;
    if (ctx_alloc(c, sizeof(oec_status_t), &st) != OEC_OK) {
        oec_ctx_destroy(c);
        return OEC_ERR_CUDA;
    }
    c->status = static_cast<oec_status_t *>(st);
    *out = c;
    return OEC_OK;
}

extern "C" int oec_ctx_destroy(oec_ctx_t *c) {
    if (!c) return OEC_ERR_INVALID;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (void *p : c->allocs) cudaFree(p);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return OEC_OK;
}

extern "C" int oec_ctx_stream(oec_ctx_t *c, void **stream) {
    if (!c || !stream) return OEC_ERR_INVALID;
    *stream = c->stream;
    return OEC_OK;
}

extern "C" int oec_ctx_synchronize(oec_ctx_t *c) {
    if (!c) return OEC_ERR_INVALID;
    OEC_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return OEC_OK;
}

extern "C" int oec_ctx_alloc(oec_ctx_t *c, int64_t bytes, void **dev) {
    if (!c || !dev || bytes < 0) return OEC_ERR_INVALID;
    return ctx_alloc(c, (size_t)bytes, dev);
}

extern "C" int oec_status(oec_ctx_t *c, oec_status_t *out) {
    if (!c || !out) return OEC_ERR_INVALID;
    OEC_CUDA_TRY(cudaMemcpyAsync(out, c->status, sizeof(*out), cudaMemcpyDeviceToHost, c->stream));
    OEC_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return OEC_OK;
}

extern "C" int oec_run_create(oec_ctx_t *c, const oec_run_desc_t *desc, oec_run_t **out) {
    if (!c || !out) return OEC_ERR_INVALID;
    *out = nullptr;
    if (!valid_desc(desc)) return OEC_ERR_INVALID;
    OEC_CUDA_TRY(cudaSetDevice(c->device));
    oec_run *r = new oec_run();
    const int rc = create_run(c, desc, r);
    if (rc != OEC_OK) {
        // the partial allocations stay with the context and go with it
        delete r;
        return rc;
    }
    *out = r;
    return OEC_OK;
}

extern "C" int oec_run_steps(oec_run_t *r, int32_t n_steps, int32_t use_graph) {
    if (!r || n_steps < 0) return OEC_ERR_INVALID;
    if (r->steps_done + n_steps > r->d.table_len - 1) return OEC_ERR_CAPACITY;  // beam table / history length
    OEC_CUDA_TRY(cudaSetDevice(r->ctx->device));
    const int every = r->d.management_every;
    int k = 0;
    while (k < n_steps) {
        if (r->steps_done > 0 && r->steps_done % every == 0) {
            nvtxRangePushA("oec_run management");
            const int rc = manage(r);
            nvtxRangePop();
            OEC_TRY(rc);
        }
        const int nxt = std::min<int64_t>(n_steps - k, every - r->steps_done % every);
        nvtxRangePushA("oec_run steps");
        const int rc = replay(r, nxt, use_graph != 0);
        nvtxRangePop();
        OEC_TRY(rc);
        k += nxt;
        r->steps_done += nxt;
    }
    OEC_CUDA_TRY(cudaStreamSynchronize(r->ctx->stream));
    return OEC_OK;
}

extern "C" int oec_run_history(oec_run_t *r, int32_t *counts_host, double *weights_host, int32_t n) {
    if (!r || !counts_host || !weights_host || n < 0 || n > r->d.table_len) return OEC_ERR_INVALID;
    cudaStream_t s = r->ctx->stream;
    OEC_CUDA_TRY(cudaMemcpyAsync(counts_host, r->hist_n, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
    OEC_CUDA_TRY(cudaMemcpyAsync(weights_host, r->hist_w, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    OEC_CUDA_TRY(cudaStreamSynchronize(s));
    return OEC_OK;
}

extern "C" int oec_run_get_rows(oec_run_t *r, double *rows_host, int64_t max_rows, int64_t *n_out) {
    if (!r || !n_out || max_rows < 0 || (max_rows > 0 && !rows_host)) return OEC_ERR_INVALID;
    int32_t n = 0;
    OEC_TRY(read_count(r, &n));
    *n_out = n;
    const int64_t rows = n < max_rows ? n : max_rows;
    if (rows == 0) return OEC_OK;
    if (!r->stage) OEC_TRY(ctx_array(r->ctx, 6 * (size_t)r->d.capacity, &r->stage));
    OEC_TRY(oec_particles_to_aos(&r->d.grid, &r->p, r->stage, rows, r->ctx->stream));
    OEC_CUDA_TRY(cudaMemcpyAsync(rows_host, r->stage, sizeof(double) * 6 * (size_t)rows, cudaMemcpyDeviceToHost,
                                 r->ctx->stream));
    OEC_CUDA_TRY(cudaStreamSynchronize(r->ctx->stream));
    return OEC_OK;
}

extern "C" int oec_run_particles(oec_run_t *r, oec_particles_t *out) {
    if (!r || !out) return OEC_ERR_INVALID;
    *out = r->p;
    return OEC_OK;
}

extern "C" int oec_run_destroy(oec_run_t *r) {
    if (!r) return OEC_ERR_INVALID;
    cudaSetDevice(r->ctx->device);
    cudaStreamSynchronize(r->ctx->stream);
    if (r->graph) cudaGraphExecDestroy(r->graph);
    delete r;  // device memory belongs to the context
    return OEC_OK;
}
