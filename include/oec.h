/*
 * oec.h -- C ABI of liboec.so, the B200 (sm_100a) implementation of the
 * openECLOUD per-timestep particle-in-cell loop.
 *
 * Conventions
 *  - Every function returns int status: 0 = OEC_OK, >0 = an OEC_ERR_* code.
 *    Nothing aborts or traps; device-side anomalies are counted in an
 *    oec_status_t block that lives in device memory.
 *  - Pointers named *_dev are device pointers; *_host are host pointers.
 *    `stream` is a cudaStream_t passed as void* (NULL = legacy default).
 *  - Counts that change on the device (macro-particle count, absorbed count,
 *    secondary count) live in device memory (int32) so a whole time step can
 *    run without host synchronisation and be captured in a CUDA graph.
 *  - Particle storage is structure-of-arrays, FP32, cell-relative:
 *      cell  int32   inCell index ix + iy*nxExt of the extended grid
 *      ox,oy float   offset inside the cell, in cell units, [0,1)
 *      vx,vy,vz,w    float
 *    The absolute position is x = (ix + ox)*dx - lxExt/2 (likewise y).
 *    Arrays are 16-byte aligned with capacity a multiple of 1024.
 *  - Each entry point names the reference function it replaces
 *    (file:line inside the openECLOUD source tree).
 */
#ifndef OEC_H
#define OEC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status */
#define OEC_OK 0
#define OEC_ERR_INVALID 1      /* bad argument (null pointer, size, enum) */
#define OEC_ERR_CUDA 2         /* a CUDA runtime call failed */
#define OEC_ERR_CAPACITY 3     /* particle / secondary capacity exceeded */
#define OEC_ERR_NOT_CONVERGED 4/* iterative solve missed its tolerance */
#define OEC_ERR_OVERFLOW 5     /* fixed-point deposit range exceeded */
#define OEC_ERR_HOST 6         /* host-side allocation / geometry failure */

/* Device-resident anomaly counters (all int32, zeroed by the caller). */
typedef struct oec_status {
    int32_t n_absorbed;        /* particles flagged outside by the last inside test */
    int32_t n_secondaries;     /* secondaries produced by the last emission */
    int32_t n_nonfinite;       /* particles with non-finite state (absorbed) */
    int32_t n_clipped;         /* cut-cell clip to grid (particleBoundary.pyx:485) */
    int32_t n_not_found;       /* wall intersection not found (particleBoundary.pyx:443) */
    int32_t n_capacity_drop;   /* secondaries dropped for lack of capacity */
    int32_t deposit_overflow;  /* a fixed-point node left the safe range */
    int32_t n_wait_timeout;    /* bounded device waits that gave up */
    int32_t warn_derm;         /* delta_E+delta_R >= cap (particleEmitter.pyx:201-206) */
    int32_t warn_tsprime;      /* delta_TS' >= m (particleEmitter.pyx:209-214) */
    int32_t n_out_of_grid;     /* particles that left the extended grid (absorbed) */
    int32_t n_rows_dropped;    /* absorbed particles beyond the absorbed-row capacity of
                                  oec_wall_interaction: removed without a wall row, so
                                  they emit no secondaries (the caller must grow the rows) */
    int32_t n_emit_skipped;    /* absorbed rows with a non-finite position, energy or wall
                                  normal: they emit no secondaries */
    int32_t reserved[3];
} oec_status_t;

/* ------------------------------------------------------------ types */
typedef struct oec_particles {
    int32_t *cell;             /* [capacity] */
    float *ox, *oy;            /* [capacity] */
    float *vx, *vy, *vz;       /* [capacity] */
    float *w;                  /* [capacity] macro-particle weight */
    int32_t *count;            /* device scalar: macro-particle count */
    int64_t capacity;
} oec_particles_t;

/* Extended grid (grid.pyx:57-72): nx, ny are nxExt, nyExt (= n + 2). */
typedef struct oec_grid {
    int32_t nx, ny;
    double dx, dy;             /* cell size */
    double lx, ly;             /* inner domain size (boundary geometry) */
} oec_grid_t;

/* Particle boundary (particleBoundary.pyx). kind: 0 rect, 1 ellipse, 2 cut-cell. */
#define OEC_BOUNDARY_RECT 0
#define OEC_BOUNDARY_ELLIPSE 1
#define OEC_BOUNDARY_CUTCELL 2
typedef struct oec_boundary {
    int32_t kind;
    int32_t n_boundary_points;
    const uint16_t *inside_faces_dev;      /* cut-cell: [G] */
    const double *boundary_points_dev;     /* cut-cell: [nb*2] */
    const int32_t *cut_cell_points_ind_dev;/* cut-cell: [G*2] */
    const double *cut_cell_normals_dev;    /* cut-cell: [G*2] */
} oec_boundary_t;

/* ------------------------------------------------ particle store (A1) */

/* setParticleData (particles.pyx:126-140): (n,6) f64 AoS rows
 * [x,y,vx,vy,vz,w] already on the device -> SoA.  Sets *count = n. */
int oec_particles_from_aos(const oec_grid_t *grid, const double *aos_dev, int64_t n,
                           oec_particles_t *p, void *stream);

/* getParticleData (particles.pyx:142-143): SoA -> (count,6) f64 AoS. */
int oec_particles_to_aos(const oec_grid_t *grid, const oec_particles_t *p, double *aos_dev,
                         int64_t max_rows, void *stream);

/* Streamed host round trip of the above: pinned/pageable host AoS in,
 * chunks overlapped on two internal streams.  Used for end-to-end timing. */
int oec_particles_upload_host(const oec_grid_t *grid, const double *aos_host, int64_t n,
                              oec_particles_t *p, double *staging_dev, int64_t staging_rows,
                              void *stream);
int oec_particles_download_host(const oec_grid_t *grid, const oec_particles_t *p,
                                double *aos_host, int64_t n, double *staging_dev,
                                int64_t staging_rows, void *stream);

/* One step from host rows to host rows: setParticleData + the fused
 * oec_push_gather + getParticleData (particles.pyx:126, :142 around the
 * pushes) with the copies overlapped.  The rows go through a ring of 4
 * staging slots in staging_dev (staging_rows rows of 6 doubles; each slot
 * holds ((staging_rows - 1) / 4) rounded down to a multiple of 1024 rows, at
 * least 1024; the row after the slots holds the slots' counts): uploads on
 * one stream, the conversion, the fused kernel on that chunk of the store and
 * the conversion back on `stream`, downloads on a third, so both copy
 * directions run while the kernels do.  rows_out_host may be rows_in_host.
 * The store ends with count n; rho, the absorbed bits and the status as
 * oec_push_gather.  Pinned host memory lets the copies overlap.  Returns
 * when queued; the work is ordered on `stream`.  Overlapping calls race. */
int oec_push_gather_host(const oec_grid_t *grid, oec_particles_t *p, const double *rows_in_host,
                         double *rows_out_host, int64_t n, double *staging_dev, int64_t staging_rows,
                         const float *e_cell_dev, const float *b_cell_dev, const double bconst[3], double dt,
                         double charge_over_mass, int32_t type_b_field, const oec_boundary_t *boundary,
                         uint32_t *absorbed_mask_dev, int64_t *rho_fix_dev, const double *wscale_dev,
                         oec_status_t *status_dev, void *stream);

/* ------------------------------------------- weights, gather, push (A2-A8) */

/* calcGridWeights (particles.pyx:52-56, :400-418): inCell and the four CIC
 * weights in f64 (LowXLowY, UpXLowY, LowXUpY, UpXUpY). */
int oec_calc_grid_weights(const oec_grid_t *grid, const oec_particles_t *p, uint32_t *in_cell_dev,
                          double *w00_dev, double *w10_dev, double *w01_dev, double *w11_dev,
                          void *stream);

/* Node field [Fx | Fy (| Fz)] f64 (poissonSolver.pyx:63 layout) ->
 * cell-centric float4 corner table used by every gather: per cell and
 * component {F[c], F[c+1], F[c+nx], F[c+nx+1]}.  ncomp = 2 (E) or 3 (B). */
int oec_field_prepare(const oec_grid_t *grid, const double *node_field_dev, int32_t ncomp,
                      float *cell_field_dev, void *stream);

/* eFieldToParticles / bFieldToParticles (particles.pyx:58-68, :354-397):
 * bilinear gather to (count, ncomp) f64 rows. */
int oec_gather(const oec_grid_t *grid, const oec_particles_t *p, const float *cell_field_dev,
               int32_t ncomp, double *out_dev, void *stream);

/* borisPush (particles.pyx:79-92 -> :324 / :298 / :272) with the field at
 * the particles given as (count,2) E rows and, for type 2, (count,3) B rows. */
int oec_boris_push(const oec_grid_t *grid, oec_particles_t *p, const double *e_at_particles_dev,
                   const double *b_at_particles_dev, const double bconst[3], double dt,
                   double charge_over_mass, int32_t type_b_field, void *stream);

/* Fixed-point deposit scale: charge of a particle of weight w is stored as
 * llrint(w * wscale) integer units, wscale = 2^(bits - ceil(log2(wmax))).
 * Computes wscale on the device from the particles' max |w|; bits =
 * min(50, 63 - ceil(log2(capacity))): every particle's charge stays below
 * 2^bits units, so capacity * 2^bits <= 2^63 and no node can leave the int64
 * range whatever the particle distribution. */
int oec_deposit_scale(const oec_particles_t *p, double *wscale_dev, void *stream);

/* The same scale for one shard of a particle store split over several
 * stores (one per GPU) whose int64 deposits are summed afterwards: bits =
 * min(50, 63 - ceil(log2(total_capacity))) with total_capacity the sum of
 * the shards' capacities (>= p->capacity), so the summed grid stays inside
 * int64.  The shards then take the smallest of their scales (the largest
 * weight), which keeps every shard's charges exact.  Replaces the charge
 * scaling of chargeToGrid (particles.pyx:70-77) for a sharded run. */
int oec_deposit_scale_capacity(const oec_particles_t *p, int64_t total_capacity, double *wscale_dev,
                               void *stream);

/* THE HOT PATH.  One pass over all particles:
 *   gather E (and B for type 2) at the current position, Boris push
 *   (type 0/1/2), move, inside test of `boundary` at the new position,
 *   set the absorbed bit in absorbed_mask_dev (1 bit per particle), and,
 *   when rho_fix_dev != NULL, clear rho_fix_dev and deposit the surviving
 *   particles' weights into that int64 fixed-point node grid
 *   (warp-aggregated atomics).
 * Replaces calcGridWeights + eFieldToParticles + borisPush + indexInside +
 * chargeToGrid of the next step (example01_basic.py:66-91).
 * wscale_dev: device scalar from oec_deposit_scale (may be NULL if no deposit).
 * absorbed_mask_dev must hold ceil(capacity/32) words (zeroed inside). */
int oec_push_gather(const oec_grid_t *grid, oec_particles_t *p, const float *e_cell_dev,
                    const float *b_cell_dev, const double bconst[3], double dt,
                    double charge_over_mass, int32_t type_b_field,
                    const oec_boundary_t *boundary, uint32_t *absorbed_mask_dev,
                    int64_t *rho_fix_dev, const double *wscale_dev,
                    oec_status_t *status_dev, void *stream);

/* chargeToGrid (particles.pyx:70-77, :336-351) as an order-independent
 * int64 fixed-point deposit.  zero_first: clear rho_fix first. */
int oec_deposit(const oec_grid_t *grid, const oec_particles_t *p, int64_t *rho_fix_dev,
                const double *wscale_dev, int32_t zero_first, oec_status_t *status_dev,
                void *stream);

/* int64 fixed point -> f64 charge per node: rho = q * fix / wscale. */
int oec_deposit_finalize(const oec_grid_t *grid, const int64_t *rho_fix_dev,
                         const double *wscale_dev, double particle_charge, double *rho_dev,
                         void *stream);

/* No counterpart in the reference.  The charge deposit above (scale + deposit
 * + finalize, f64 charge per node into rho_dev) for callers that cannot
 * allocate device memory: hosts that own the whole device memory budget
 * through their own pool, or run with a memory plan fixed before the
 * simulation starts.  The int64 scratch grid and the fixed-point scale live in
 * file-scope device arrays (about 8.8 MB per GPU, held until the process
 * exits); nothing is allocated.  Limit: nx*ny of the extended grid at most
 * 1,100,000 nodes (a 1024 x 1024 grid), else OEC_ERR_CAPACITY.  All calls
 * share the scratch, so calls that overlap on the GPU (other streams, other
 * threads) race: serialise them.  Each call clears the scratch it uses; the
 * first call on a device looks up the scratch address with that device
 * current, so make it before any stream capture. */
int oec_deposit_charge_noalloc(const oec_grid_t *grid, const oec_particles_t *p,
                               double particle_charge, double *rho_dev, void *stream);

/* ---------------------------------------------------- boundary (A17-A20) */

/* indexInside (particleBoundary.pyx:84-97 / :227-242 / :336-370): absorbed
 * bit per particle (1 = outside) and status->n_absorbed.  For the cut-cell
 * kind the positions are first clipped to the grid (:485-508). */
int oec_index_inside(const oec_grid_t *grid, oec_particles_t *p, const oec_boundary_t *boundary,
                     uint32_t *absorbed_mask_dev, oec_status_t *status_dev, void *stream);

/* Absorbed set as the ascending list of absorbed particle indices
 * (saveAbsorbed's scan order, particleBoundary.pyx:48-65).  n_abs_dev gets
 * the count (also copied to status->n_absorbed when status_dev != NULL);
 * scratch_dev: >= 1024 int32. */
int oec_absorbed_index(const oec_particles_t *p, const uint32_t *absorbed_mask_dev, int32_t *index_dev,
                       int32_t index_cap, int32_t *n_abs_dev, int32_t *scratch_dev, oec_status_t *status_dev,
                       void *stream);

/* saveAbsorbed (particleBoundary.pyx:38-65): the absorbed particles as
 * (n_abs, 6) f64 rows [x,y,vx,vy,vz,w] (at most cap rows). */
int oec_save_absorbed(const oec_grid_t *grid, const oec_particles_t *p, const int32_t *index_dev,
                      const int32_t *n_abs_dev, int32_t cap, double *rows_dev, void *stream);

/* calculateInteractionPoint + calculateNormalVectors for the boundary kind
 * (particleBoundary.pyx:99-221 rect, :252-297 ellipse, :373-481 cut-cell):
 * moves each row back onto the wall, writes (n_abs, 2) inward normals;
 * dt is the last push step (used by the cut-cell back step).  Rows whose
 * intersection is not found are counted in status->n_not_found: for the
 * rectangle a zero velocity across the crossed side (the point is clamped
 * onto the wall), for the ellipse a back step that misses the wall (the
 * point is projected radially onto it); the reference's formulas give NaN
 * there. */
int oec_wall_interaction(const oec_grid_t *grid, const oec_boundary_t *boundary, double dt, double *rows_dev,
                         const int32_t *n_abs_dev, int32_t cap, double *normals_dev, oec_status_t *status_dev,
                         void *stream);

/* addAndRemoveParticles (particles.pyx:94-121): remove the absorbed
 * particles (holes = ascending absorbed indices) and insert the added rows,
 * leaving every particle in the slot the reference's array gives it:
 *  - no added rows (_removeParticles, :254-269): each hole below the new
 *    count, in ascending order, takes the last kept particle of the tail;
 *  - new count above *array_len_dev (_addAndRemoveParticlesNewArray,
 *    :109-116, :201-219): the kept particles in order, then the added rows;
 *    *array_len_dev becomes int(1.1 * new count);
 *  - otherwise (_addAndRemoveParticles, :222-252): added row k fills hole k;
 *    extra rows are appended after the old count, or, with fewer rows than
 *    holes, the kept particles after the last filled hole shift down in
 *    order.
 * array_len_dev: the row count of the reference's particle array (set to
 * the count wherever the reference calls setParticleData), or NULL to never
 * take the new-array rule.  tmp: a scratch store of at least p's capacity
 * (count pointer unused).  Optionally deposits the added rows into rho_fix
 * (same scale as oec_push_gather).  The count is updated on the device;
 * rows beyond the capacity are dropped and counted. */
int oec_add_remove(const oec_grid_t *grid, oec_particles_t *p, oec_particles_t *tmp,
                   const uint32_t *absorbed_mask_dev, const int32_t *holes_dev, const int32_t *n_holes_dev,
                   int32_t holes_cap, const double *add_rows_dev, const int32_t *n_add_dev, int32_t add_cap,
                   int32_t *array_len_dev, int64_t *rho_fix_dev, const double *wscale_dev, oec_status_t *status_dev,
                   void *stream);

/* keepParticles u16 array (1 = keep) -> absorbed bitmask (1 = remove). */
int oec_mask_from_keep(const uint16_t *keep_dev, int64_t n, uint32_t *mask_dev, int64_t mask_words, void *stream);

/* ------------------------------------------- emission (A21-A24) */

/* Furman-Pivi model parameters (particleEmitter.pyx:77-152 copperMod /
 * stainlessMod); m <= 10 secondaries. */
typedef struct oec_furman {
    double p1EInf, p1Ehat, eEHat, w, p, e1, e2;
    double p1RInf, eR, r, r1, r2, q, sigmaE;
    double deltaTSHat, s, eHat0, t1, t2, t3, t4;
    double theta0max, deltaERmax;
    double epsN[10], pSmallN[10];
    double particle_mass;
    int32_t m;
    int32_t scaleSigmaE;
    int32_t compat_last;   /* 1: single-secondary split uses the last absorbed
                              particle's yields, as the reference does
                              (particleEmitter.pyx:245-246); 0: its own */
    int32_t reserved;
} oec_furman_t;

/* Parameters of the simplified emitters: model 0 = SecElecEmitter with the
 * stainless parameters of stainlessMod (particleEmitter.pyx:316-352, seyMax
 * and reflec applied), model 1 = SimpleSecEmitter (:489-597, fixed yields,
 * electron mass; the other fields unused).  max_ts (1..10) caps the number
 * of true secondaries of one absorbed particle (the reference has no cap;
 * a capped particle is counted in status->warn_tsprime). */
typedef struct oec_secelec {
    int32_t model, max_ts;
    double p1EInf, p1Ehat, eEHat, w, p, e1, e2, p1RInf, eR, r, r1, r2;
    double deltaTSHat, s, eHat0, t1, t2, t3, t4, sigmaETS, muETS, theta0max, deltaERmax, q;
    double particle_mass;
} oec_secelec_t;

/* Bytes of `work_dev` oec_secelec_emit needs for `cap` absorbed rows
 * (cap <= 2^26; -1 beyond). */
int64_t oec_secelec_work_bytes(int32_t cap);

/* SecElecEmitter / SimpleSecEmitter.generateSecondaries
 * (particleEmitter.pyx:355-484, :506-597): per absorbed row an elastic
 * secondary (reversed velocity) with probability delta_E, a rediffused one
 * (velocity scaled by rand^(1/(2(1+q))), simple: sqrt(rand)) with
 * probability delta_R, and floor(delta_TS) (+1 with probability of the
 * fraction) true secondaries: lognormal energies (a uniform split of E0 when
 * they sum above E0) emitted about the wall normal by theta = asin(rand),
 * phi = 2 pi rand (simple: uniform 0-5 eV along the reversed velocity).
 * Output order and arguments as oec_furman_emit; replay_uniforms_dev, if
 * given, holds 64 uniforms per absorbed row consumed in the reference's
 * order (a normal deviate = Box-Muller of two). */
int oec_secelec_emit(const oec_secelec_t *params, const double *rows_dev, const double *normals_dev,
                     const int32_t *n_abs_dev, int32_t cap, const int32_t *ids_dev, uint64_t seed, uint32_t step,
                     const int32_t *step_dev, const double *replay_uniforms_dev, void *work_dev,
                     double *out_rows_dev, int32_t out_cap, int32_t *n_out_dev, oec_status_t *status_dev,
                     void *stream);

/* Bytes of `work_dev` oec_furman_emit needs for `cap` absorbed rows
 * (cap <= 2^26; -1 beyond). */
int64_t oec_furman_work_bytes(int32_t cap);

/* generateSecondaries (particleEmitter.pyx:154-308) on the absorbed rows at
 * the wall (after oec_wall_interaction) with their normals.  Secondaries are
 * written as (n_out, 6) f64 rows, grouped by absorbed row in order.  Random
 * draws: Philox4x32-10 keyed by `seed`, counter (ids[i] or i, step + *step_dev
 * (when step_dev != NULL: the device step counter of a replayed graph), draw);
 * with replay_uniforms_dev != NULL the uniforms are read from it instead
 * (32 per absorbed row: draw 0 selects the secondary count, the rest are
 * consumed in the reference's order; a normal deviate takes two). */
int oec_furman_emit(const oec_furman_t *params, const double *rows_dev, const double *normals_dev,
                    const int32_t *n_abs_dev, int32_t cap, const int32_t *ids_dev, uint64_t seed, uint32_t step,
                    const int32_t *step_dev, const double *replay_uniforms_dev, void *work_dev,
                    double *out_rows_dev, int32_t out_cap, int32_t *n_out_dev, oec_status_t *status_dev,
                    void *stream);

/* homoLoader (particleEmitter.pyx:41-72): n particles uniform inside the
 * boundary by rejection sampling, velocities N(0, vsigma), weight w0
 * (or w0*(0.5+U) with randomize_weight).  Sets *count = n. */
int oec_homo_load(const oec_grid_t *grid, const oec_boundary_t *boundary, oec_particles_t *p, int64_t n,
                  double weight, double vsigma, int32_t randomize_weight, uint64_t seed, int32_t *failed_dev,
                  void *stream);

/* ---------------------------------------- time-loop kernels (A28, histories) */

/* Poisson right-hand side of step *step_dev: electron charge from the
 * fixed-point deposit plus the beam imprint table[*step]*profile
 * (example01_basic.py:81, beam.py:68-78); profile/table may be NULL. */
int oec_rhs_with_beam(const oec_grid_t *grid, const int64_t *rho_fix_dev, const double *wscale_dev,
                      double particle_charge, const double *profile_dev, const double *table_dev,
                      const int32_t *step_dev, int32_t table_len, double *rho_dev, void *stream);

/* hist_w[*step] = sum w, hist_n[*step] = count (example01_basic.py:56-57).
 * scratch_dev: 256 doubles. */
int oec_history(const oec_particles_t *p, int32_t *step_dev, int32_t hist_len, double *hist_w_dev,
                int32_t *hist_n_dev, double *scratch_dev, void *stream);

/* ++*step_dev (keeps the step index on the device for graph replay). */
int oec_step_advance(int32_t *step_dev, void *stream);

/* --------------------------------------- particle management (A10, A25-A27) */

/* Bytes of the work buffer of oec_sort_particles / oec_cell_merge. */
int64_t oec_sort_work_bytes(int64_t capacity);

/* sortByColumn (particles.pyx:49-50, :431-459): stable radix sort of the
 * particles by column 2..5 (vx, vy, vz, w) or 6 (cell index); the sorted
 * store is written to `tmp` (same capacity), the caller swaps the two. */
int oec_sort_particles(oec_particles_t *p, oec_particles_t *tmp, int32_t column, void *work_dev, void *stream);

/* w *= factor for every particle (globalRandom, particleManagement.pyx:51,60). */
int oec_scale_weights(oec_particles_t *p, double factor, void *stream);

/* Removal bits for n_remove of the first n particles, chosen uniformly
 * without replacement (globalRandom, particleManagement.pyx:52-55); Philox
 * keyed by seed, counter `call`.  fails_dev counts darts that gave up. */
int oec_roulette_select(int32_t n, int32_t n_remove, uint32_t *mask_dev, int64_t mask_words, uint64_t seed,
                        uint32_t call, int32_t *fails_dev, void *stream);

/* k rows copied from particles drawn uniformly with replacement
 * (globalRandom clone step, particleManagement.pyx:62-66). */
int oec_clone_rows(const oec_grid_t *grid, const oec_particles_t *p, int32_t n, int32_t k, uint64_t seed,
                   uint32_t call, double *rows_dev, void *stream);

/* acc_dev[0] = sum w, acc_dev[1] = sum |v|^2 w^2 (localRandom :124-128). */
int oec_weight_stats(const oec_particles_t *p, double *acc_dev, void *stream);

/* Halve the weights of the last k of the first n particles and write their
 * duplicates as rows (localRandom split, particleManagement.pyx:130-163). */
int oec_split_rows(const oec_grid_t *grid, oec_particles_t *p, int32_t n, int32_t k, double *rows_dev, void *stream);

/* _searchSorted (particleManagement.pyx:244-262) twice on the store sorted
 * by weight (ascending): out_dev[0] / [1] = the reference's answer for lo /
 * hi (the first index with w > value; 0 as soon as w[0] >= value; n when
 * w[n-1] <= value). */
int oec_weight_thresholds(const oec_particles_t *p, double lo, double hi, int32_t *out_dev, void *stream);

/* Binned merge (localRandom :165-236): the first n_cand particles are
 * ordered along a 5-D Morton curve of their weighted phase-space coordinates
 * (x, y, lambda v; one scale for all axes); neighbouring pairs in that order
 * whose squared phase-space distance dx^2 + dy^2 + lambda^2 |dv|^2 is below
 * `limit` merge with probability min(1, n_merge / qualifying pairs); the
 * survivor is drawn with probability proportional to weight and takes the
 * summed weight; the other gets its removal bit.  scheme 1 rescales the
 * survivor's velocity as the reference does.  counters_dev[0] = qualifying
 * pairs, [1] = merges. */
int oec_cell_merge(const oec_grid_t *grid, oec_particles_t *p, int32_t n_cand, int32_t n_merge, double lambda,
                   double limit, int32_t scheme, uint64_t seed, uint32_t call, double vscale, uint32_t *mask_dev,
                   int32_t *counters_dev, void *work_dev, void *stream);

/* ------------------------------------------------ Poisson solve (A15-A16) */

/* Device form of SuperLU's P_r A P_c = L U (poissonSolver.pyx:59).
 * Rows [0, head) of each factor are solved level by level; the last
 * m = n - head rows ("tail") use dense inverses of their triangular blocks.
 * The head CSR of each factor is stored in level order: its row w is factor
 * row l_rows[w] (u_rows[w]), and level k holds rows [level_ptr[k],
 * level_ptr[k+1]) of that order; column indices are factor row numbers.
 * The first level of L has no entries (any entry would be a dependency) and
 * is not visited: its rows keep their right-hand side.
 * Level pointers are HOST arrays (the launch loop runs on the host); every
 * other pointer is a device pointer. */
typedef struct oec_lu {
    int32_t n;                 /* unknowns (inside nodes) */
    int32_t head;              /* rows solved by levels */
    int32_t n_nodes;           /* grid nodes G (phi length) */
    const int32_t *rhs_node;   /* [n] node feeding row k of P_r b */
    const int32_t *sol_src;    /* [n] perm_c: unknown i = z[sol_src[i]] */
    const int32_t *sol_node;   /* [n] node of unknown i */
    int32_t l_nlevels;
    const int32_t *l_level_ptr;/* HOST [l_nlevels+1] */
    const int32_t *l_rows;     /* [head] head rows of L ordered by level */
    const int32_t *l_ptr, *l_idx; const double *l_val;    /* strict lower L, head rows in level order */
    const int32_t *lc_ptr, *lc_idx; const double *lc_val; /* L[tail, head] */
    const double *tl_inv;      /* [m*m] inverse of unit-lower L[tail,tail], row-major */
    int32_t u_nlevels;
    const int32_t *u_level_ptr;/* HOST [u_nlevels+1], backward order */
    const int32_t *u_rows;     /* [head] */
    const int32_t *u_ptr, *u_idx; const double *u_val;    /* strict upper U, head rows in level order */
    const double *u_diag;      /* [head] diagonal of U, in level order */
    const double *tu_inv;      /* [m*m] inverse of U[tail,tail], row-major */
    int32_t head_path;         /* how the head levels run: OEC_LU_HEAD_* (0: chosen by size) */
    const int8_t *l_level_lanes; /* HOST [l_nlevels] or NULL: per level, 0 or the lanes per row (1, 2, 4, ..., 32)
                                    of a level that runs inside a one-CTA run (its rows * lanes <= 1024) */
    const int8_t *u_level_lanes; /* HOST [u_nlevels] or NULL, likewise for U */
} oec_lu_t;

/* Head-level execution of oec_lu_solve.  AUTO: every run of two or more
 * consecutive levels marked in l_level_lanes / u_level_lanes goes to one CTA
 * (narrow levels: a __syncthreads instead of a launch between them); the
 * levels between the runs go, segment by segment, to one cooperative launch
 * (2 to 64 levels) or a launch per level.  PER_LEVEL: a launch per level.
 * COOPERATIVE: one cooperative launch per factor of at most 64 levels, else a
 * launch per level.  ONE_CTA (n <= 28672 and at most 64 levels per factor):
 * each whole factor in one CTA with the vector in shared memory; it ties with
 * COOPERATIVE on a warm L2 and is slower when the factors come from HBM, so
 * AUTO does not take it.  A path that does not fit falls back as AUTO does. */
#define OEC_LU_HEAD_AUTO 0
#define OEC_LU_HEAD_PER_LEVEL 1    /* one launch per level, a warp per row */
#define OEC_LU_HEAD_COOPERATIVE 2  /* one cooperative launch per factor, grid barrier between levels */
#define OEC_LU_HEAD_ONE_CTA 3      /* one CTA per factor, the vector in shared memory */

/* phi = A^-1 q on the inside nodes, 0 elsewhere (poissonSolver.pyx:85).
 * q_dev, phi_dev: [n_nodes]; work_dev: n + (n - head) doubles. */
int oec_lu_solve(const oec_lu_t *lu, const double *q_dev, double *phi_dev, double *work_dev, void *stream);

/* y = A x, CSR with int32 indices (E = phiToE . phi, poissonSolver.pyx:87). */
int oec_spmv_csr(int32_t nrows, const int32_t *ptr_dev, const int32_t *idx_dev, const double *val_dev,
                 const double *x_dev, double *y_dev, void *stream);

/* Host helper: dependency level of each row of a triangular CSR factor. */
int oec_trsv_levels(int32_t nrows, const int32_t *ptr, const int32_t *idx, int32_t lower, int32_t ncols_dep,
                    int32_t *level_out, int32_t *nlevels_out);

/* ---------------------------------------- iterative Poisson solve (A16) */

/* The reference's system matrix A = S diag(meps) S^T restricted to the inside
 * nodes (poissonSolver.pyx:41-58) is a 5-point operator; it is stored by edge
 * on the full extended grid: ex[i] is the weight meps of the x edge between
 * nodes i and i+1, ey[i] that of the y edge between i and i+nx.  For an
 * inside node i, (A x)_i = sum over its four edges of meps * (x_i - x_j) with
 * x_j = 0 for outside nodes j (their value is fixed at 0).  Vectors live on
 * the full extended grid [G = nx*ny] and are zero outside.  The f32 copies
 * hold scale32 * the f64 weights (scale32 brings them to order one);
 * dinv32 = 1 / diag of that scaled operator (0 outside). */
typedef struct oec_stencil {
    int32_t nx, ny;
    const double *ex64, *ey64;
    const float *ex32, *ey32, *dinv32;
    const uint8_t *inside;
    double scale32;
} oec_stencil_t;

/* y = A x in f64 on the inside nodes, 0 outside (used by the solver's
 * residual and by the tests; poissonSolver.pyx:57 assembles the same A). */
int oec_stencil_apply(const oec_stencil_t *st, const double *x_dev, double *y_dev, void *stream);

#define OEC_PRECOND_NONE 0
#define OEC_PRECOND_JACOBI 1
#define OEC_PRECOND_CNN 2
#define OEC_PRECOND_MG 3

/* Multigrid preconditioner for oec_pcg_solve (precond = OEC_PRECOND_MG,
 * precond_ctx = an oec_mg_t): one V-cycle of aggregation multigrid on the
 * scaled operator.  No counterpart in the reference, whose only solve is the
 * direct one (poissonSolver.pyx:83-88).  Level 0 is the solver's f32 operator
 * (leak 0); level l+1 aggregates 2x2 nodes of level l (node (r, c) ->
 * (r/2, c/2), nx_{l+1} = (nx_l + 1) / 2), and its operator is the Galerkin
 * product P^T A P with the piecewise-constant P: again a 5-point stencil plus
 * a diagonal "leak" (the weight of edges from inside nodes to the fixed
 * outside).  On a level, (A x)_i = leak_i x_i + sum over the 4 grid edges of
 * w (x_i - x_j), with x = 0 outside; a node is inside exactly when its
 * dinv (1/diagonal) is nonzero.  Two damped-Jacobi sweeps (weight omega)
 * before and after the coarse correction, which is scaled by `scale`.
 * Levels block_level .. nlevels-1 are solved by one CTA in shared memory
 * (7 floats per node of those levels, at most 226 KB), the last of them by
 * its dense inverse over its inside nodes. */
typedef struct oec_mg_level {
    int32_t nx, ny;
    const float *ex, *ey, *leak, *dinv;  /* [nx*ny] edge weights (ex: (r,c)-(r,c+1), ey: (r,c)-(r+1,c)), leak,
                                            1/diagonal (0 outside) */
    const uint8_t *inside;               /* [nx*ny] (informational; dinv decides) */
    float *b, *x, *y;                    /* [nx*ny] work: right-hand side, pre-smoothed iterate, result */
} oec_mg_level_t;

typedef struct oec_mg {
    int32_t nlevels;                 /* 1..16 */
    const oec_mg_level_t *levels;    /* HOST array, level 0 the fine grid */
    int32_t block_level;             /* first level solved inside one CTA; at most 8 levels from there */
    int32_t ncoarse;                 /* inside nodes of the coarsest level (1..1024) */
    const int32_t *coarse_idx;       /* [ncoarse] their node indices */
    const float *coarse_inv;         /* [ncoarse*ncoarse] row-major inverse of its operator */
    float omega;                     /* damped-Jacobi weight */
    float scale;                     /* coarse-correction scale */
    int32_t cluster_top;             /* > 0: the levels from the first one of at most cluster_top nodes
                                        (no lower than block_level) to the bottom are solved by one
                                        thread-block cluster of 8 or 16 CTAs (their bands of b, x, y in
                                        distributed shared memory) instead of the one-CTA kernel;
                                        0: one CTA.  The one-CTA path is also taken when the cluster
                                        levels do not fit 226 KB of shared memory per CTA. */
} oec_mg_t;

/* z = M r, one V-cycle (r, z f32 [nx*ny] of level 0; z is 0 outside).
 * Overlapping calls with one oec_mg_t race on its work vectors. */
int oec_mg_apply(const oec_mg_t *mg, const float *r_dev, float *z_dev, void *stream);

typedef struct oec_pcg_stats {
    int32_t iterations;   /* f32 inner iterations, all refinements */
    int32_t refinements;  /* f64 residual evaluations */
    int32_t converged;    /* 1 if the f64 relative residual reached tol */
    int32_t breakdown;    /* 1 if an inner solve stopped on a non-positive or non-finite curvature */
    double rel_residual;  /* final ||q - A phi||_2 / ||q||_2 over the inside nodes, in f64 */
    double rel_residual0; /* the same for the warm start */
} oec_pcg_stats_t;

int64_t oec_pcg_work_bytes(int32_t nx, int32_t ny);

/* No counterpart in the reference.  Warm start of the next iterative solve
 * by linear extrapolation in time: phi <- 2 phi - phi_prev and phi_prev <- the
 * old phi, elementwise over n doubles (phi holds the last solution, phi_prev
 * the one before).  history_dev (device int32, start at 0; NULL: always
 * extrapolate) counts the solutions seen, saturating at 2: below 2 phi is
 * kept and only copied to phi_prev.  Call it before each solve; enqueued on
 * the stream, no synchronisation, so a captured step replays it. */
int oec_warm_start_extrapolate(double *phi_dev, double *phi_prev_dev, int64_t n, int32_t *history_dev,
                               void *stream);

/* No counterpart in the reference (it only has the direct solve of
 * poissonSolver.pyx:85).  phi = A^-1 q on the inside nodes by f64 iterative
 * refinement around an f32 flexible preconditioned conjugate-gradient solve:
 * each refinement forms r = q - A phi in f64, solves A d = r in f32 to a
 * relative max(1e-6, tol / (2 ||r||/||q||)) (or stagnation: the best inner
 * residual did not drop by 10 % in 1024 iterations), and adds d in f64; it
 * stops when ||r||/||q|| <= tol, after max_iter inner iterations in total,
 * after 12 refinements, or when a refinement gained less than a factor 2.
 * phi_dev holds the warm start on entry (zeros for none) and the solution on
 * return (0 outside).  precond: OEC_PRECOND_NONE / _JACOBI / _CNN
 * (precond_ctx = an oec_cnn_t, see below) / _MG (precond_ctx = an oec_mg_t).
 * max_iter <= 2^24.  The solve runs as one CUDA graph whose loops the device
 * controls (conditional nodes); it is instantiated on the first call with
 * given arguments and cached by the argument values and the contents of the
 * structures they point to.  stats (host) reports convergence; the caller
 * falls back to oec_lu_solve when stats->converged is 0.  work_dev:
 * oec_pcg_work_bytes.  Synchronises the stream once, at the end; not
 * callable on a capturing stream (use oec_pcg_solve_async). */
int oec_pcg_solve(const oec_stencil_t *st, const double *q_dev, double *phi_dev, double tol, int32_t max_iter,
                  int32_t precond, const void *precond_ctx, void *work_dev, oec_pcg_stats_t *stats,
                  void *stream);

/* The same solve without any host synchronisation: stats_dev (device
 * oec_pcg_stats_t) receives the statistics.  With fallback (an oec_lu_t, its
 * work in lu_work_dev) the device runs oec_lu_solve when the solve missed tol
 * and adds 1 to *fallback_count_dev (optional).  On a capturing stream the
 * solve is recorded into the capture (a buildup step graph replays it with
 * its loops intact); otherwise the cached graph is launched on the stream.
 * Overlapping solves with one work_dev race. */
int oec_pcg_solve_async(const oec_stencil_t *st, const double *q_dev, double *phi_dev, double tol,
                        int32_t max_iter, int32_t precond, const void *precond_ctx, void *work_dev,
                        oec_pcg_stats_t *stats_dev, const oec_lu_t *fallback, double *lu_work_dev,
                        int32_t *fallback_count_dev, void *stream);

/* ------------------------------------- learned preconditioner (no counterpart
 * in the reference): a linear 4-level U-Net (16-32-64-64 channels, 3x3
 * convolutions, bf16 weights and activations, f32 accumulation) on the
 * extended grid, z = inside * N(inside * x). */
typedef struct oec_cnn {
    int32_t nx, ny;         /* extended grid */
    const uint8_t *inside;  /* [nx*ny] */
    void *w16;              /* bf16 parameters, oec_cnn_num_params() of them */
    void *act;              /* workspace of oec_cnn_act_bytes(nx, ny, training) bytes */
    int32_t conv_kernel;    /* 3x3 convolutions with 16..64 input channels: OEC_CNN_CONV_TCGEN05 (0,
                               tcgen05.mma issued by one thread, f32 accumulators in tensor memory)
                               or OEC_CNN_CONV_MMA_SYNC (warp-level mma.sync m16n8k16) */
} oec_cnn_t;

#define OEC_CNN_CONV_TCGEN05 0
#define OEC_CNN_CONV_MMA_SYNC 1

int32_t oec_cnn_num_params(void);
/* offsets[9]: start of each layer's weights in the flat parameter vector
 * (7 conv layers e0 e1 e2 e3 d2 d1 d0, the 1x1 output, the total);
 * shapes[24]: (out channels, taps, in channels) per layer.  Layer weights are
 * [out][tap][in] with tap = 3*ty + tx. */
int oec_cnn_param_layout(int32_t *offsets, int32_t *shapes);
int64_t oec_cnn_act_bytes(int32_t nx, int32_t ny, int32_t training);
/* z = N(x) (f32 [nx*ny] in and out, device). */
int oec_cnn_forward(const oec_cnn_t *c, const float *x_dev, float *z_dev, void *stream);
/* Bounded tensor-memory waits of the tcgen05 convolutions that gave up since
 * the last forward pass or training step began (0 on a healthy device; the
 * results of that pass are then invalid).  Synchronises the stream. */
int oec_cnn_status(const oec_cnn_t *c, int32_t *wait_timeouts_host, void *stream);
/* Warm start of the iterative solve: phi0 = |b| N(b / |b|) with
 * b = scale32 * q on the inside nodes (the network approximates the inverse
 * of the scaled operator); phi0 = 0 outside.  work_dev:
 * oec_cnn_warm_start_work_bytes. */
int64_t oec_cnn_warm_start_work_bytes(int32_t nx, int32_t ny);
int oec_cnn_warm_start(const oec_cnn_t *c, double scale32, const double *q_dev, double *phi_dev, void *work_dev,
                       void *stream);
/* Learned correction of the extrapolated warm start: with d = q - 2 q1 + q2,
 * the second difference in time of the charge (q1, q2: the two previous
 * charges, kept in q_hist_dev [2*nx*ny] and advanced here; *count_dev, the
 * number of earlier charges saturating at 2, starts at 0), phi += |b| N(b/|b|)
 * with b = scale32 * d on the inside nodes.  Since A (phi_n - 2 phi_n-1 +
 * phi_n-2) = d, this adds the network's estimate of what the linear
 * extrapolation 2 phi_n-1 - phi_n-2 misses.  Nothing is added while fewer
 * than two earlier charges exist.  work_dev: oec_cnn_correct_work_bytes. */
int64_t oec_cnn_correct_work_bytes(int32_t nx, int32_t ny);
int oec_cnn_correct(const oec_cnn_t *c, double scale32, const double *q_dev, double *q_hist_dev, int32_t *count_dev,
                    double *phi_dev, void *work_dev, void *stream);
/* bf16 parameters from f32 ones. */
int oec_cnn_set_weights(const oec_cnn_t *c, const float *w32_dev, void *stream);
/* One training step on one input x: z = N(x); the loss is either the
 * supervised sum(z-t)^2 / sum t^2 (op NULL, target t) or, with the scaled
 * FIT operator op (its ex32/ey32 weights), the scale-free residual loss
 * min_s sum(s A z - x)^2 / sum x^2 (target unused); numerator and
 * denominator go to loss_dev[2], sums over the inside nodes.  The gradient w.r.t. the parameters goes to grad_dev
 * (f32), and with update != 0 an Adam step (lr, beta 0.9 / 0.999,
 * step = 1, 2, ...) updates the f32 master weights w32_dev with moments m, v
 * and refreshes c->w16.  wt16_dev: bf16 scratch of oec_cnn_num_params()
 * entries (flipped weights of the data gradients).  c->act must hold
 * oec_cnn_act_bytes(nx, ny, 1) bytes. */
int oec_cnn_train_step(const oec_cnn_t *c, const oec_stencil_t *op, const float *x_dev, const float *target_dev,
                       float *z_dev, float *w32_dev, float *grad_dev, float *adam_m_dev, float *adam_v_dev,
                       void *wt16_dev, float lr, int32_t step, int32_t update, double *loss_dev, void *stream);

/* ------------------------------------------- grid geometry (A11-A14, host) */

/* Boundary function of the grid (grid.pyx:88-105). */
#define OEC_BOUND_RECT 0      /* p0 = lx/2, p1 = ly/2 (grid.pyx:1437) */
#define OEC_BOUND_ELLIPSE 1   /* p0 = 4/lx^2, p1 = 4/ly^2 (grid.pyx:1443) */
#define OEC_BOUND_POLYGON 2   /* poly: quadrant polygon, winding test of |x|,|y| */
#define OEC_BOUND_CALLBACK 3  /* fn(x, y, ctx) -> 0/1 (a user boundFunc) */
typedef int (*oec_bound_fn)(double x, double y, void *ctx);

typedef struct oec_geom_in {
    int32_t nx, ny;            /* nxExt, nyExt */
    double dx, dy;
    const double *x_mesh;      /* [nx] */
    const double *y_mesh;      /* [ny] */
    double scan_around_point;  /* relative probe offset (grid.pyx:49) */
    double cut_cell_acc;       /* bisection accuracy (cut-cell only) */
    int32_t cut_cell;          /* 0: staircase (grid.pyx:166), 1: cut-cell (:468) */
    int32_t bound_kind;        /* OEC_BOUND_* */
    double p0, p1;
    const double *poly;
    int32_t n_poly;
    oec_bound_fn fn;
    void *ctx;
} oec_geom_in_t;

/* Caller-allocated outputs; G = nx*ny.  Capacities: boundary points
 * cap_boundary_points (<= 2G), each COO stage cap_coo (8G is enough). */
typedef struct oec_geom_out {
    uint16_t *inside_points;   /* [G] */
    uint16_t *inside_edges;    /* [2G] x-edges then y-edges */
    uint16_t *inside_faces;    /* [G] */
    double *ds, *dsi;          /* [2G] */
    double *da, *dai;          /* [G] */
    double *dst, *dsti;        /* [2G] */
    double *dat, *dati;        /* [G] */
    double *boundary_points;   /* [cap_boundary_points*2] */
    uint32_t *boundary_points_ind;
    int32_t cap_boundary_points;
    int32_t n_boundary_points; /* out */
    int32_t *cut_cell_points_ind;  /* [G*2], -1 where unused */
    double *cut_cell_center;       /* [G*2] */
    double *cut_cell_normals;      /* [G*2] */
    int64_t cap_coo;
    int32_t *r1, *c1; double *v1; int64_t n1;  /* edge average (grid.pyx:390 / :900) */
    int32_t *r2, *c2; double *v2; int64_t n2;  /* boundary extrapolation (:432 / :1133) */
    int32_t *r3, *c3; double *v3; int64_t n3;  /* triangle cells (:1206); n3 = -1 if absent */
} oec_geom_out_t;

/* computeStaircaseGridGeom / computeCutCellGridGeom (grid.pyx:166-1330). */
int oec_grid_geometry(const oec_geom_in_t *in, oec_geom_out_t *out);

/* pointInPolygon (grid.pyx:108-120): 1 if (|x|,|y|) is inside. Not a status. */
int oec_point_in_polygon(const double *poly, int32_t n, double x, double y);

/* prepareBoundFuncPoints (grid.pyx:123-159): drop collinear vertices. */
int oec_polygon_prepare(const double *pts, int32_t n, double *out, int32_t *n_out);

/* ---------------------------------------------------------- fields, diagnostics */

/* multipoleExpansion (magneticField.pyx:23-59): B = [Bx | By | Bz=0] f64
 * [3*nx*ny] on the extended grid nodes (xmesh_dev [nx], ymesh_dev [ny]: the
 * node coordinates, Grid.getXMesh/getYMesh) from normal[n_normal] and
 * skew[n_skew] coefficients in T/m^k (host arrays, order <= 32; a shorter skew
 * list is padded with zeros, a longer one cut to n_normal). */
int oec_multipole_field(int32_t nx, int32_t ny, const double *xmesh_dev, const double *ymesh_dev,
                        const double *normal, int32_t n_normal, const double *skew, int32_t n_skew, double *b_dev,
                        void *stream);

/* averageEnergy (util.pyx:8-20): sums_dev[0] = sum |v|^2 w, sums_dev[1] =
 * sum w over the store (f64); the mean energy in eV is
 * m / (2 e) * sums[0] / sums[1]. */
int oec_average_energy_sums(const oec_particles_t *p, double *sums_dev, void *stream);

/* Index checks of the bounds-checked build (liboec_checked.so, built with
 * -DOEC_BOUNDS_CHECK): the number of out-of-range grid node and particle
 * indices that its kernels met and skipped since load (or the last reset);
 * -1 from the normal build, which does not check. */
int oec_bound_violations(int64_t *out, int32_t reset);

/* ------------------------------------- context and owned handles (session.cu)
 *
 * The layer above for hosts that bring no GPU framework of their own: a
 * context owns a device, a CUDA stream, a device status block and every
 * device allocation made through it (freed by oec_ctx_destroy); a run owns a
 * whole buildup run in its context.  The caller-owned entry points above
 * stay the low-level layer (oec_run_particles hands out the store in that
 * form).  A context and its runs are used from one host thread at a time. */
typedef struct oec_ctx oec_ctx_t;
typedef struct oec_run oec_run_t;

/* A context on CUDA device `device` (its own non-blocking stream). */
int oec_ctx_create(int32_t device, oec_ctx_t **out);
/* Waits for the context's stream, frees its allocations and runs' memory. */
int oec_ctx_destroy(oec_ctx_t *ctx);
/* The context's stream (cudaStream_t) for the low-level entry points. */
int oec_ctx_stream(oec_ctx_t *ctx, void **stream);
int oec_ctx_synchronize(oec_ctx_t *ctx);
/* `bytes` of zeroed device memory owned by the context. */
int oec_ctx_alloc(oec_ctx_t *ctx, int64_t bytes, void **dev);
/* Host copy of the context's status block (the anomaly counters of every
 * run of the context; synchronises its stream). */
int oec_status(oec_ctx_t *ctx, oec_status_t *out);

/* The LU factors as oec_lu_t lays them out, every pointer a HOST array of
 * the host-side setup (SuperLU's factors, poissonSolver.pyx:59, in the
 * head/tail form; tl_inv/tu_inv the dense inverses of the tail blocks).
 * Sizes: rhs_node/sol_src/sol_node n; l_rows/u_rows/u_diag head; l_ptr/u_ptr
 * head+1 (nnz = ptr[head]); lc_ptr m+1 (m = n - head); tl_inv/tu_inv m*m. */
typedef oec_lu_t oec_lu_host_t;

/* One buildup run (example01_basic.py:36-97).  HOST arrays, copied by
 * oec_run_create (not kept): rows (n_rows x 6 f64, setParticleData),
 * beam_profile (nx*ny: LHCBeam*.getTransversalProfile, beam.py:47-63),
 * beam_table (table_len: the beam's charge factor per step, beam.py:68-78 /
 * :129-136; the run holds table_len - 1 steps and table_len history
 * entries), the LU factors and the E operator phiToEAtGridPoints as CSR
 * (2*nx*ny rows, poissonSolver.pyx:63). */
typedef struct oec_run_desc {
    oec_grid_t grid;
    int32_t boundary_kind;      /* OEC_BOUNDARY_RECT or OEC_BOUNDARY_ELLIPSE */
    int32_t type_b;             /* borisPush typeBField 0 or 1 (bconst) */
    double dt, charge, mass;
    double bconst[3];
    int64_t capacity;           /* particle store (rounded up to a multiple of 1024) */
    int32_t abs_cap;            /* absorbed rows per step (more: status n_rows_dropped) */
    int32_t target;             /* globalRandom target */
    int32_t management_every;   /* globalRandom cadence in steps (+-5 % band) */
    int32_t table_len;
    const double *rows;
    int64_t n_rows;
    oec_furman_t furman;
    uint64_t emit_seed;         /* Philox key of the emission */
    uint64_t manage_seed;       /* Philox key of the roulette (plus the step) */
    const double *beam_profile;
    const double *beam_table;
    oec_lu_host_t lu;
    const int32_t *e_ptr, *e_idx;
    const double *e_val;
} oec_run_desc_t;

/* Allocates the run in ctx and loads its initial particles (their deposit
 * and the first history entry included); returns when the host arrays may
 * be released. */
int oec_run_create(oec_ctx_t *ctx, const oec_run_desc_t *desc, oec_run_t **out);
/* Advances n_steps time steps: every step the launch sequence of the loop
 * (beam + electron right-hand side, LU solve, E, fused push/gather/wall
 * test/deposit, absorbed set, wall rows, Furman emission, refill, history),
 * from a CUDA graph captured on the first call when use_graph != 0; at every
 * management_every-th step globalRandom toward target first.  Returns
 * OEC_ERR_CAPACITY past the beam table.  Synchronises at the end. */
int oec_run_steps(oec_run_t *run, int32_t n_steps, int32_t use_graph);
/* The first n history entries: macro count and sum of weights at the start
 * of each step (example01_basic.py:56-57). */
int oec_run_history(oec_run_t *run, int32_t *counts_host, double *weights_host, int32_t n);
/* getParticleData: up to max_rows (N, 6) f64 rows into rows_host; *n = N. */
int oec_run_get_rows(oec_run_t *run, double *rows_host, int64_t max_rows, int64_t *n);
/* The run's particle store in the low-level form (device arrays). */
int oec_run_particles(oec_run_t *run, oec_particles_t *out);
/* Releases the run's graph; its device memory goes with the context. */
int oec_run_destroy(oec_run_t *run);

#ifdef __cplusplus
}
#endif
#endif /* OEC_H */
