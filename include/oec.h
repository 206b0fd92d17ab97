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
    int32_t reserved[5];
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
 * min(50, 62 - ceil(log2(capacity))), so capacity * 2^bits <= 2^62 and no
 * node can leave the int64 range whatever the particle distribution. */
int oec_deposit_scale(const oec_particles_t *p, double *wscale_dev, void *stream);

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

/* ---------------------------------------------------- boundary (A17-A20) */

/* indexInside (particleBoundary.pyx:84-97 / :227-242 / :336-370): absorbed
 * bit per particle (1 = outside) and status->n_absorbed.  For the cut-cell
 * kind the positions are first clipped to the grid (:485-508). */
int oec_index_inside(const oec_grid_t *grid, oec_particles_t *p, const oec_boundary_t *boundary,
                     uint32_t *absorbed_mask_dev, oec_status_t *status_dev, void *stream);

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

#ifdef __cplusplus
}
#endif
#endif /* OEC_H */
