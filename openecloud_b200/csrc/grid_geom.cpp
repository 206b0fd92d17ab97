// grid_geom.cpp -- host construction of the extended-grid geometry.
//
// Restates grid.pyx: computeStaircaseGridGeom (:166-458) and
// computeCutCellGridGeom (:468-1330), pointInPolygon/_wn_PnPoly
// (:108-120, :1452-1480) and prepareBoundFuncPoints (:123-159).
// The geometry is built once per run on the host; the arrays it returns are
// the reference's, in the reference's layout (node index i + j*nxExt, x-edge
// block followed by the y-edge block), so that the Poisson operator and the
// cut-cell wall data match element for element.  The three sparse stages of
// the edge-to-node interpolation are returned as COO triplets and multiplied
// in the same order as the reference (stage3 * (stage2 * stage1)).
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "oec.h"

namespace {

struct Bound {
    const oec_geom_in_t *in;
    int operator()(double x, double y) const {
        switch (in->bound_kind) {
            case OEC_BOUND_RECT:  // grid.pyx:1437-1441
                return (x < in->p0 && x > -in->p0 && y < in->p1 && y > -in->p1) ? 1 : 0;
            case OEC_BOUND_ELLIPSE:  // grid.pyx:1443-1447 (x**2 is pow(x,2), exact)
                return (1 > x * x * in->p0 + y * y * in->p1) ? 1 : 0;
            case OEC_BOUND_POLYGON:
                return oec_point_in_polygon(in->poly, in->n_poly, x, y);
            default:
                return in->fn ? (in->fn(x, y, in->ctx) != 0 ? 1 : 0) : 0;
        }
    }
};

struct Coo {
    int32_t *r, *c;
    double *v;
    int64_t n, cap;
    bool ok = true;
    void add(int64_t row, int64_t col, double val) {
        if (n >= cap) {
            ok = false;
            return;
        }
        r[n] = (int32_t)row;
        c[n] = (int32_t)col;
        v[n] = val;
        ++n;
    }
};

// Zero pattern shared by both geometries for the primary-edge arrays
// (grid.pyx:240-273 / :565-597).
void zero_edge_frame(double *a, int nx, int ny, int np) {
    for (int i = 0; i < nx; ++i) {
        a[i] = 0.; a[i + nx] = 0.; a[i + (ny - 2) * nx] = 0.; a[i + (ny - 1) * nx] = 0.;
        a[i + np] = 0.; a[i + (ny - 2) * nx + np] = 0.; a[i + (ny - 1) * nx + np] = 0.;
    }
    for (int j = 1; j < ny - 2; ++j) {
        a[j * nx + np] = 0.; a[1 + j * nx + np] = 0.; a[(nx - 2) + j * nx + np] = 0.; a[(nx - 1) + j * nx + np] = 0.;
    }
    for (int j = 2; j < ny - 2; ++j) {
        a[j * nx] = 0.; a[(nx - 2) + j * nx] = 0.; a[(nx - 1) + j * nx] = 0.;
    }
}

// Zero pattern of the face arrays (grid.pyx:304-319).
template <typename T>
void zero_face_frame(T *a, int nx, int ny) {
    for (int i = 0; i < nx; ++i) {
        a[i] = 0; a[i + (ny - 2) * nx] = 0; a[i + (ny - 1) * nx] = 0;
    }
    for (int j = 1; j < ny - 2; ++j) {
        a[j * nx] = 0; a[(nx - 2) + j * nx] = 0; a[(nx - 1) + j * nx] = 0;
    }
}

void inside_points(const oec_geom_in_t &in, const Bound &f, uint16_t *ip) {
    const int nx = in.nx, ny = in.ny;
    const double *xm = in.x_mesh, *ym = in.y_mesh;
    const double ex = in.scan_around_point * in.dx, ey = in.scan_around_point * in.dy;
    for (int i = 0; i < nx; ++i) {
        ip[i] = 0; ip[i + nx] = 0; ip[i + (ny - 2) * nx] = 0; ip[i + (ny - 1) * nx] = 0;
    }
    for (int j = 2; j < ny - 2; ++j) {
        ip[j * nx] = 0; ip[1 + j * nx] = 0; ip[(nx - 2) + j * nx] = 0; ip[(nx - 1) + j * nx] = 0;
    }
    // grid.pyx:205-213: all four probe points around the node must be inside.
    for (int i = 2; i < nx - 2; ++i)
        for (int j = 2; j < ny - 2; ++j)
            ip[i + j * nx] = (f(xm[i] + ex, ym[j] + ey) && f(xm[i] + ex, ym[j] - ey) && f(xm[i] - ex, ym[j] + ey) &&
                              f(xm[i] - ex, ym[j] - ey))
                                 ? 1
                                 : 0;
}

void inside_edges(int nx, int ny, int np, const uint16_t *ip, uint16_t *ie) {
    for (int i = 0; i < nx; ++i) {
        ie[i] = 0; ie[i + nx] = 0; ie[i + (ny - 2) * nx] = 0; ie[i + (ny - 1) * nx] = 0;
        ie[i + np] = 0; ie[i + (ny - 1) * nx + np] = 0;
    }
    for (int j = 0; j < ny; ++j) {
        ie[j * nx + np] = 0; ie[1 + j * nx + np] = 0; ie[(nx - 2) + j * nx + np] = 0; ie[(nx - 1) + j * nx + np] = 0;
        ie[j * nx] = 0; ie[(nx - 1) + j * nx] = 0;
    }
    // 0 outside, 1 one endpoint inside (boundary / cut edge), 2 inside.
    for (int j = 2; j < ny - 2; ++j)
        for (int i = 1; i < nx - 1; ++i) ie[i + j * nx] = ip[i + j * nx] + ip[i + 1 + j * nx];
    for (int j = 1; j < ny - 1; ++j)
        for (int i = 2; i < nx - 2; ++i) ie[i + j * nx + np] = ip[i + j * nx] + ip[i + (j + 1) * nx];
}

void faces_from_edges(int nx, int ny, int np, const uint16_t *ie, uint16_t *fa) {
    zero_face_frame(fa, nx, ny);
    for (int j = 1; j < ny - 2; ++j)
        for (int i = 1; i < nx - 2; ++i) {
            int c = i + j * nx;
            fa[c] = ie[c] + ie[c + nx] + ie[c + np] + ie[c + 1 + np];
        }
}

// Dual edge lengths and dual areas (identical for both geometries,
// grid.pyx:348-386 / :861-898).
void dual_grid(const oec_geom_in_t &in, oec_geom_out_t *o) {
    const int nx = in.nx, ny = in.ny, np = nx * ny;
    const double dx = in.dx, dy = in.dy, dxi = 1. / dx, dyi = 1. / dy;
    const double dxh = 0.5 * dx, dyh = 0.5 * dy, dxhi = 1. / dxh, dyhi = 1. / dyh;
    double *dst = o->dst, *dsti = o->dsti;
    for (int i = 0; i < nx; ++i) {
        dst[i] = 0.; dst[i + (ny - 1) * nx] = 0.; dst[i + np] = 0.; dst[i + (ny - 1) * nx + np] = 0.;
        dsti[i] = 0.; dsti[i + (ny - 1) * nx] = 0.; dsti[i + np] = 0.; dsti[i + (ny - 1) * nx + np] = 0.;
    }
    for (int j = 1; j < ny - 1; ++j) {
        dst[j * nx] = 0.; dst[(nx - 1) + j * nx] = 0.; dst[j * nx + np] = 0.; dst[(nx - 1) + j * nx + np] = 0.;
        dsti[j * nx] = 0.; dsti[(nx - 1) + j * nx] = 0.; dsti[j * nx + np] = 0.; dsti[(nx - 1) + j * nx + np] = 0.;
    }
    for (int i = 2; i < nx - 2; ++i)
        for (int j = 1; j < ny - 1; ++j) {
            dst[i + j * nx] = dx;
            dsti[i + j * nx] = dxi;
        }
    for (int i = 1; i < nx - 1; ++i)
        for (int j = 2; j < ny - 2; ++j) {
            dst[i + j * nx + np] = dy;
            dsti[i + j * nx + np] = dyi;
        }
    for (int j = 1; j < ny - 1; ++j) {
        dst[1 + j * nx] = dxh; dst[(nx - 2) + j * nx] = dxh;
        dsti[1 + j * nx] = dxhi; dsti[(nx - 2) + j * nx] = dxhi;
    }
    for (int i = 1; i < nx - 1; ++i) {
        dst[i + nx + np] = dyh; dst[i + (ny - 2) * nx + np] = dyh;
        dsti[i + nx + np] = dyhi; dsti[i + (ny - 2) * nx + np] = dyhi;
    }
    for (int c = 0; c < np; ++c) {
        o->dat[c] = dst[c] * dst[c + np];
        o->dati[c] = dsti[c] * dsti[c + np];
    }
}

// ------------------------------------------------------------ staircase
int staircase(const oec_geom_in_t &in, const Bound &f, oec_geom_out_t *o) {
    const int nx = in.nx, ny = in.ny, np = nx * ny;
    const double dx = in.dx, dy = in.dy, dxi = 1. / dx, dyi = 1. / dy, dxdy = dx * dy, dxdyi = 1. / dxdy;
    uint16_t *ip = o->inside_points, *ie = o->inside_edges, *fa = o->inside_faces;
    double *ds = o->ds, *dsi = o->dsi;
    inside_points(in, f, ip);
    inside_edges(nx, ny, np, ip, ie);
    zero_edge_frame(ds, nx, ny, np);
    zero_edge_frame(dsi, nx, ny, np);
    for (int j = 2; j < ny - 2; ++j)
        for (int i = 1; i < nx - 2; ++i) {
            int c = i + j * nx;
            ds[c] = ie[c] == 0 ? 0. : dx;
            dsi[c] = ie[c] == 0 ? 0. : dxi;
        }
    for (int j = 1; j < ny - 2; ++j)
        for (int i = 2; i < nx - 2; ++i) {
            int c = i + j * nx + np;
            ds[c] = ie[c] == 0 ? 0. : dy;
            dsi[c] = ie[c] == 0 ? 0. : dyi;
        }
    faces_from_edges(nx, ny, np, ie, fa);
    zero_face_frame(o->da, nx, ny);
    zero_face_frame(o->dai, nx, ny);
    for (int j = 1; j < ny - 2; ++j)
        for (int i = 1; i < nx - 2; ++i) {
            int c = i + j * nx;
            o->da[c] = fa[c] == 0 ? 0. : dxdy;
            o->dai[c] = fa[c] == 0 ? 0. : dxdyi;
        }
    dual_grid(in, o);
    o->n_boundary_points = 0;
    for (int c = 0; c < 2 * np; ++c) o->cut_cell_points_ind[c] = -1;
    memset(o->cut_cell_center, 0, sizeof(double) * 2 * np);
    memset(o->cut_cell_normals, 0, sizeof(double) * 2 * np);

    // Stage 1: edge average to inside nodes (grid.pyx:390-427).
    Coo s1{o->r1, o->c1, o->v1, 0, o->cap_coo};
    for (int i = 1; i < nx - 2; ++i)
        for (int j = 2; j < ny - 2; ++j) {
            int c = i + j * nx;
            if (ip[c] == 1) s1.add(c, c, ds[c] / (ds[c - 1] + ds[c]));
        }
    for (int i = 2; i < nx - 1; ++i)
        for (int j = 2; j < ny - 2; ++j) {
            int c = i + j * nx;
            if (ip[c] == 1) s1.add(c, c - 1, ds[c - 1] / (ds[c - 1] + ds[c]));
        }
    for (int i = 2; i < nx - 2; ++i)
        for (int j = 1; j < ny - 2; ++j) {
            int c = i + j * nx;
            if (ip[c] == 1) s1.add(c + np, c + np, ds[c + np] / (ds[c + np - nx] + ds[c + np]));
        }
    for (int i = 2; i < nx - 2; ++i)
        for (int j = 2; j < ny - 1; ++j) {
            int c = i + j * nx;
            if (ip[c] == 1) s1.add(c + np, c + np - nx, ds[c + np - nx] / (ds[c + np - nx] + ds[c + np]));
        }
    // Stage 2: copy the neighbouring inside value to boundary nodes
    // (grid.pyx:432-456; the y entries land in the x rows as written there).
    Coo s2{o->r2, o->c2, o->v2, 0, o->cap_coo};
    for (int j = 1; j < ny - 1; ++j)
        for (int i = 1; i < nx - 1; ++i) {
            int c = i + j * nx;
            if (ip[c] == 1) {
                s2.add(c, c, 1.);
                s2.add(c + np, c + np, 1.);
                continue;
            }
            if (ie[c] == 1) {
                if (ip[c + nx] == 1 && ip[c - nx] == 1) s2.add(c, c + 1, 1.);
            } else if (ie[c - 1] == 1) {
                if (ip[c + nx] == 1 && ip[c - nx] == 1) s2.add(c, c - 1, 1.);
            }
            if (ie[c + np] == 1) {
                if (ip[c + 1] == 1 && ip[c - 1] == 1) s2.add(c, c + nx, 1.);
            } else if (ie[c + np - nx] == 1) {
                if (ip[c + 1] == 1 && ip[c - 1] == 1) s2.add(c, c - nx, 1.);
            }
        }
    o->n1 = s1.n;
    o->n2 = s2.n;
    o->n3 = -1;  // no third stage for staircase grids
    return (s1.ok && s2.ok) ? OEC_OK : OEC_ERR_HOST;
}

// ------------------------------------------------------------- cut-cell
int cutcell(const oec_geom_in_t &in, const Bound &f, oec_geom_out_t *o) {
    const int nx = in.nx, ny = in.ny, np = nx * ny;
    const double dx = in.dx, dy = in.dy, dxi = 1. / dx, dyi = 1. / dy, dxdy = dx * dy, dxdyi = 1. / dxdy;
    const double *xm = in.x_mesh, *ym = in.y_mesh;
    const unsigned iters = (unsigned)(log2(1. / in.cut_cell_acc) + 2.);
    uint16_t *ip = o->inside_points, *ie = o->inside_edges, *fa = o->inside_faces;
    double *ds = o->ds, *dsi = o->dsi;
    inside_points(in, f, ip);
    inside_edges(nx, ny, np, ip, ie);
    zero_edge_frame(ds, nx, ny, np);
    zero_edge_frame(dsi, nx, ny, np);

    // Cut edge lengths by bisection of the boundary function (grid.pyx:600-661).
    for (int j = 2; j < ny - 2; ++j)
        for (int i = 1; i < nx - 2; ++i) {
            int c = i + j * nx;
            if (ie[c] == 2) {
                ds[c] = dx;
                dsi[c] = dxi;
            } else if (ie[c] == 0) {
                ds[c] = 0.;
                dsi[c] = 0.;
            } else {
                double a = xm[i], b = xm[i + 1], y = ym[j];
                int fa_ = f(a, y), fb = f(b, y);
                if (fa_ == 1 && fb == 1) {
                    ds[c] = dx;
                } else {
                    for (unsigned k = 0; k < iters; ++k) {
                        double m = 0.5 * (a + b);
                        int fm = f(m, y);
                        if (fa_ == fm) { a = m; fa_ = fm; } else { b = m; fb = fm; }
                    }
                    ds[c] = ip[c] == 1 ? 0.5 * (a + b) - xm[i] : xm[i + 1] - 0.5 * (a + b);
                }
                dsi[c] = 1. / ds[c];
            }
        }
    for (int j = 1; j < ny - 2; ++j)
        for (int i = 2; i < nx - 2; ++i) {
            int c = i + j * nx, e = c + np;
            if (ie[e] == 2) {
                ds[e] = dy;
                dsi[e] = dyi;
            } else if (ie[e] == 0) {
                ds[e] = 0.;
                dsi[e] = 0.;
            } else {
                double a = ym[j], b = ym[j + 1], x = xm[i];
                int fa_ = f(x, a), fb = f(x, b);
                if (fa_ == 1 && fb == 1) {
                    ds[e] = dy;
                } else {
                    for (unsigned k = 0; k < iters; ++k) {
                        double m = 0.5 * (a + b);
                        int fm = f(x, m);
                        if (fa_ == fm) { a = m; fa_ = fm; } else { b = m; fb = fm; }
                    }
                    ds[e] = ip[c] == 1 ? 0.5 * (a + b) - ym[j] : ym[j + 1] - 0.5 * (a + b);
                }
                dsi[e] = 1. / ds[e];
            }
        }

    // Boundary points on cut edges and the two per cut cell (grid.pyx:664-719).
    double *bp = o->boundary_points;
    uint32_t *bpi = o->boundary_points_ind;
    int32_t *cpi = o->cut_cell_points_ind;
    for (int c = 0; c < 2 * np; ++c) cpi[c] = -1;
    auto attach = [&](int cell, int k) {
        if (cpi[2 * cell] == -1)
            cpi[2 * cell] = k;
        else
            cpi[2 * cell + 1] = k;
    };
    int k = 0;
    for (int j = 1; j < ny - 1; ++j)
        for (int i = 1; i < nx - 1; ++i) {
            int c = i + j * nx;
            if (ie[c] == 1) {
                if (k >= o->cap_boundary_points) return OEC_ERR_HOST;
                if (ip[c] == 1) {
                    bp[2 * k] = xm[i] + ds[c];
                    bp[2 * k + 1] = ym[j];
                    bpi[k] = c + 1;
                } else {
                    bp[2 * k] = xm[i + 1] - ds[c];
                    bp[2 * k + 1] = ym[j];
                    bpi[k] = c;
                }
                attach(c, k);
                attach(c - nx, k);
                ++k;
            }
            if (ie[c + np] == 1) {
                if (k >= o->cap_boundary_points) return OEC_ERR_HOST;
                if (ip[c] == 1) {
                    bp[2 * k] = xm[i];
                    bp[2 * k + 1] = ym[j] + ds[c + np];
                    bpi[k] = c + nx + np;
                } else {
                    bp[2 * k] = xm[i];
                    bp[2 * k + 1] = ym[j + 1] - ds[c + np];
                    bpi[k] = c + np;
                }
                attach(c, k);
                attach(c - 1, k);
                ++k;
            }
        }
    o->n_boundary_points = k;

    faces_from_edges(nx, ny, np, ie, fa);

    // Cut-cell centres and counter-clockwise ordering of the two points
    // (grid.pyx:723-790).
    double *cc = o->cut_cell_center;
    memset(cc, 0, sizeof(double) * 2 * np);
    for (int j = 1; j < ny - 1; ++j)
        for (int i = 1; i < nx - 1; ++i) {
            int c = i + j * nx;
            if (fa[c] == 0 || fa[c] == 8) continue;
            double *x = cc + 2 * c, *y = cc + 2 * c + 1;
            if (fa[c] == 2) {
                if (ip[c] == 1) { *x = xm[i] + ds[c] / 3.; *y = ym[j] + ds[c + np] / 3.; }
                else if (ip[c + 1] == 1) { *x = xm[i + 1] - ds[c] / 3.; *y = ym[j] + ds[c + np + 1] / 3.; }
                else if (ip[c + nx] == 1) { *x = xm[i] + ds[c + nx] / 3.; *y = ym[j + 1] - ds[c + np] / 3.; }
                else if (ip[c + nx + 1] == 1) { *x = xm[i + 1] - ds[c + nx] / 3.; *y = ym[j + 1] - ds[c + np + 1] / 3.; }
            } else if (fa[c] == 4) {
                if (ip[c] == 1 && ip[c + 1] == 1) {
                    *x = (xm[i] + xm[i + 1]) * 0.5;
                    *y = ym[j] + (ds[c + np] + ds[c + np + 1]) * 0.25;
                } else if (ip[c + nx] == 1 && ip[c + nx + 1] == 1) {
                    *x = (xm[i] + xm[i + 1]) * 0.5;
                    *y = ym[j + 1] - (ds[c + np] + ds[c + np + 1]) * 0.25;
                } else if (ip[c] == 1 && ip[c + nx] == 1) {
                    *x = xm[i] + (ds[c] + ds[c + nx]) * 0.25;
                    *y = (ym[j] + ym[j + 1]) * 0.5;
                } else if (ip[c + 1] == 1 && ip[c + nx + 1] == 1) {
                    *x = xm[i + 1] - (ds[c] + ds[c + nx]) * 0.25;
                    *y = (ym[j] + ym[j + 1]) * 0.5;
                }
            } else if (fa[c] == 6) {
                if (ip[c] == 0) {
                    *x = (2. * xm[i] + 3. * xm[i + 1] - ds[c]) * 0.2;
                    *y = (2. * ym[j] + 3. * ym[j + 1] - ds[c + np]) * 0.2;
                } else if (ip[c + 1] == 0) {
                    *x = (3. * xm[i] + 2. * xm[i + 1] + ds[c]) * 0.2;
                    *y = (2. * ym[j] + 3. * ym[j + 1] - ds[c + np + 1]) * 0.2;
                } else if (ip[c + nx] == 0) {
                    *x = (2. * xm[i] + 3. * xm[i + 1] - ds[c + nx]) * 0.2;
                    *y = (3. * ym[j] + 2. * ym[j + 1] + ds[c + np]) * 0.2;
                } else if (ip[c + nx + 1] == 0) {
                    *x = (3. * xm[i] + 2. * xm[i + 1] + ds[c + nx]) * 0.2;
                    *y = (3. * ym[j] + 2. * ym[j + 1] + ds[c + np + 1]) * 0.2;
                }
            }
            int a = cpi[2 * c], b = cpi[2 * c + 1];
            if (a < 0 || b < 0) continue;  // a cell with a single cut point: nothing to order
            if ((bp[2 * a] - *x) * (bp[2 * b + 1] - *y) < (bp[2 * a + 1] - *y) * (bp[2 * b] - *x)) {
                cpi[2 * c] = b;
                cpi[2 * c + 1] = a;
            }
        }

    // Wall normals of the cut cells (grid.pyx:792-805).
    double *cn = o->cut_cell_normals;
    memset(cn, 0, sizeof(double) * 2 * np);
    for (int j = 1; j < ny - 1; ++j)
        for (int i = 1; i < nx - 1; ++i) {
            int c = i + j * nx;
            if (fa[c] == 0 || fa[c] == 8) continue;
            int a = cpi[2 * c], b = cpi[2 * c + 1];
            if (a < 0 || b < 0) continue;
            double u = bp[2 * a + 1] - bp[2 * b + 1];
            double v = bp[2 * b] - bp[2 * a];
            double inv = 1. / sqrt(u * u + v * v);
            cn[2 * c] = u * inv;
            cn[2 * c + 1] = v * inv;
        }

    // Face areas (grid.pyx:807-853).
    double *da = o->da, *dai = o->dai;
    zero_face_frame(da, nx, ny);
    zero_face_frame(dai, nx, ny);
    for (int j = 1; j < ny - 2; ++j)
        for (int i = 1; i < nx - 2; ++i) {
            int c = i + j * nx;
            if (fa[c] == 8) {
                da[c] = dxdy;
                dai[c] = dxdyi;
            } else if (fa[c] == 0) {
                da[c] = 0.;
                dai[c] = 0.;
            } else if (fa[c] == 2) {
                if (ip[c] == 1) da[c] = 0.5 * ds[c] * ds[c + np];
                else if (ip[c + 1] == 1) da[c] = 0.5 * ds[c] * ds[c + 1 + np];
                else if (ip[c + nx] == 1) da[c] = 0.5 * ds[c + nx] * ds[c + np];
                else da[c] = 0.5 * ds[c + nx] * ds[c + 1 + np];
                dai[c] = 1. / da[c];
            } else if (fa[c] == 4) {
                da[c] = 0.5 * (ds[c] + ds[c + nx]) * (ds[c + np] + ds[c + 1 + np]);
                dai[c] = 1. / da[c];
            } else if (fa[c] == 6) {
                if (ip[c] == 0) da[c] = dxdy - 0.5 * (dx - ds[c]) * (dy - ds[c + np]);
                else if (ip[c + 1] == 0) da[c] = dxdy - 0.5 * (dx - ds[c]) * (dy - ds[c + 1 + np]);
                else if (ip[c + nx] == 0) da[c] = dxdy - 0.5 * (dx - ds[c + nx]) * (dy - ds[c + np]);
                else da[c] = dxdy - 0.5 * (dx - ds[c + nx]) * (dy - ds[c + 1 + np]);
                dai[c] = 1. / da[c];
            }
        }
    dual_grid(in, o);

    // Stage 1: edge average to inside nodes (grid.pyx:900-925).
    Coo s1{o->r1, o->c1, o->v1, 0, o->cap_coo};
    for (int i = 2; i < nx - 2; ++i)
        for (int j = 2; j < ny - 2; ++j) {
            int c = i + j * nx;
            if (ip[c] != 1) continue;
            s1.add(c, c, ds[c] / (ds[c - 1] + ds[c]));
            s1.add(c, c - 1, ds[c - 1] / (ds[c - 1] + ds[c]));
            int e = c + np;
            s1.add(e, e, ds[e] / (ds[e - nx] + ds[e]));
            s1.add(e, e - nx, ds[e - nx] / (ds[e - nx] + ds[e]));
        }

    // Stage 2: boundary nodes average their connected cut edges
    // (grid.pyx:1133-1203).
    std::vector<double> cei(np, 0.);
    for (int j = 1; j < ny - 1; ++j)
        for (int i = 1; i < nx - 1; ++i) {
            int c = i + j * nx;
            if (ip[c] == 0) cei[c] = ie[c] + ie[c - 1] + ie[c + np] + ie[c - nx + np];
            if (cei[c] > 1.) cei[c] = 1. / cei[c];
        }
    Coo s2{o->r2, o->c2, o->v2, 0, o->cap_coo};
    for (int j = 1; j < ny - 1; ++j)
        for (int i = 1; i < nx - 1; ++i) {
            int c = i + j * nx;
            if (ip[c] == 1) {
                s2.add(c, c, 1.);
                s2.add(c + np, c + np, 1.);
                continue;
            }
            if (ie[c] == 1) {
                s2.add(c, c + 1, cei[c]);
                s2.add(c + np, c + np + 1, cei[c]);
            } else if (ie[c - 1] == 1) {
                s2.add(c, c - 1, cei[c]);
                s2.add(c + np, c + np - 1, cei[c]);
            }
            if (ie[c + np] == 1) {
                s2.add(c, c + nx, cei[c]);
                s2.add(c + np, c + np + nx, cei[c]);
            }
            if (ie[c + np - nx] == 1) {
                s2.add(c, c - nx, cei[c]);
                s2.add(c + np, c + np - nx, cei[c]);
            }
        }

    // Stage 3: linear extrapolation into triangular boundary cells
    // (grid.pyx:1206-1330).
    Coo s3{o->r3, o->c3, o->v3, 0, o->cap_coo};
    auto tri = [&](int c, int diag, int side1, int side2) {
        s3.add(c, diag, -1.);
        s3.add(c, side1, 1.);
        s3.add(c, side2, 1.);
        s3.add(c + np, diag + np, -1.);
        s3.add(c + np, side1 + np, 1.);
        s3.add(c + np, side2 + np, 1.);
    };
    for (int j = 1; j < ny - 1; ++j)
        for (int i = 1; i < nx - 1; ++i) {
            int c = i + j * nx;
            s3.add(c, c, 1.);
            s3.add(c + np, c + np, 1.);
            if (ip[c] != 0) continue;
            if (ip[c - 1] == 0 && ip[c + nx] == 0 && ip[c - 1 + nx] == 1)
                tri(c, c - 1 + nx, c - 1, c + nx);
            else if (ip[c + 1] == 0 && ip[c + nx] == 0 && ip[c + 1 + nx] == 1)
                tri(c, c + 1 + nx, c + 1, c + nx);
            else if (ip[c + 1] == 0 && ip[c - nx] == 0 && ip[c + 1 - nx] == 1)
                tri(c, c + 1 - nx, c + 1, c - nx);
            else if (ip[c - 1] == 0 && ip[c - nx] == 0 && ip[c - 1 - nx] == 1)
                tri(c, c - 1 - nx, c - 1, c - nx);
        }
    o->n1 = s1.n;
    o->n2 = s2.n;
    o->n3 = s3.n;
    return (s1.ok && s2.ok && s3.ok) ? OEC_OK : OEC_ERR_HOST;
}

int is_left(const double *p0, const double *p1, const double *p2) {
    double r = (p1[0] - p0[0]) * (p2[1] - p0[1]) - (p2[0] - p0[0]) * (p1[1] - p0[1]);
    return r > 0 ? 1 : (r < 0 ? -1 : 0);
}

}  // namespace

// Winding-number test of (|x|, |y|) against the quadrant polygon
// (grid.pyx:108-120, :1464-1480).  The polygon is closed implicitly: the last
// edge runs from the last vertex back to the first.
extern "C" int oec_point_in_polygon(const double *poly, int32_t n, double x, double y) {
    if (!poly || n < 2) return 0;
    double p[2] = {fabs(x), fabs(y)};
    int wn = 0;
    for (int i = 0; i < n; ++i) {
        const double *a = poly + 2 * i;
        const double *b = poly + 2 * ((i + 1) % n);
        if (a[1] <= p[1]) {
            if (b[1] > p[1] && is_left(a, b, p) > 0) ++wn;
        } else {
            if (b[1] <= p[1] && is_left(a, b, p) < 0) --wn;
        }
    }
    return wn != 0 ? 1 : 0;
}

// Drop (nearly) collinear interior vertices (grid.pyx:123-159).
extern "C" int oec_polygon_prepare(const double *pts, int32_t n, double *out, int32_t *n_out) {
    if (!pts || !out || !n_out || n < 0) return OEC_ERR_INVALID;
    std::vector<char> keep(n, 1);
    int i = 0;
    while (i + 2 < n) {
        int inc = 0;
        while (i + 2 + inc < n) {
            const double *a = pts + 2 * i, *b = pts + 2 * (i + 1), *c = pts + 2 * (i + 1 + inc),
                         *d = pts + 2 * (i + 2 + inc);
            double min_area = 1.e-16 * (sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1])) *
                                        sqrt((c[0] - d[0]) * (c[0] - d[0]) + (c[1] - d[1]) * (c[1] - d[1])));
            double area = a[0] * (c[1] - d[1]) + c[0] * (d[1] - a[1]) + d[0] * (a[1] - c[1]);
            if (fabs(min_area) > fabs(area))
                ++inc;
            else
                break;
        }
        for (int j = i + 1; j < i + inc + 1; ++j) keep[j] = 0;
        i += inc + 1;
    }
    int m = 0;
    for (int j = 0; j < n; ++j)
        if (keep[j]) {
            out[2 * m] = pts[2 * j];
            out[2 * m + 1] = pts[2 * j + 1];
            ++m;
        }
    *n_out = m;
    return OEC_OK;
}

extern "C" int oec_grid_geometry(const oec_geom_in_t *in, oec_geom_out_t *out) {
    if (!in || !out || in->nx < 5 || in->ny < 5 || !in->x_mesh || !in->y_mesh || !(in->dx > 0) || !(in->dy > 0))
        return OEC_ERR_INVALID;
    if (in->bound_kind == OEC_BOUND_CALLBACK && !in->fn) return OEC_ERR_INVALID;
    if (in->bound_kind == OEC_BOUND_POLYGON && (!in->poly || in->n_poly < 2)) return OEC_ERR_INVALID;
    if (in->cut_cell && !(in->cut_cell_acc > 0)) return OEC_ERR_INVALID;
    Bound f{in};
    return in->cut_cell ? cutcell(*in, f, out) : staircase(*in, f, out);
}
