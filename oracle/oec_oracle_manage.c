/*
 * oec_oracle_manage.c -- CPU restatement of particle management: the three
 * compaction variants of addAndRemoveParticles (particles.pyx:94-121,
 * :201-269), sortByColumn's random-pivot quicksort (particles.pyx:431-459),
 * globalRandom (particleManagement.pyx:35-67), localRandom with its
 * _searchSorted (particleManagement.pyx:74-262) and the sliding-midpoint
 * kd-tree (kdTree.pyx:19-257).  TEST INFRASTRUCTURE ONLY (see oec_oracle.c).
 *
 * The random calls go to the same global MT19937 stand-in the reference is
 * linked with, in the reference's order, so a seeded run replays the
 * compiled reference exactly.  Data: (n, 6) rows [x, y, vx, vy, vz, w].
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define NC 6
double orc_rand(void);
unsigned long orc_randi(unsigned long n);

/* ------------------------------------------- particles.pyx:94-121 + :201-269
 * data has room for `cap` rows; returns the new count (or -1 if the rows do
 * not fit, when the reference would allocate a larger array). */
int64_t orc_add_and_remove(double *data, int64_t cap, int64_t n_old, const double *add, int64_t n_add,
                           const uint16_t *keep) {
    int64_t n_keep = 0;
    for (int64_t i = 0; i < n_old; ++i) n_keep += keep[i];
    int64_t n_new = n_keep + n_add;
    if (n_add == 0 && n_keep == n_old) return n_old;
    if (n_add == 0) {
        /* _removeParticles: the last kept row fills each hole */
        int64_t l = n_old;
        for (int64_t j = 0; j < n_new; ++j) {
            if (keep[j] == 0) {
                do { --l; } while (keep[l] != 1);
                memcpy(data + NC * j, data + NC * l, NC * sizeof(double));
            }
        }
        return n_new;
    }
    if (n_new > cap) {
        /* the reference allocates a larger array and writes the kept rows in
         * order followed by the added rows (_addAndRemoveParticlesNewArray);
         * `data` has room for n_new rows here */
        double *tmp = (double *)malloc(sizeof(double) * NC * (size_t)n_new);
        int64_t j = 0;
        for (int64_t i = 0; i < n_old; ++i)
            if (keep[i] == 1) memcpy(tmp + NC * j++, data + NC * i, NC * sizeof(double));
        memcpy(tmp + NC * j, add, NC * sizeof(double) * (size_t)n_add);
        memcpy(data, tmp, sizeof(double) * NC * (size_t)n_new);
        free(tmp);
        return n_new;
    }
    /* _addAndRemoveParticles (in place) */
    int64_t ii = 0, jj = 0;
    while (ii < n_add && jj < n_old) {
        if (keep[jj] == 0) {
            memcpy(data + NC * jj, add + NC * ii, NC * sizeof(double));
            ++ii;
        }
        ++jj;
    }
    if (ii == n_add) {
        ii = jj - n_add;
        while (ii < n_keep) {
            if (keep[jj] == 1) {
                memcpy(data + NC * (ii + n_add), data + NC * jj, NC * sizeof(double));
                ++ii;
            }
            ++jj;
        }
    } else if (jj == n_old) {
        while (ii < n_add) {
            memcpy(data + NC * jj, add + NC * ii, NC * sizeof(double));
            ++ii;
            ++jj;
        }
    }
    return n_new;
}

/* _addAndRemoveParticlesNewArray (:201-219): kept rows then added rows. */
int64_t orc_add_and_remove_new_array(const double *data, int64_t n_old, const double *add, int64_t n_add,
                                     const uint16_t *keep, double *out) {
    int64_t j = 0;
    for (int64_t i = 0; i < n_old; ++i)
        if (keep[i] == 1) memcpy(out + NC * j++, data + NC * i, NC * sizeof(double));
    memcpy(out + NC * j, add, NC * sizeof(double) * n_add);
    return j + n_add;
}

/* ---------------------------------------------- particles.pyx:431-459 */
static void swap_rows(double *a, int64_t i, int64_t j) {
    double t[NC];
    memcpy(t, a + NC * i, sizeof t);
    memcpy(a + NC * i, a + NC * j, sizeof t);
    memcpy(a + NC * j, t, sizeof t);
}

void orc_quicksort_by_column(double *a, int64_t left, int64_t right, int col) {
    if (left >= right) return;
    int64_t piv = left + (int64_t)orc_randi((unsigned long)(right - left));
    double pv = a[NC * piv + col];
    swap_rows(a, piv, right);
    int64_t nr = left;
    for (int64_t i = left; i < right; ++i) {
        if (a[NC * i + col] <= pv) {
            swap_rows(a, i, nr);
            ++nr;
        }
    }
    swap_rows(a, nr, right);
    int64_t nl = nr;
    while (nl > left && a[NC * (nl - 1) + col] == pv) --nl;
    orc_quicksort_by_column(a, left, nl - 1, col);
    orc_quicksort_by_column(a, nr + 1, right, col);
}

/* ------------------------------------- particleManagement.pyx:35-67
 * out must hold max(n, target) rows; returns the new count. */
int64_t orc_global_random(double *data, int64_t n, int64_t target, double *scratch) {
    int64_t diff = n - target;
    double factor = (double)n / (double)target;
    unsigned long ri = orc_randi((unsigned long)n);
    uint16_t *keep = (uint16_t *)malloc(sizeof(uint16_t) * (n > 0 ? n : 1));
    for (int64_t i = 0; i < n; ++i) keep[i] = 1;
    int64_t res = n;
    if (diff > 0) {
        for (int64_t i = 0; i < n; ++i) data[NC * i + 5] *= factor;
        for (int64_t k = 0; k < diff; ++k) {
            while (keep[ri] == 0) ri = orc_randi((unsigned long)n);
            keep[ri] = 0;
        }
        res = orc_add_and_remove(data, n, n, NULL, 0, keep);
    } else if (target > n) {
        int64_t na = -diff;
        for (int64_t i = 0; i < n; ++i) data[NC * i + 5] *= factor;
        for (int64_t k = 0; k < na; ++k) {
            ri = orc_randi((unsigned long)n);
            memcpy(scratch + NC * k, data + NC * ri, NC * sizeof(double));
        }
        res = orc_add_and_remove(data, target, n, scratch, na, keep);
    }
    free(keep);
    return res;
}

/* ------------------------------------------------- kdTree.pyx:19-257 */
typedef struct Node {
    struct Node *left, *right;
    double loc;
    unsigned axis, leaf;
    unsigned *inds;
} Node;

typedef struct {
    const double *data;  /* rows of stride NC, first 5 coords used */
    const double *w;     /* phase-space weights [5] */
    unsigned n;
    Node *root, *last;
    unsigned *inds;
} Tree;

static Node *kd_build(const double *data, unsigned *inds, unsigned np, const double *mins, const double *maxs,
                      const double *w, unsigned leaf) {
    const double eps = DBL_EPSILON;
    Node *nd;
    if (np < 1) return NULL;
    nd = (Node *)calloc(1, sizeof(Node));
    if (np <= leaf) {
        nd->inds = inds;
        nd->leaf = np;
        return nd;
    }
    double span = 0.;
    unsigned ax = 5;
    for (unsigned i = 0; i < 5; ++i) {
        if (span <= maxs[i] - mins[i]) {
            span = maxs[i] - mins[i];
            ax = i;
        }
    }
    if (span <= sqrt(pow(maxs[ax], 2) + pow(mins[ax], 2)) * 1.e4 * eps) {
        nd->inds = inds;
        nd->leaf = np;
        return nd;
    }
    nd->axis = ax;
    double loc = 0.5 * (maxs[ax] + mins[ax]);
    nd->leaf = 0;
    int64_t k = 0, l = (int64_t)np - 1;
    while (k <= l) {
        if (data[inds[k] * NC + ax] * w[ax] < loc) ++k;
        else if (data[inds[l] * NC + ax] * w[ax] >= loc) --l;
        else {
            unsigned t = inds[l];
            inds[l] = inds[k];
            inds[k] = t;
            --l;
            ++k;
        }
    }
    if (k == 0) {
        loc = maxs[ax];
        for (unsigned i = 0; i < np; ++i)
            if (data[inds[i] * NC + ax] * w[ax] < loc) loc = data[inds[i] * NC + ax] * w[ax];
        loc -= 100. * eps * fabs(loc);
    } else if (l == (int64_t)np - 1) {
        loc = mins[ax];
        for (unsigned i = 0; i < np; ++i)
            if (data[inds[i] * NC + ax] * w[ax] > loc) loc = data[inds[i] * NC + ax] * w[ax];
        loc += 100. * eps * fabs(loc);
    }
    nd->loc = loc;
    double mids[5];
    memcpy(mids, maxs, sizeof mids);
    mids[ax] = loc;
    nd->left = kd_build(data, inds, (unsigned)k, mins, mids, w, leaf);
    memcpy(mids, mins, sizeof mids);
    mids[ax] = loc;
    nd->right = kd_build(data, inds + k, np - (unsigned)k, mids, maxs, w, leaf);
    return nd;
}

static void kd_free(Node *nd) {
    if (!nd) return;
    kd_free(nd->left);
    kd_free(nd->right);
    free(nd);
}

static void kd_query(const Tree *t, Node *nd, const double *pt, double *best, unsigned *ib, Node **found) {
    if (!nd) return;
    if (nd->leaf != 0) {
        for (unsigned i = 0; i < nd->leaf; ++i) {
            double d = 0.;
            for (int j = 0; j < 5; ++j) d += pow(t->data[nd->inds[i] * NC + j] * t->w[j] - pt[j], 2);
            if (d < *best) {
                *ib = nd->inds[i];
                *best = d;
                *found = nd;
            }
        }
        return;
    }
    Node *first = pt[nd->axis] < nd->loc ? nd->left : nd->right;
    Node *second = pt[nd->axis] < nd->loc ? nd->right : nd->left;
    kd_query(t, first, pt, best, ib, found);
    if (pow(pt[nd->axis] - nd->loc, 2) < *best) kd_query(t, second, pt, best, ib, found);
}

/* 0: not found, 1: removed, 2: the (single-point) leaf itself must go */
static unsigned kd_remove_node(Tree *t, Node *nd, unsigned ri) {
    if (!nd) return 0;
    if (nd->leaf > 1) {
        for (unsigned i = 0; i < nd->leaf; ++i) {
            if (nd->inds[i] == ri) {
                nd->inds[i] = nd->inds[nd->leaf - 1];
                nd->inds[nd->leaf - 1] = ri;
                nd->leaf -= 1;
                return 1;
            }
        }
        return 0;
    }
    if (nd->leaf == 1) return nd->inds[0] == ri ? 2 : 0;
    Node **child = (t->data[ri * NC + nd->axis] * t->w[nd->axis] < nd->loc) ? &nd->left : &nd->right;
    unsigned s = kd_remove_node(t, *child, ri);
    if (s == 2) {
        if (t->last == *child) t->last = nd;
        free(*child);
        *child = NULL;
        return 1;
    }
    return s;
}

static unsigned kd_remove(Tree *t, unsigned ri) {
    unsigned s = kd_remove_node(t, t->last, ri);
    if (s != 1) {
        s = kd_remove_node(t, t->root, ri);
        if (s == 1) {
            t->n -= 1;
            return 1;
        }
        return 0;
    }
    return 1;
}

/* kd-tree nearest neighbour of row q (5 coords, unweighted) among rows
 * [0, n) of data with weights w, leaf size `leaf`; for tests. */
void orc_kdtree_query_all(const double *data, unsigned n, const double *w, unsigned leaf, const double *queries,
                          unsigned nq, unsigned *ind_out, double *dist_out) {
    Tree t = {data, w, n, NULL, NULL, NULL};
    double mins[5], maxs[5];
    for (int j = 0; j < 5; ++j) {
        mins[j] = DBL_MAX;
        maxs[j] = -DBL_MAX;
    }
    for (unsigned i = 0; i < n; ++i)
        for (int j = 0; j < 5; ++j) {
            if (data[i * NC + j] < mins[j]) mins[j] = data[i * NC + j];
            if (data[i * NC + j] > maxs[j]) maxs[j] = data[i * NC + j];
        }
    for (int j = 0; j < 5; ++j) {
        mins[j] *= w[j];
        maxs[j] *= w[j];
    }
    t.inds = (unsigned *)malloc(sizeof(unsigned) * (n ? n : 1));
    for (unsigned i = 0; i < n; ++i) t.inds[i] = i;
    t.root = kd_build(data, t.inds, n, mins, maxs, w, leaf);
    t.last = t.root;
    for (unsigned q = 0; q < nq; ++q) {
        double pt[5];
        for (int j = 0; j < 5; ++j) pt[j] = queries[q * NC + j] * w[j];
        double best = DBL_MAX;
        unsigned ib = 0;
        kd_query(&t, t.root, pt, &best, &ib, &t.last);
        ind_out[q] = ib;
        dist_out[q] = best;
    }
    kd_free(t.root);
    free(t.inds);
}

/* ------------------------------ particleManagement.pyx:244-262 (_searchSorted) */
static int64_t search_sorted(const double *a, double v, int64_t n) {
    if (a[NC * (n - 1) + 5] <= v) return n;
    if (a[5] >= v) return 0;
    int64_t i0 = 0, i2 = n - 1, i1 = (int64_t)((i2 + i0) * 0.5);
    while (i1 != i0) {
        if (a[NC * i1 + 5] > v) i2 = i1;
        else i0 = i1;
        i1 = (int64_t)((i2 + i0) * 0.5);
    }
    return i1 + 1;
}

/* ----------------------------------- particleManagement.pyx:74-238
 * data: rows with room for `cap`; returns the new count (-1 if cap too small).
 * `inside` is the boundary predicate used by the (rarely effective) split. */
typedef int (*orc_inside_fn)(double x, double y, void *ctx);

int64_t orc_local_random(double *data, int64_t cap, int64_t n, int64_t target, double dx, double dy, double lx,
                         double ly, orc_inside_fn inside, void *ctx, double threshold_factor, double lambda_factor,
                         double dis_limit, int merge_scheme, unsigned leaf, double *add_scratch) {
    double mean = 0;
    for (int64_t i = 0; i < n; ++i) mean += data[NC * i + 5];
    mean /= n;
    double goal = mean * n / target;
    double maxT = threshold_factor * goal, minT = goal / threshold_factor;
    double dxi = 1. / dx, dyi = 1. / dy, ds = dx <= dy ? dx : dy, lxh = lx * 0.5, lyh = ly * 0.5;
    uint16_t *keep = (uint16_t *)malloc(sizeof(uint16_t) * (n ? n : 1));
    for (int64_t i = 0; i < n; ++i) keep[i] = 1;
    orc_quicksort_by_column(data, 0, n - 1, 5);
    unsigned to_merge = (unsigned)search_sorted(data, minT, n);
    unsigned to_split = (unsigned)(n - search_sorted(data, maxT, n));
    if (2 * to_merge + to_split >= n) {
        double f = 0.95 * n / (2 * to_merge + to_split);
        to_merge = (unsigned)(to_merge * f);
        to_split = (unsigned)(to_split * f);
    }
    int64_t nn = n + to_split - to_merge;
    if (nn > target) to_merge += (unsigned)(nn - target);
    else if (nn < target) to_split += (unsigned)(target - nn);
    if (2 * to_merge + to_split >= n) {
        double f = 0.95 * n / (2 * to_merge + to_split);
        to_merge = (unsigned)(to_merge * f);
        to_split = (unsigned)(to_split * f);
    }
    double vt = 0.;
    for (int64_t i = 0; i < n; ++i)
        vt += (pow(data[NC * i + 2], 2) + pow(data[NC * i + 3], 2) + pow(data[NC * i + 4], 2)) * pow(data[NC * i + 5], 2);
    vt = sqrt(vt) / (n * mean);
    if (vt < 1.e-12 * 299792458.0) vt = 1.e-12 * 299792458.0;
    /* split: halve the heaviest; the cell coordinate is truncated to an
     * unsigned integer as in the reference (:127-128), so the trial points
     * are in cell units */
    unsigned j = 0;
    for (int64_t i = n - to_split; i < n; ++i, ++j) {
        double *r = data + NC * i, *a = add_scratch + NC * j;
        r[5] *= 0.5;
        a[2] = r[2]; a[3] = r[3]; a[4] = r[4]; a[5] = r[5];
        unsigned cx = (unsigned)((r[0] + lxh) * dxi), cy = (unsigned)((r[1] + lyh) * dyi);
        double t, c0[2], c1[2];
        if (cx < 0.5) t = orc_rand() * fmin((double)cx, 0.5 - cx);
        else t = orc_rand() * fmin(cx - 0.5, 1. - cx);
        c0[0] = cx + t; c1[0] = cx - t;
        if (cy < 0.5) t = orc_rand() * fmin((double)cy, 0.5 - cy);
        else t = orc_rand() * fmin(cy - 0.5, 1. - cy);
        c0[1] = cy + t; c1[1] = cy - t;
        if (inside(c0[0], c0[1], ctx) == 0 || inside(c1[0], c1[1], ctx) == 0) {
            a[0] = r[0]; a[1] = r[1];
        } else {
            r[0] = c0[0]; r[1] = c0[1];
            a[0] = c1[0]; a[1] = c1[1];
        }
    }
    /* merge */
    double w[5] = {1., 1., 1., 1., 1.};
    double lam = lambda_factor * ds / vt;
    w[2] = w[3] = w[4] = lam;
    unsigned nt = (unsigned)(n - to_split);
    Tree t = {data, w, nt, NULL, NULL, NULL};
    double mins[5], maxs[5];
    for (int k = 0; k < 5; ++k) { mins[k] = DBL_MAX; maxs[k] = -DBL_MAX; }
    for (unsigned i = 0; i < nt; ++i)
        for (int k = 0; k < 5; ++k) {
            if (data[i * NC + k] < mins[k]) mins[k] = data[i * NC + k];
            if (data[i * NC + k] > maxs[k]) maxs[k] = data[i * NC + k];
        }
    for (int k = 0; k < 5; ++k) { mins[k] *= w[k]; maxs[k] *= w[k]; }
    t.inds = (unsigned *)malloc(sizeof(unsigned) * (nt ? nt : 1));
    for (unsigned i = 0; i < nt; ++i) t.inds[i] = i;
    t.root = nt ? kd_build(data, t.inds, nt, mins, maxs, w, leaf) : NULL;
    t.last = t.root;
    unsigned ii = 0, jj = 0;
    while (jj < to_merge && ii + 1 < nt) {
        if (keep[ii] == 0) { ++ii; continue; }
        if (kd_remove(&t, ii) != 1) { ++ii; continue; }
        double pt[5];
        for (int k = 0; k < 5; ++k) pt[k] = data[ii * NC + k] * w[k];
        double best = DBL_MAX;
        unsigned fi = 0;
        kd_query(&t, t.root, pt, &best, &fi, &t.last);
        if (best < dis_limit * ds) {
            double *a = data + NC * ii, *b = data + NC * fi;
            if (orc_rand() < a[5] / (b[5] + a[5])) {
                if (merge_scheme == 1) {
                    double f = a[5] / (b[5] + a[5]) + (pow(b[2], 2) + pow(b[3], 2) + pow(b[4], 2)) /
                               (pow(a[2], 2) + pow(a[3], 2) + pow(a[4], 2)) * b[5] / (b[5] + a[5]);
                    a[2] *= f; a[3] *= f; a[4] *= f;
                }
                a[5] += b[5];
                keep[fi] = 0;
            } else {
                if (merge_scheme == 1) {
                    double f = b[5] / (b[5] + a[5]) + (pow(a[2], 2) + pow(a[3], 2) + pow(a[4], 2)) /
                               (pow(b[2], 2) + pow(b[3], 2) + pow(b[4], 2)) * a[5] / (b[5] + a[5]);
                    b[2] *= f; b[3] *= f; b[4] *= f;
                }
                b[5] += a[5];
                keep[ii] = 0;
            }
            kd_remove(&t, fi);
            ++ii;
            ++jj;
        } else {
            ++ii;
        }
    }
    kd_free(t.root);
    free(t.inds);
    int64_t res = orc_add_and_remove(data, cap, n, add_scratch, to_split, keep);
    free(keep);
    return res;
}

/* inside predicates for the split trial points */
int orc_inside_rect_cb(double x, double y, void *ctx) {
    const double *l = (const double *)ctx;
    return (x < -l[0] * 0.5 || x > l[0] * 0.5 || y < -l[1] * 0.5 || y > l[1] * 0.5) ? 0 : 1;
}

int orc_inside_ellipse_cb(double x, double y, void *ctx) {
    const double *l = (const double *)ctx;
    return (pow(x, 2) * (4. / pow(l[0], 2)) + pow(y, 2) * (4. / pow(l[1], 2)) >= 1.) ? 0 : 1;
}

int64_t orc_local_random_ellipse(double *data, int64_t cap, int64_t n, int64_t target, double dx, double dy, double lx,
                                 double ly, int rect, double threshold_factor, double lambda_factor, double dis_limit,
                                 int merge_scheme, unsigned leaf, double *add_scratch) {
    double l[2] = {lx, ly};
    return orc_local_random(data, cap, n, target, dx, dy, lx, ly, rect ? orc_inside_rect_cb : orc_inside_ellipse_cb, l,
                            threshold_factor, lambda_factor, dis_limit, merge_scheme, leaf, add_scratch);
}
