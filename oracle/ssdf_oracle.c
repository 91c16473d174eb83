/*
 * ssdf_oracle.c -- CPU oracle for ssdf's closest-point distance path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the CUDA library (ssdf_b200/) is compared
 * against. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it; the
 * product never links, calls or falls back to it.
 *
 * What it restates (paths relative to the zulianp/ssdf source tree):
 *   - point_triangle_dist_sq / point_triangle_closest_point (serial/ssdf.hpp:49-121, 143-239),
 *     point_aabb_distance_squared / point_aabb_signed_distance (serial/edf/edf.hpp:55-69,
 *     193-221), the edf / edf_celllist value (serial/ssdf.hpp:447-963) and the node-grid
 *     convention (serial/bvh/bvh.cpp:1665-1667, 1744): ssdf_oracle_impl.h, float and double;
 *   - the angle-weighted pseudo-normals and the barycentric sign rule of sample_sdf_bvh
 *     (serial/bvh/bvh.cpp:1669-1721, 1751-1792), here evaluated in double on the closest
 *     point of the double argmin triangle;
 *   - closest_point_bvh's update-if-better outputs (serial/bvh/bvh.cpp:178-194) and
 *     sample_sqedf_bvh's min-with-incoming squared distance (serial/bvh/bvh.cpp:1615-1636).
 *
 * Tie rule (this build's, the reference's edf returns no index): the closest triangle is the
 * lowest index among those whose squared distance equals the minimum.
 *
 * Pinned by tests/test_oracle.py against the reference compiled from its own sources
 * (oracle/_ref, built by oracle/Makefile) and against the golden vectors in tests/golden/.
 * Build: oracle/Makefile (gcc -std=c11 -O2 -ffp-contract=off -fopenmp).
 */

#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define REAL double
#define SUF _d
#define OR_ABS fabs
#define OR_SQRT sqrt
#include "ssdf_oracle_impl.h"
#undef REAL
#undef SUF
#undef OR_ABS
#undef OR_SQRT

#define REAL float
#define SUF _f
#define OR_ABS fabsf
#define OR_SQRT sqrtf
#include "ssdf_oracle_impl.h"
#undef REAL
#undef SUF
#undef OR_ABS
#undef OR_SQRT

/* ------------------------------------------------------------------------------------------ */
/* Pseudo-normals (serial/bvh/bvh.cpp:1669-1721)                                               */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
    uint64_t key;
    int64_t occ; /* 3 * face + local edge, in the order the reference visits them */
} edge_occ;

static int edge_occ_cmp(const void *a, const void *b) {
    const edge_occ *x = (const edge_occ *)a, *y = (const edge_occ *)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return (x->occ > y->occ) - (x->occ < y->occ);
}

/*
 * face_n[3 * nsel]: unit normal of (s1 - s0) x (s2 - s0) (left unnormalised when its length is 0);
 * vertex_n[3 * nsp]: sum over incident faces, in face order, of interior angle * face normal;
 * edge_n[9 * nsel]: for local edge e of face t (vertex e to vertex (e + 1) % 3) the sum of the
 * unit normals of the two faces sharing it, the face's own normal on a boundary edge.
 *
 * The reference keeps, per undirected edge key min * nsp + max, the first occurrence in an
 * unordered_map; every later occurrence k writes first + k into both its own slot and the
 * first's. Sorting the occurrences by (key, visit order) and replaying that gives the same
 * values for manifold and non-manifold edges alike.
 */
int oracle_pseudonormals_d(const ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                           const ptrdiff_t nspoints, const double *sx, const double *sy, const double *sz,
                           double *face_n, double *edge_n, double *vertex_n) {
    const int *s[3] = {s0, s1, s2};
    memset(vertex_n, 0, sizeof(double) * 3 * (size_t)nspoints);
    for (ptrdiff_t t = 0; t < nselements; t++) {
        double p[3][3];
        for (int v = 0; v < 3; v++) {
            p[v][0] = sx[s[v][t]];
            p[v][1] = sy[s[v][t]];
            p[v][2] = sz[s[v][t]];
        }
        const double u[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
        const double w[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
        double n[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
        const double len = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        if (len > 0) {
            for (int d = 0; d < 3; d++) n[d] /= len;
        }
        for (int d = 0; d < 3; d++) face_n[3 * t + d] = n[d];
        for (int v = 0; v < 3; v++) {
            const double *a = p[v], *b = p[(v + 1) % 3], *c = p[(v + 2) % 3];
            const double e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
            const double e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
            const double l1 = sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
            const double l2 = sqrt(e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2]);
            const double cosine =
                (l1 > 0 && l2 > 0) ? (e1[0] * e2[0] + e1[1] * e2[1] + e1[2] * e2[2]) / (l1 * l2) : 1.0;
            /* std::max(-1.0, std::min(1.0, cosine)) */
            const double mn = (cosine < 1.0) ? cosine : 1.0;
            const double cl = (-1.0 < mn) ? mn : -1.0;
            const double angle = acos(cl);
            for (int d = 0; d < 3; d++) vertex_n[3 * (ptrdiff_t)s[v][t] + d] += angle * n[d];
        }
        for (int e = 0; e < 3; e++)
            for (int d = 0; d < 3; d++) edge_n[9 * t + 3 * e + d] = n[d];
    }

    edge_occ *occ = (edge_occ *)malloc(sizeof(edge_occ) * 3 * (size_t)(nselements > 0 ? nselements : 1));
    if (!occ) return 1;
    for (ptrdiff_t t = 0; t < nselements; t++)
        for (int e = 0; e < 3; e++) {
            const uint64_t a = (uint64_t)s[e][t], b = (uint64_t)s[(e + 1) % 3][t];
            const uint64_t lo = a < b ? a : b, hi = a < b ? b : a;
            occ[3 * t + e].key = lo * (uint64_t)nspoints + hi;
            occ[3 * t + e].occ = 3 * t + e;
        }
    qsort(occ, 3 * (size_t)nselements, sizeof(edge_occ), edge_occ_cmp);
    for (ptrdiff_t g = 0; g < 3 * nselements;) {
        ptrdiff_t h = g + 1;
        while (h < 3 * nselements && occ[h].key == occ[g].key) h++;
        const int64_t first = occ[g].occ;
        for (ptrdiff_t k = g + 1; k < h; k++) {
            const int64_t o = occ[k].occ;
            for (int d = 0; d < 3; d++) {
                const double sum = face_n[3 * (first / 3) + d] + face_n[3 * (o / 3) + d];
                edge_n[9 * (o / 3) + 3 * (o % 3) + d] = sum;
                edge_n[9 * (first / 3) + 3 * (first % 3) + d] = sum;
            }
        }
        g = h;
    }
    free(occ);
    return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* Sign at one query (serial/bvh/bvh.cpp:1751-1792)                                           */
/* ------------------------------------------------------------------------------------------ */

/* Returns the signed distance of q given its closest triangle t and squared distance d2. */
static double signed_from_closest(const double q[3], const ptrdiff_t t, const double d2, const int *const s[3],
                                  const double *sx, const double *sy, const double *sz, const double *face_n,
                                  const double *edge_n, const double *vertex_n, const double tol,
                                  double cpt[3]) {
    double a[3][3];
    for (int v = 0; v < 3; v++) {
        a[v][0] = sx[s[v][t]];
        a[v][1] = sy[s[v][t]];
        a[v][2] = sz[s[v][t]];
    }
    double c[3];
    oracle_point_triangle_closest_point_d(q[0], q[1], q[2], a[0][0], a[0][1], a[0][2], a[1][0], a[1][1], a[1][2],
                                          a[2][0], a[2][1], a[2][2], &c[0], &c[1], &c[2]);
    if (cpt) cpt[0] = c[0], cpt[1] = c[1], cpt[2] = c[2];
    const double e1[3] = {a[1][0] - a[0][0], a[1][1] - a[0][1], a[1][2] - a[0][2]};
    const double e2[3] = {a[2][0] - a[0][0], a[2][1] - a[0][1], a[2][2] - a[0][2]};
    const double r[3] = {c[0] - a[0][0], c[1] - a[0][1], c[2] - a[0][2]};
    const double d11 = e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2];
    const double d12 = e1[0] * e2[0] + e1[1] * e2[1] + e1[2] * e2[2];
    const double d22 = e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2];
    const double r1 = r[0] * e1[0] + r[1] * e1[1] + r[2] * e1[2];
    const double r2 = r[0] * e2[0] + r[1] * e2[1] + r[2] * e2[2];
    const double det = d11 * d22 - d12 * d12;
    const double l1 = det > 0 ? (d22 * r1 - d12 * r2) / det : 0;
    const double l2 = det > 0 ? (d11 * r2 - d12 * r1) / det : 0;
    const double l[3] = {1 - l1 - l2, l1, l2};
    int small = 0, last_small = -1, last_large = -1;
    for (int v = 0; v < 3; v++) {
        if (l[v] < tol) {
            small++;
            last_small = v;
        } else {
            last_large = v;
        }
    }
    const double *n;
    if (small == 0) {
        n = &face_n[3 * t];
    } else if (small == 1) {
        n = &edge_n[9 * t + 3 * ((last_small + 1) % 3)];
    } else {
        n = &vertex_n[3 * (ptrdiff_t)s[last_large][t]];
    }
    const double dot = (q[0] - c[0]) * n[0] + (q[1] - c[1]) * n[1] + (q[2] - c[2]) * n[2];
    const double dist = sqrt(d2);
    return dot < 0 ? -dist : dist;
}

/*
 * Signed distance at arbitrary double points (the grid entry point feeds it grid nodes):
 * brute-force double argmin with the lowest-index tie rule, then sample_sdf_bvh's sign rule
 * with tol = 1e-4 (serial/bvh/bvh.cpp:1738). out[p] = +-sqrt(d2); outtri may be NULL.
 * Normals come from oracle_pseudonormals_d.
 */
int oracle_sdf_points_d(const ptrdiff_t npoints, const double *x, const double *y, const double *z,
                        const ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                        const ptrdiff_t nspoints, const double *sx, const double *sy, const double *sz,
                        const double *face_n, const double *edge_n, const double *vertex_n, double *out,
                        int *outtri) {
    (void)nspoints;
    if (nselements == 0) return 1;
    const int *const s[3] = {s0, s1, s2};
#pragma omp parallel for schedule(dynamic, 64)
    for (ptrdiff_t p = 0; p < npoints; p++) {
        const double q[3] = {x[p], y[p], z[p]};
        double best = INFINITY;
        ptrdiff_t bt = 0;
        for (ptrdiff_t t = 0; t < nselements; t++) {
            const int i0 = s0[t], i1 = s1[t], i2 = s2[t];
            const double d2 = oracle_point_triangle_dist_sq_d(q[0], q[1], q[2], sx[i0], sy[i0], sz[i0], sx[i1],
                                                              sy[i1], sz[i1], sx[i2], sy[i2], sz[i2]);
            if (d2 < best) {
                best = d2;
                bt = t;
            }
        }
        out[p] = signed_from_closest(q, bt, best, s, sx, sy, sz, face_n, edge_n, vertex_n, 1e-4, NULL);
        if (outtri) outtri[p] = (int)bt;
    }
    return 0;
}

/*
 * closest_point_bvh (serial/bvh/bvh.cpp:125-219): distance, closest point and triangle, all
 * written only where the distance is below the incoming outd (outd[p] > dist). The closest
 * point is the double closest point on the argmin triangle.
 */
int oracle_closest_point_d(const ptrdiff_t npoints, const double *x, const double *y, const double *z,
                           const ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                           const ptrdiff_t nspoints, const double *sx, const double *sy, const double *sz,
                           double *outd, double *outx, double *outy, double *outz, int *outtri) {
    (void)nspoints;
    if (nselements == 0) return 0;
#pragma omp parallel for schedule(dynamic, 64)
    for (ptrdiff_t p = 0; p < npoints; p++) {
        double best = INFINITY;
        ptrdiff_t bt = 0;
        for (ptrdiff_t t = 0; t < nselements; t++) {
            const int i0 = s0[t], i1 = s1[t], i2 = s2[t];
            const double d2 = oracle_point_triangle_dist_sq_d(x[p], y[p], z[p], sx[i0], sy[i0], sz[i0], sx[i1],
                                                              sy[i1], sz[i1], sx[i2], sy[i2], sz[i2]);
            if (d2 < best) {
                best = d2;
                bt = t;
            }
        }
        const double dist = sqrt(best);
        if (outd[p] > dist) {
            const int i0 = s0[bt], i1 = s1[bt], i2 = s2[bt];
            outd[p] = dist;
            oracle_point_triangle_closest_point_d(x[p], y[p], z[p], sx[i0], sy[i0], sz[i0], sx[i1], sy[i1], sz[i1],
                                                  sx[i2], sy[i2], sz[i2], &outx[p], &outy[p], &outz[p]);
            outtri[p] = (int)bt;
        }
    }
    return 0;
}

/*
 * sample_sqedf_bvh's update (serial/bvh/bvh.cpp:1615-1636): out[p] = MIN(out[p], d2) on the
 * squared distance, at arbitrary double points.
 */
int oracle_sqedf_points_d(const ptrdiff_t npoints, const double *x, const double *y, const double *z,
                          const ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                          const ptrdiff_t nspoints, const double *sx, const double *sy, const double *sz,
                          double *out) {
    (void)nspoints;
#pragma omp parallel for schedule(dynamic, 64)
    for (ptrdiff_t p = 0; p < npoints; p++) {
        double best = INFINITY;
        for (ptrdiff_t t = 0; t < nselements; t++) {
            const int i0 = s0[t], i1 = s1[t], i2 = s2[t];
            const double d2 = oracle_point_triangle_dist_sq_d(x[p], y[p], z[p], sx[i0], sy[i0], sz[i0], sx[i1],
                                                              sy[i1], sz[i1], sx[i2], sy[i2], sz[i2]);
            if (d2 < best) best = d2;
        }
        out[p] = (out[p] < best) ? out[p] : best;
    }
    return 0;
}
