/*
 * ssdf_oracle_rebuild.c -- CPU oracle of the level-set path (marching tetrahedra, cubic refinement,
 * banded rebuild), restating serial/bvh/sdf_rebuild.cpp. TEST INFRASTRUCTURE ONLY.
 * Compiled like ssdf_oracle.c (-ffp-contract=off): its double arithmetic is the reference's.
 */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>

double oracle_point_triangle_dist_sq_d(double px, double py, double pz, double ax, double ay, double az, double bx,
                                       double by, double bz, double cx, double cy, double cz);

/* The six tetrahedra of a cell about its corner-0-to-7 diagonal (sdf_rebuild.cpp:15-17). */
static const int kOracleTets[6][4] = {{0, 1, 3, 7}, {0, 1, 5, 7}, {0, 2, 3, 7}, {0, 2, 6, 7}, {0, 4, 5, 7}, {0, 4, 6, 7}};

/* The crossing on edge (a, b), from the corner of lower grid index (sdf_rebuild.cpp:56-70). */
static void oracle_crossing(const ptrdiff_t g[8], const double v[8], const double p[8][3], int a, int b, double q[3]) {
    if (g[b] < g[a]) {
        const int s = a;
        a = b;
        b = s;
    }
    const double t = v[a] / (v[a] - v[b]);
    for (int d = 0; d < 3; d++) q[d] = p[a][d] + t * (p[b][d] - p[a][d]);
}

/* The 0, 1 or 2 triangles of one tetrahedron before the degenerate filter (sdf_rebuild.cpp:77-105). */
static int oracle_tet_triangles(const ptrdiff_t g[8], const double v[8], const double p[8][3], const int t[4],
                                double tri[2][3][3]) {
    int up[4], down[4], nu = 0, nd = 0;
    for (int a = 0; a < 4; a++) {
        if (v[t[a]] > 0)
            up[nu++] = t[a];
        else
            down[nd++] = t[a];
    }
    if (nu == 0 || nd == 0) return 0;
    if (nu == 1 || nd == 1) {
        const int lone = nu == 1 ? up[0] : down[0];
        const int *others = nu == 1 ? down : up;
        for (int a = 0; a < 3; a++) oracle_crossing(g, v, p, lone, others[a], tri[0][a]);
        return 1;
    }
    double q[4][3];
    oracle_crossing(g, v, p, up[0], down[0], q[0]);
    oracle_crossing(g, v, p, up[0], down[1], q[1]);
    oracle_crossing(g, v, p, up[1], down[1], q[2]);
    oracle_crossing(g, v, p, up[1], down[0], q[3]);
    const int quad[2][3] = {{0, 1, 2}, {0, 2, 3}};
    for (int s = 0; s < 2; s++)
        for (int a = 0; a < 3; a++)
            for (int d = 0; d < 3; d++) tri[s][a][d] = q[quad[s][a]][d];
    return 2;
}

#define REAL double
#define SUF _d
#include "ssdf_oracle_rebuild_impl.h"
#undef REAL
#undef SUF

#define REAL float
#define SUF _f
#include "ssdf_oracle_rebuild_impl.h"
#undef REAL
#undef SUF
