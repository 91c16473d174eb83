/*
 * ssdf_oracle_contact.c -- CPU oracle for the closest-primitive-within-a-radius queries
 * (ssdf::closest_within_radius_bvh, _local_bvh, _quads_bvh, _quads_local_bvh;
 * serial/bvh/bvh.cpp:367-832).
 *
 * TEST INFRASTRUCTURE ONLY: the checker the CUDA library is compared against. The product never
 * links, calls or falls back to it.
 *
 * Restated here (paths relative to the zulianp/ssdf source tree):
 *   - point_segment_parameter (serial/edf/edf.hpp:222-249), point_triangle_barycentric
 *     (serial/edf/edf.hpp:251-386) and point_to_quad_closest_point (serial/edf/edf.hpp:388-489),
 *     in float and double; pinned against the reference's own templates (oracle/_ref) by
 *     tests/test_oracle.py;
 *   - triangle_local_coordinates_st (serial/bvh/bvh.cpp:60-83), in float and double;
 *   - the per-point loop of the four queries: the primitive's closest point in float (the
 *     reference computes it in cuBQL's vec3f), kept when its squared distance is at most the
 *     running value, which starts at radius_squared[pid * stride] converted to float.
 *
 * What cannot be pinned: cuBQL (an absent, un-vendored dependency) supplies the reference's
 * triangle closest point (triangles::computeClosestPoint) and the traversal order. Here the
 * triangle closest point is the reference's own point_triangle_closest_point<float>
 * (serial/ssdf.hpp:143-239), the same routine as the float distance path, and among primitives
 * at the same squared distance the lowest index wins (the reference's `<=` keeps the last one
 * its traversal visits, an order this build cannot reproduce). Primitives are evaluated by brute
 * force, every one of them.
 *
 * Build: oracle/Makefile (gcc -std=c11 -O2 -ffp-contract=off -fopenmp).
 */

#include <float.h>
#include <math.h>
#include <stddef.h>

/* ---- primitives, in REAL ------------------------------------------------------------------- */

#define REAL double
#define SUF _d
#define OR_ABS fabs
#define OR_EPS DBL_EPSILON
#include "ssdf_oracle_contact_prim.h"
#undef REAL
#undef SUF
#undef OR_ABS
#undef OR_EPS

#define REAL float
#define SUF _f
#define OR_ABS fabsf
#define OR_EPS FLT_EPSILON
#include "ssdf_oracle_contact_prim.h"
#undef REAL
#undef SUF
#undef OR_ABS
#undef OR_EPS

/* The float closest point of serial/ssdf.hpp:143-239 (restated in ssdf_oracle_impl.h). */
void oracle_point_triangle_closest_point_f(float px, float py, float pz, float ax, float ay, float az, float bx,
                                           float by, float bz, float cx, float cy, float cz, float *outx,
                                           float *outy, float *outz);

/* ---- the queries, over (G, T) = (float, float), (float, double), (double, double) ----------- */

#define GREAL float
#define TREAL float
#define SUF2 _ff
#define OQ_LOCAL_ST oracle_triangle_local_st_f
#include "ssdf_oracle_contact_query.h"
#undef GREAL
#undef TREAL
#undef SUF2
#undef OQ_LOCAL_ST

#define GREAL float
#define TREAL double
#define SUF2 _fd
#define OQ_LOCAL_ST oracle_triangle_local_st_d
#include "ssdf_oracle_contact_query.h"
#undef GREAL
#undef TREAL
#undef SUF2
#undef OQ_LOCAL_ST

#define GREAL double
#define TREAL double
#define SUF2 _dd
#define OQ_LOCAL_ST oracle_triangle_local_st_d
#include "ssdf_oracle_contact_query.h"
#undef GREAL
#undef TREAL
#undef SUF2
#undef OQ_LOCAL_ST

/* ---- candidate contact pairs (serial/bvh/bvh.cpp:834-1196) --------------------------------- */

/* Corner k of element e as float (the reference's vec3f). */
static void pc_corner(const int *const s[4], const ptrdiff_t e, const int k, const void *sx, const void *sy,
                      const void *sz, const int f64, float p[3]) {
    const int i = s[k][e];
    if (f64) {
        p[0] = (float)((const double *)sx)[i], p[1] = (float)((const double *)sy)[i], p[2] = (float)((const double *)sz)[i];
    } else {
        p[0] = ((const float *)sx)[i], p[1] = ((const float *)sy)[i], p[2] = ((const float *)sz)[i];
    }
}

static void pc_cross(const float a[3], const float b[3], float out[3]) {
    out[0] = a[1] * b[2] - a[2] * b[1];
    out[1] = a[2] * b[0] - a[0] * b[2];
    out[2] = a[0] * b[1] - a[1] * b[0];
}

/* v / |v| as v * (1 / sqrt(v . v)), float */
static void pc_normalize(float v[3]) {
    const float inv = 1.0f / sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    v[0] = v[0] * inv, v[1] = v[1] * inv, v[2] = v[2] * inv;
}

/* Tight box (lo[3], hi[3]) of element e, and with extrude != 0 the box grown by every corner moved
 * `ext` along its normal and `inner` against it. Triangles: one normal, cross(b - a, c - a)
 * normalised (cuBQL's Triangle::normal(), taken as the unit normal). Quads: per corner,
 * serial/bvh/bvh.cpp:1019-1030. min / max ignore NaN (fminf / fmaxf). */
static void pc_box(const int *const s[4], const int nk, const ptrdiff_t e, const void *sx, const void *sy,
                   const void *sz, const int f64, const int extrude, const float ext, const float inner, float lo[3],
                   float hi[3]) {
    float c[4][3], n[4][3];
    for (int k = 0; k < nk; k++) pc_corner(s, e, k, sx, sy, sz, f64, c[k]);
    for (int d = 0; d < 3; d++) {
        lo[d] = c[0][d], hi[d] = c[0][d];
        for (int k = 1; k < nk; k++) lo[d] = fminf(lo[d], c[k][d]), hi[d] = fmaxf(hi[d], c[k][d]);
    }
    if (!extrude) return;
    if (nk == 3) {
        float u[3], v[3];
        for (int d = 0; d < 3; d++) u[d] = c[1][d] - c[0][d], v[d] = c[2][d] - c[0][d];
        pc_cross(u, v, n[0]);
        pc_normalize(n[0]);
        for (int k = 1; k < 3; k++)
            for (int d = 0; d < 3; d++) n[k][d] = n[0][d];
    } else {
        float ab[3], dc[3], ad[3], bc[3];
        for (int d = 0; d < 3; d++) {
            ab[d] = c[1][d] - c[0][d], dc[d] = c[2][d] - c[3][d];
            ad[d] = c[3][d] - c[0][d], bc[d] = c[2][d] - c[1][d];
        }
        pc_cross(ab, ad, n[0]);
        pc_cross(ab, bc, n[1]);
        pc_cross(dc, bc, n[2]);
        pc_cross(dc, ad, n[3]);
        for (int k = 0; k < 4; k++) pc_normalize(n[k]);
    }
    for (int k = 0; k < nk; k++)
        for (int d = 0; d < 3; d++) {
            const float out = c[k][d] + n[k][d] * ext, in = c[k][d] - n[k][d] * inner;
            lo[d] = fminf(lo[d], out), hi[d] = fmaxf(hi[d], out);
            lo[d] = fminf(lo[d], in), hi[d] = fmaxf(hi[d], in);
        }
}

/*
 * potential_contact_triangles_bvh (s3 == NULL) / potential_contact_quads_bvh, by brute force: for
 * each element pid, every other element whose tight box meets (closed intervals) pid's box grown by
 * `ext` along its normals and `inner` against them, and which shares no corner index with pid.
 * ext = (float)extrusion and inner = (float)(T(0.1) * extrusion) are passed in already converted.
 * pc_ptr[ne + 1] gets the CSR offsets; idx (capacity cap, may be NULL) the candidates in ascending
 * order per element (the reference's order within a row is its threads' order). Returns the total.
 */
ptrdiff_t oracle_potential_contact(const ptrdiff_t ne, const int *s0, const int *s1, const int *s2, const int *s3,
                                   const void *sx, const void *sy, const void *sz, const int f64, const float ext,
                                   const float inner, ptrdiff_t *pc_ptr, int *idx, const ptrdiff_t cap) {
    const int *s[4] = {s0, s1, s2, s3};
    const int nk = s3 ? 4 : 3;
    ptrdiff_t total = 0;
    pc_ptr[0] = 0;
    for (ptrdiff_t p = 0; p < ne; p++) {
        float elo[3], ehi[3];
        pc_box(s, nk, p, sx, sy, sz, f64, 1, ext, inner, elo, ehi);
        for (ptrdiff_t t = 0; t < ne; t++) {
            int shared = 0;
            for (int i = 0; i < nk && !shared; i++)
                for (int j = 0; j < nk; j++)
                    if (s[i][p] == s[j][t]) shared = 1;
            if (shared) continue;
            float lo[3], hi[3];
            pc_box(s, nk, t, sx, sy, sz, f64, 0, 0.f, 0.f, lo, hi);
            int meet = 1;
            for (int d = 0; d < 3; d++) meet &= elo[d] <= hi[d] && lo[d] <= ehi[d];
            if (!meet) continue;
            if (idx && total < cap) idx[total] = (int)t;
            total++;
        }
        pc_ptr[p + 1] = total;
    }
    return total;
}
