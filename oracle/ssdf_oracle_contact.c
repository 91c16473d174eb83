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
