/*
 * ssdf_b200.h -- C ABI of the B200 (sm_100a) closest-point distance-field library.
 *
 * Everything here is plain C: pointers, sizes and integer status codes. Paths in the comments are
 * zulianp/ssdf source files, the interface each entry point stands in for.
 *
 * Conventions shared by every entry point:
 *   - SoA layout exactly as ssdf's: query points x, y, z [npoints]; triangles s0, s1, s2
 *     [nselements] (0-based int32 vertex ids); vertices sx, sy, sz [nspoints].
 *   - The drop-in entry points take HOST pointers and are blocking, like the reference
 *     (serial/ssdf.hpp:447-460, serial/bvh/bvh.hpp:19-227). The handle API (ssdf_mesh_*,
 *     ssdf_query_*) takes DEVICE pointers and a cudaStream_t (as void*), and is asynchronous.
 *   - `out` of the edf family is in/out: on entry the current best distance (squared for the
 *     sqedf family), on exit min(incoming, surface distance) (serial/ssdf.hpp:439-440).
 *   - Closest triangle: the lowest triangle index among those at the minimum squared distance.
 *   - Sign: positive on the side the right-handed (s0, s1, s2) normals point to, negative inside a
 *     closed outward-oriented surface, + where the pseudo-normal dot product is 0
 *     (serial/bvh/bvh.hpp:203-208, serial/bvh/bvh.cpp:1790-1792).
 *   - An empty mesh leaves the outputs untouched and returns SSDF_OK (serial/ssdf.hpp:462).
 *   - Every entry point returns a status code and never aborts the process; the CUDA path is the
 *     only path (no CPU fallback): without a usable GPU they return SSDF_ERR_CUDA.
 */
#ifndef SSDF_B200_H
#define SSDF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------------------------- */
#define SSDF_OK 0
#define SSDF_ERR_INVALID_ARGUMENT 1 /* null pointer, negative size, out-of-range index        */
#define SSDF_ERR_OUT_OF_MEMORY 2    /* a device or pinned host allocation failed              */
#define SSDF_ERR_CUDA 3             /* a CUDA runtime call or kernel launch failed            */
#define SSDF_ERR_NOT_SUPPORTED 4    /* a size or option beyond what this build handles        */
#define SSDF_ERR_INTERNAL 5         /* a device-side check fired (bounded wait, stack depth)  */
#define SSDF_ERR_BUSY 6             /* the server's queue is over its admission limit: retry  */

/* Human-readable name of a status code. */
const char *ssdf_status_string(int status);
/* The calling thread's last error message ("" when none). */
const char *ssdf_last_error(void);
/* Library version string. */
const char *ssdf_b200_version(void);

/* ---- drop-in: the reference's exported C ABI ------------------------------------------------ */

/* ssdf_edf_f / ssdf_edf_d (serial/ssdf.cpp:36-66): unsigned distance, in/out `out`, dispatched as
 * ssdf::edf_select (serial/ssdf.hpp:965-1016) by the same environment variables:
 * SSDF_USE_BVH (default 1: the device BVH), SSDF_CELL_VALIDATE (run edf and edf_celllist and
 * report their relative difference on stderr), SSDF_USE_CELL_LIST (default 1) else edf. */
int ssdf_edf_f(ptrdiff_t npoints, const float *x, const float *y, const float *z, ptrdiff_t nselements,
               const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints, const float *sx, const float *sy,
               const float *sz, float *out);
int ssdf_edf_d(ptrdiff_t npoints, const double *x, const double *y, const double *z, ptrdiff_t nselements,
               const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints, const double *sx, const double *sy,
               const double *sz, double *out);

/* ---- drop-in: one symbol per template instantiation of the C++ API ---------------------------
 * include/ssdf.hpp maps ssdf::<name><G, T, int> onto these. Suffix: G then T, f = float,
 * d = double (edf and edf_celllist are instantiated for G == T only, serial/ssdf.cpp:4-30). */

/* ssdf::edf (serial/ssdf.hpp:447-619): brute force on the GPU, triangle tiles staged in shared
 * memory. Result bitwise equal to the reference's in T's precision. */
int ssdf_b200_edf_ff(ptrdiff_t npoints, const float *x, const float *y, const float *z, ptrdiff_t nselements,
                     const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints, const float *sx,
                     const float *sy, const float *sz, float *out);
int ssdf_b200_edf_dd(ptrdiff_t npoints, const double *x, const double *y, const double *z, ptrdiff_t nselements,
                     const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints, const double *sx,
                     const double *sy, const double *sz, double *out);

/* ssdf::edf_celllist (serial/ssdf.hpp:642-963): 2-D cell list over the two widest axes on the
 * GPU. Result bitwise equal to the reference's in T's precision. */
int ssdf_b200_edf_celllist_ff(ptrdiff_t npoints, const float *x, const float *y, const float *z,
                              ptrdiff_t nselements, const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints,
                              const float *sx, const float *sy, const float *sz, float *out);
int ssdf_b200_edf_celllist_dd(ptrdiff_t npoints, const double *x, const double *y, const double *z,
                              ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                              ptrdiff_t nspoints, const double *sx, const double *sy, const double *sz,
                              double *out);

/* ssdf::edf_bvh (serial/bvh/bvh.hpp:19-32, bvh.cpp:298-316; instantiations bvh.cpp:1216-1256):
 * device BVH. <float,float> computes in the reference's float arithmetic; <float,double> and
 * <double,double> return the double result (FP32 traversal with FP64 fix-up by default,
 * SSDF_B200_PRECISION=f64 for the plain double kernel). */
int ssdf_b200_edf_bvh_ff(ptrdiff_t npoints, const float *x, const float *y, const float *z, ptrdiff_t nselements,
                         const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints, const float *sx,
                         const float *sy, const float *sz, float *out);
int ssdf_b200_edf_bvh_fd(ptrdiff_t npoints, const float *x, const float *y, const float *z, ptrdiff_t nselements,
                         const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints, const float *sx,
                         const float *sy, const float *sz, double *out);
int ssdf_b200_edf_bvh_dd(ptrdiff_t npoints, const double *x, const double *y, const double *z,
                         ptrdiff_t nselements, const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints,
                         const double *sx, const double *sy, const double *sz, double *out);

/* ssdf::closest_point_bvh (serial/bvh/bvh.hpp:34-51, bvh.cpp:125-219): distance, closest point
 * and triangle, all four written only where the distance is below the incoming outd. */
int ssdf_b200_closest_point_bvh_ff(ptrdiff_t npoints, const float *x, const float *y, const float *z,
                                   ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                   ptrdiff_t nspoints, const float *sx, const float *sy, const float *sz, float *outd,
                                   float *outx, float *outy, float *outz, int *outtri);
/* closest_point_bvh<float, double, int> (serial/bvh/bvh.cpp:1162-1179): float points and mesh, double
 * distance (the FP64 distance of the float-valued inputs), closest point rounded to float. */
int ssdf_b200_closest_point_bvh_fd(ptrdiff_t npoints, const float *x, const float *y, const float *z,
                                   ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                   ptrdiff_t nspoints, const float *sx, const float *sy, const float *sz, double *outd,
                                   float *outx, float *outy, float *outz, int *outtri);
int ssdf_b200_closest_point_bvh_dd(ptrdiff_t npoints, const double *x, const double *y, const double *z,
                                   ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                   ptrdiff_t nspoints, const double *sx, const double *sy, const double *sz,
                                   double *outd, double *outx, double *outy, double *outz, int *outtri);

/* ssdf::sample_sqedf_bvh (serial/bvh/bvh.hpp:183-201, bvh.cpp:1574-1639): squared distance on
 * the node grid nx*ny*nz over [min, max] (x fastest), out = min(out, d^2). */
int ssdf_b200_sample_sqedf_bvh_ff(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                  ptrdiff_t nspoints, const float *sx, const float *sy, const float *sz, ptrdiff_t nx,
                                  ptrdiff_t ny, ptrdiff_t nz, float xmin, float ymin, float zmin, float xmax,
                                  float ymax, float zmax, float *out);
int ssdf_b200_sample_sqedf_bvh_dd(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                  ptrdiff_t nspoints, const double *sx, const double *sy, const double *sz,
                                  ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz, double xmin, double ymin, double zmin,
                                  double xmax, double ymax, double zmax, double *out);

/* ssdf::sample_sdf_bvh (serial/bvh/bvh.hpp:203-227, bvh.cpp:1641-1798): signed distance on the
 * node grid; sign from the angle-weighted pseudo-normal at the closest point (barycentric
 * tolerance 1e-4, bvh.cpp:1738). */
int ssdf_b200_sample_sdf_bvh_ff(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                ptrdiff_t nspoints, const float *sx, const float *sy, const float *sz, ptrdiff_t nx,
                                ptrdiff_t ny, ptrdiff_t nz, float xmin, float ymin, float zmin, float xmax,
                                float ymax, float zmax, float *out);
int ssdf_b200_sample_sdf_bvh_dd(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                ptrdiff_t nspoints, const double *sx, const double *sy, const double *sz,
                                ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz, double xmin, double ymin, double zmin,
                                double xmax, double ymax, double zmax, double *out);

/* ---- drop-in: inside flags --------------------------------------------------------------------
 * ssdf::points_inside_bvh<G, int> (serial/bvh/bvh.hpp:54-66, bvh.cpp:318-365) and
 * ssdf::sample_inside_bvh<G, int> (bvh.hpp:230-247, bvh.cpp:1800-1866): out = 1 inside the closed
 * surface, 0 outside, one byte per point / grid node. Inside is where sample_sdf_bvh's signed
 * distance (pseudo-normal rule, in double) is negative; the reference asks cuBQL's
 * pointIsInsideSurface, which cannot be built here. */
int ssdf_b200_points_inside_bvh_f(ptrdiff_t npoints, const float *x, const float *y, const float *z,
                                  ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                  ptrdiff_t nspoints, const float *sx, const float *sy, const float *sz, uint8_t *out);
int ssdf_b200_points_inside_bvh_d(ptrdiff_t npoints, const double *x, const double *y, const double *z,
                                  ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                  ptrdiff_t nspoints, const double *sx, const double *sy, const double *sz,
                                  uint8_t *out);
int ssdf_b200_sample_inside_bvh_f(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                  ptrdiff_t nspoints, const float *sx, const float *sy, const float *sz, ptrdiff_t nx,
                                  ptrdiff_t ny, ptrdiff_t nz, float xmin, float ymin, float zmin, float xmax,
                                  float ymax, float zmax, uint8_t *out);
int ssdf_b200_sample_inside_bvh_d(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                  ptrdiff_t nspoints, const double *sx, const double *sy, const double *sz,
                                  ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz, double xmin, double ymin, double zmin,
                                  double xmax, double ymax, double zmax, uint8_t *out);

/* ---- drop-in: closest primitive within a radius ----------------------------------------------
 * ssdf::closest_within_radius_bvh, _local_bvh, _quads_bvh, _quads_local_bvh<G, T, int>
 * (serial/bvh/bvh.hpp:68-154, bvh.cpp:367-832), for (G, T) = (float, float) _ff, (float, double) _fd
 * and (double, double) _dd. Per point pid: the primitive (triangle s0/s1/s2, or quad s0/s1/s2/s3)
 * whose float closest point is nearest, among those at squared distance at most
 * radius_squared[pid * radius_stride] (stride 0: one radius for all), skipping primitives that have
 * pid as a corner when skip_self != 0 (node-to-surface self contact). Outputs, written for every
 * point: outtri (-1 when none), out_sqr_dist (the float squared distance, or the float radius
 * squared when none), and the closest point (closest_x/y/z; zeros when none) or its local
 * coordinates (closest_s/t: triangle_local_coordinates_st in T for triangles, the clamped bilinear
 * parameters for quads; zeros when none). Arithmetic is float as in the reference; cuBQL's triangle
 * closest point is replaced by the reference's point_triangle_closest_point<float>, and among
 * primitives at the same squared distance the lowest index wins. The reference's skip_self defaults
 * to false; here it is an explicit argument. */
int ssdf_b200_closest_within_radius_bvh_ff(ptrdiff_t npoints, const float *x, const float *y, const float *z,
                                           ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                           ptrdiff_t nspoints, const float *sx, const float *sy, const float *sz,
                                           ptrdiff_t radius_stride, const float *radius_squared, int *outtri,
                                           float *out_sqr_dist, float *closest_x, float *closest_y,
                                           float *closest_z, int skip_self);
int ssdf_b200_closest_within_radius_bvh_fd(ptrdiff_t npoints, const float *x, const float *y, const float *z,
                                           ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                           ptrdiff_t nspoints, const float *sx, const float *sy, const float *sz,
                                           ptrdiff_t radius_stride, const double *radius_squared, int *outtri,
                                           double *out_sqr_dist, double *closest_x, double *closest_y,
                                           double *closest_z, int skip_self);
int ssdf_b200_closest_within_radius_bvh_dd(ptrdiff_t npoints, const double *x, const double *y, const double *z,
                                           ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                           ptrdiff_t nspoints, const double *sx, const double *sy, const double *sz,
                                           ptrdiff_t radius_stride, const double *radius_squared, int *outtri,
                                           double *out_sqr_dist, double *closest_x, double *closest_y,
                                           double *closest_z, int skip_self);
int ssdf_b200_closest_within_radius_local_bvh_ff(ptrdiff_t npoints, const float *x, const float *y, const float *z,
                                                 ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                                 ptrdiff_t nspoints, const float *sx, const float *sy,
                                                 const float *sz, ptrdiff_t radius_stride,
                                                 const float *radius_squared, int *outtri, float *out_sqr_dist,
                                                 float *closest_s, float *closest_t, int skip_self);
int ssdf_b200_closest_within_radius_local_bvh_fd(ptrdiff_t npoints, const float *x, const float *y, const float *z,
                                                 ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                                 ptrdiff_t nspoints, const float *sx, const float *sy,
                                                 const float *sz, ptrdiff_t radius_stride,
                                                 const double *radius_squared, int *outtri, double *out_sqr_dist,
                                                 double *closest_s, double *closest_t, int skip_self);
int ssdf_b200_closest_within_radius_local_bvh_dd(ptrdiff_t npoints, const double *x, const double *y,
                                                 const double *z, ptrdiff_t nselements, const int *s0, const int *s1,
                                                 const int *s2, ptrdiff_t nspoints, const double *sx,
                                                 const double *sy, const double *sz, ptrdiff_t radius_stride,
                                                 const double *radius_squared, int *outtri, double *out_sqr_dist,
                                                 double *closest_s, double *closest_t, int skip_self);
int ssdf_b200_closest_within_radius_quads_bvh_ff(ptrdiff_t npoints, const float *x, const float *y, const float *z,
                                                 ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                                 const int *s3, ptrdiff_t nspoints, const float *sx, const float *sy,
                                                 const float *sz, ptrdiff_t radius_stride,
                                                 const float *radius_squared, int *outtri, float *out_sqr_dist,
                                                 float *closest_x, float *closest_y, float *closest_z, int skip_self);
int ssdf_b200_closest_within_radius_quads_bvh_fd(ptrdiff_t npoints, const float *x, const float *y, const float *z,
                                                 ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                                 const int *s3, ptrdiff_t nspoints, const float *sx, const float *sy,
                                                 const float *sz, ptrdiff_t radius_stride,
                                                 const double *radius_squared, int *outtri, double *out_sqr_dist,
                                                 double *closest_x, double *closest_y, double *closest_z,
                                                 int skip_self);
int ssdf_b200_closest_within_radius_quads_bvh_dd(ptrdiff_t npoints, const double *x, const double *y,
                                                 const double *z, ptrdiff_t nselements, const int *s0, const int *s1,
                                                 const int *s2, const int *s3, ptrdiff_t nspoints, const double *sx,
                                                 const double *sy, const double *sz, ptrdiff_t radius_stride,
                                                 const double *radius_squared, int *outtri, double *out_sqr_dist,
                                                 double *closest_x, double *closest_y, double *closest_z,
                                                 int skip_self);
int ssdf_b200_closest_within_radius_quads_local_bvh_ff(ptrdiff_t npoints, const float *x, const float *y,
                                                       const float *z, ptrdiff_t nselements, const int *s0,
                                                       const int *s1, const int *s2, const int *s3,
                                                       ptrdiff_t nspoints, const float *sx, const float *sy,
                                                       const float *sz, ptrdiff_t radius_stride,
                                                       const float *radius_squared, int *outtri, float *out_sqr_dist,
                                                       float *closest_s, float *closest_t, int skip_self);
int ssdf_b200_closest_within_radius_quads_local_bvh_fd(ptrdiff_t npoints, const float *x, const float *y,
                                                       const float *z, ptrdiff_t nselements, const int *s0,
                                                       const int *s1, const int *s2, const int *s3,
                                                       ptrdiff_t nspoints, const float *sx, const float *sy,
                                                       const float *sz, ptrdiff_t radius_stride,
                                                       const double *radius_squared, int *outtri,
                                                       double *out_sqr_dist, double *closest_s, double *closest_t,
                                                       int skip_self);
int ssdf_b200_closest_within_radius_quads_local_bvh_dd(ptrdiff_t npoints, const double *x, const double *y,
                                                       const double *z, ptrdiff_t nselements, const int *s0,
                                                       const int *s1, const int *s2, const int *s3,
                                                       ptrdiff_t nspoints, const double *sx, const double *sy,
                                                       const double *sz, ptrdiff_t radius_stride,
                                                       const double *radius_squared, int *outtri,
                                                       double *out_sqr_dist, double *closest_s, double *closest_t,
                                                       int skip_self);

/* ---- drop-in: candidate contact pairs -----------------------------------------------------------
 * ssdf::potential_contact_triangles_bvh / potential_contact_quads_bvh<G, G, int, int>
 * (serial/bvh/bvh.hpp:156-181, bvh.cpp:834-1196), for G = float _ff and double _dd. For each
 * element (triangle s0/s1/s2 or quad s0/s1/s2/s3), the other elements whose tight float box meets
 * its own box grown by `extrusion` along its unit normal(s) and by a tenth of it against them, and
 * which share no corner index with it. pc_ptr[nselements + 1] receives the CSR offsets and
 * *out_pc_idx a malloc'd array of pc_ptr[nselements] element indices (the caller frees it with
 * free(), or ssdf_b200_free), each row in the order of the BVH walk (deterministic; the reference's
 * is its threads' order). The triangle normal is taken as the unit
 * normal (cuBQL's Triangle::normal(), not available to this build); quads use the reference's
 * per-corner normals. */
int ssdf_b200_potential_contact_triangles_bvh_ff(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                                 ptrdiff_t nspoints, const float *sx, const float *sy, const float *sz,
                                                 float extrusion, ptrdiff_t *pc_ptr, int **out_pc_idx);
int ssdf_b200_potential_contact_triangles_bvh_dd(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                                 ptrdiff_t nspoints, const double *sx, const double *sy,
                                                 const double *sz, double extrusion, ptrdiff_t *pc_ptr,
                                                 int **out_pc_idx);
int ssdf_b200_potential_contact_quads_bvh_ff(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                             const int *s3, ptrdiff_t nspoints, const float *sx, const float *sy,
                                             const float *sz, float extrusion, ptrdiff_t *pc_ptr, int **out_pc_idx);
int ssdf_b200_potential_contact_quads_bvh_dd(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                             const int *s3, ptrdiff_t nspoints, const double *sx, const double *sy,
                                             const double *sz, double extrusion, ptrdiff_t *pc_ptr,
                                             int **out_pc_idx);
/* free() from the library's C runtime, for callers (ctypes and the like) that cannot call it. */
void ssdf_b200_free(void *p);

/* ---- drop-in: grid and box helpers ------------------------------------------------------------
 * ssdf::compute_aabb<G, T> (serial/edf/edf.hpp:500-539): the bounding box of npoints (>= 1) points,
 * each converted to T, written to the six scalars. Bitwise the reference's for NaN-free input (a
 * NaN coordinate is skipped). Zero points: SSDF_ERR_INVALID_ARGUMENT (the reference reads x[0]). */
int ssdf_b200_compute_aabb_ff(ptrdiff_t npoints, const float *x, const float *y, const float *z, float *xmin,
                              float *xmax, float *ymin, float *ymax, float *zmin, float *zmax);
int ssdf_b200_compute_aabb_fd(ptrdiff_t npoints, const float *x, const float *y, const float *z, double *xmin,
                              double *xmax, double *ymin, double *ymax, double *zmin, double *zmax);
int ssdf_b200_compute_aabb_df(ptrdiff_t npoints, const double *x, const double *y, const double *z, float *xmin,
                              float *xmax, float *ymin, float *ymax, float *zmin, float *zmax);
int ssdf_b200_compute_aabb_dd(ptrdiff_t npoints, const double *x, const double *y, const double *z, double *xmin,
                              double *xmax, double *ymin, double *ymax, double *zmin, double *zmax);
/* ssdf::all_points_aabb_signed_distance<G, T> (serial/edf/edf.hpp:541-557, point_aabb_signed_distance
 * at 193-221): out[i] = signed distance of point i (converted to T) to the box, negative inside,
 * bitwise the reference's T arithmetic. The reference's driver starts `out` at its absolute value
 * over the query points' own box (drivers/sdf.exe.cpp:316-326). */
int ssdf_b200_all_points_aabb_signed_distance_ff(ptrdiff_t npoints, const float *x, const float *y, const float *z,
                                                 float minx, float maxx, float miny, float maxy, float minz,
                                                 float maxz, float *out);
int ssdf_b200_all_points_aabb_signed_distance_fd(ptrdiff_t npoints, const float *x, const float *y, const float *z,
                                                 double minx, double maxx, double miny, double maxy, double minz,
                                                 double maxz, double *out);
int ssdf_b200_all_points_aabb_signed_distance_df(ptrdiff_t npoints, const double *x, const double *y,
                                                 const double *z, float minx, float maxx, float miny, float maxy,
                                                 float minz, float maxz, float *out);
int ssdf_b200_all_points_aabb_signed_distance_dd(ptrdiff_t npoints, const double *x, const double *y,
                                                 const double *z, double minx, double maxx, double miny,
                                                 double maxy, double minz, double maxz, double *out);

/* ---- drop-in: level sets and field rebuilds (serial/bvh/sdf_rebuild.hpp) ---------------------
 * A grid is ssdf::GridGeometry<G> (sdf_rebuild.hpp:10-21) as three arrays: n[3] samples along each
 * axis at o[d] + i h[d], x fastest. Host arrays, blocking. */

/* ssdf::level_set_triangles (sdf_rebuild.hpp:23-37): the triangles of {f = level} by marching
 * tetrahedra (six per cell about the corner-0-to-7 diagonal; crossings interpolated from the lower
 * grid index; triangles with two vertices equal in G dropped), in the reference's order, each
 * vertex bitwise its value. *ntriangles receives the count; with x non-null and capacity >= count
 * the soup (three vertices per triangle) is written to x, y, z [3 * count]. */
int ssdf_b200_level_set_triangles_ff(const ptrdiff_t n[3], const float o[3], const float h[3], const float *f,
                                     float level, ptrdiff_t capacity, float *x, float *y, float *z,
                                     ptrdiff_t *ntriangles);
int ssdf_b200_level_set_triangles_dd(const ptrdiff_t n[3], const double o[3], const double h[3], const double *f,
                                     double level, ptrdiff_t capacity, double *x, double *y, double *z,
                                     ptrdiff_t *ntriangles);
/* ssdf::rebuild_sdf (sdf_rebuild.hpp:38-50, sdf_rebuild.cpp:252-299): out[strided(stride).size()] =
 * sign(f - level) * min(band, distance to those triangles), 0 on the level set; samples with
 * |f - level| >= band get +-band unsearched. The distance is the double one from the sample (the
 * reference searches in float with cuBQL from the float-rounded sample). */
int ssdf_b200_rebuild_sdf_ff(const ptrdiff_t n[3], const float o[3], const float h[3], const float *f, float level,
                             float band, ptrdiff_t stride, float *out);
int ssdf_b200_rebuild_sdf_dd(const ptrdiff_t n[3], const double o[3], const double h[3], const double *f,
                             double level, double band, ptrdiff_t stride, double *out);
/* ssdf::refine_field (sdf_rebuild.hpp:52-56): fine[refined(factor).size()], the cubic through the four
 * nearest samples along each axis in turn, bitwise the reference's double arithmetic. */
int ssdf_b200_refine_field_ff(const ptrdiff_t n[3], const float o[3], const float h[3], const float *f,
                              ptrdiff_t factor, float *fine);
int ssdf_b200_refine_field_dd(const ptrdiff_t n[3], const double o[3], const double h[3], const double *f,
                              ptrdiff_t factor, double *fine);
/* ssdf::round_sdf (sdf_rebuild.hpp:57-78): the region f > 0 rounded by radius (opening and / or
 * closing, each a rebuild), its signed distance on every stride-th sample; f0 (may be NULL) gets
 * the first rebuild R(f, 0) on the full grid. */
int ssdf_b200_round_sdf_ff(const ptrdiff_t n[3], const float o[3], const float h[3], const float *f, float radius,
                           float band, int open, int close, ptrdiff_t stride, float *out, float *f0);
int ssdf_b200_round_sdf_dd(const ptrdiff_t n[3], const double o[3], const double h[3], const double *f, double radius,
                           double band, int open, int close, ptrdiff_t stride, double *out, double *f0);

/* ---- additive entry points (no reference counterpart; patterned on closest_point_bvh) -------- */

/* Unsigned distance (in/out, as edf_bvh) plus the closest triangle, written where it improves. */
int ssdf_b200_edf_index_dd(ptrdiff_t npoints, const double *x, const double *y, const double *z,
                           ptrdiff_t nselements, const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints,
                           const double *sx, const double *sy, const double *sz, double *out, int *outtri);
int ssdf_b200_edf_index_ff(ptrdiff_t npoints, const float *x, const float *y, const float *z,
                           ptrdiff_t nselements, const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints,
                           const float *sx, const float *sy, const float *sz, float *out, int *outtri);
/* Signed distance and closest triangle at a point list (sample_sdf_bvh's sign rule). */
int ssdf_b200_sdf_points_dd(ptrdiff_t npoints, const double *x, const double *y, const double *z,
                            ptrdiff_t nselements, const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints,
                            const double *sx, const double *sy, const double *sz, double *out, int *outtri);
/* sample_sdf_bvh plus the closest triangle per grid node. */
int ssdf_b200_sample_sdf_index_bvh_dd(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                      ptrdiff_t nspoints, const double *sx, const double *sy, const double *sz,
                                      ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz, double xmin, double ymin,
                                      double zmin, double xmax, double ymax, double zmax, double *out, int *outtri);

/* ---- device-resident meshes (no reference counterpart: the reference rebuilds per call,
 *      serial/bvh/bvh.cu:80-158) ------------------------------------------------------------ */

typedef struct ssdf_mesh ssdf_mesh;

#define SSDF_F32 0
#define SSDF_F64 1

/* Arithmetic of the closest-triangle search. */
#define SSDF_PREC_F32 0       /* float throughout, the reference's float expressions           */
#define SSDF_PREC_F64 1       /* double throughout: the plain FP64 kernel                      */
#define SSDF_PREC_F32_FIXUP 2 /* float traversal, double re-evaluation of the near-tied set:
                                 bitwise the double result                                    */

/* What a query writes. */
#define SSDF_OUT_EDF 0     /* out = sqrt(min(out^2, d^2)) (in/out), outtri where it improves   */
#define SSDF_OUT_SQEDF 1   /* out = min(out, d^2) (in/out)                                     */
#define SSDF_OUT_SDF 2     /* out = +-d (overwrite), outtri                                    */
#define SSDF_OUT_CLOSEST 3 /* closest_point_bvh: outd/outxyz/outtri where d < outd (in/out)   */

typedef struct {
    int leaf_size;    /* triangles per BVH leaf, 1..16 (0: 4)                                 */
    int keep_fp64;    /* 1: also keep double triangles and nodes (F64 and fix-up queries)      */
    int normals;      /* 1: build pseudo-normals (signed queries)                             */
    int treelet_opt;  /* rounds of SAH treelet refinement of the LBVH (0: plain LBVH; <= 8); 3 when opts is null */
} ssdf_build_opts;

typedef struct {
    int precision;    /* SSDF_PREC_*                                                          */
    int output;       /* SSDF_OUT_*                                                           */
    int coord_type;   /* SSDF_F32 / SSDF_F64: type of x, y, z or of the grid bounds (G)       */
    int out_type;     /* SSDF_F32 / SSDF_F64: type of out / outd (T)                          */
    int reserved[4];
} ssdf_query_opts;

/* Creates a device-resident mesh (triangles, BVH, optional normals) from HOST (device_ptrs=0)
 * or DEVICE (device_ptrs=1) arrays of coord_type. Blocks until built. */
int ssdf_mesh_create(ssdf_mesh **mesh, ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                     ptrdiff_t nspoints, const void *sx, const void *sy, const void *sz, int coord_type,
                     int device_ptrs, const ssdf_build_opts *opts, void *stream);
/* Frees the mesh after waiting for all work on its device (queries on any stream may still read it). */
int ssdf_mesh_destroy(ssdf_mesh *mesh);
/* Frees the mesh in stream order: after the work already queued on `stream`, without waiting. Only
 * for a mesh whose queries were all queued on that stream. */
int ssdf_mesh_destroy_async(ssdf_mesh *mesh, void *stream);
/* BVH statistics: nodes, leaves, depth, bytes resident on the device. */
int ssdf_mesh_stats(const ssdf_mesh *mesh, int64_t *nodes, int64_t *leaves, int64_t *depth, int64_t *bytes);
/* The fix-up path's view of a mesh (no counterpart in the reference): tau_rel, the relative width of
 * its FP32 window (tau = tau_rel (M + d), M the largest coordinate magnitude, d the distance; at least
 * 2^-16, wider for meshes of a few large triangles); float_filter, 1 when fix-up requests on it run the
 * FP32 filter, 0 when they run the FP64 kernel (coordinates beyond 2^28, triangles that rounding to
 * float collapses or makes smaller than 2^-23, or more than half of its triangles slivers); slivers,
 * the triangles the filter sees through a proxy. Any pointer may be null. */
int ssdf_mesh_filter_info(const ssdf_mesh *mesh, float *tau_rel, int *float_filter, int64_t *slivers);

/* Query at device points (x, y, z of coord_type). outx/outy/outz (coord_type) and outtri may be NULL
 * except for SSDF_OUT_CLOSEST. Asynchronous on `stream`. */
int ssdf_query_points(ssdf_mesh *mesh, ptrdiff_t npoints, const void *x, const void *y, const void *z, void *out,
                      int *outtri, void *outx, void *outy, void *outz, const ssdf_query_opts *opts, void *stream);
/* ssdf::edf / ssdf::edf_celllist (serial/ssdf.hpp:447-619, 642-963) on device arrays: method 0 the
 * brute force (edf), 1 the cell list (edf_celllist); points, vertices and out all of coord_type
 * (G == T, as the reference instantiates them), out in/out; outtri (the closest triangle) may be
 * NULL. Enqueued on `stream`; returns when the query has finished (it reads back a validation flag). */
int ssdf_edf_device(int method, ptrdiff_t npoints, const void *x, const void *y, const void *z, ptrdiff_t nselements,
                    const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints, const void *sx, const void *sy,
                    const void *sz, int coord_type, void *out, int *outtri, void *stream);
/* Query at the node grid nx*ny*nz over [lo, hi] (ssdf's convention, G = coord_type precision). */
int ssdf_query_grid(ssdf_mesh *mesh, ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz, const double lo[3],
                    const double hi[3], void *out, int *outtri, const ssdf_query_opts *opts, void *stream);

/* Device-array forms of the box helpers, asynchronous on `stream` (x, y, z of coord_type; results
 * of out_type, SSDF_F32 / SSDF_F64 each). ssdf_points_aabb writes xmin, xmax, ymin, ymax, zmin, zmax
 * to the DEVICE array box6 (scratch is stream-ordered). ssdf_points_aabb_signed_distance takes the
 * box from the HOST array box6 in the same order (converted to out_type) and writes out[npoints]; with
 * absolute = 1 it writes |distance|, the reference driver's initial `out`. */
int ssdf_points_aabb(ptrdiff_t npoints, const void *x, const void *y, const void *z, int coord_type, int out_type,
                     void *box6, void *stream);
int ssdf_points_aabb_signed_distance(ptrdiff_t npoints, const void *x, const void *y, const void *z, int coord_type,
                                     const double box6[6], int absolute, void *out, int out_type, void *stream);

/* ---- batches: many resident meshes and query sets in one persistent launch (no reference
 *      counterpart; ssdf answers one mesh per call) --------------------------------------------- */

typedef struct ssdf_batch ssdf_batch;

/* traversal: 0 automatic (warp packets for grids), 1 warp packets, 2 thread per query;
 * arity: 0 automatic (binary), 2, 4. One arithmetic (precision) per batch. */
int ssdf_batch_create(ssdf_batch **batch, int max_jobs, int precision, int traversal, int arity);
int ssdf_batch_destroy(ssdf_batch *batch);
/* Pre-sizes the batch's fix-up overflow lists for runs of up to max_queries queries in total, so
 * that ssdf_batch_run never grows them (growing frees and allocates device memory, which waits for
 * all work on the device). Optional; runs grow the lists themselves when needed. */
int ssdf_batch_reserve(ssdf_batch *batch, long long max_queries, void *stream);
/* Removes every job (the device table is rewritten on the next run). */
int ssdf_batch_clear(ssdf_batch *batch);
int ssdf_batch_size(const ssdf_batch *batch);
/* Adds one job: a node grid or a device point list against a resident mesh, outputs in device
 * memory; opts->precision must equal the batch's. */
int ssdf_batch_add_grid(ssdf_batch *batch, ssdf_mesh *mesh, ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz,
                        const double lo[3], const double hi[3], void *out, int *outtri, const ssdf_query_opts *opts);
int ssdf_batch_add_points(ssdf_batch *batch, ssdf_mesh *mesh, ptrdiff_t npoints, const void *x, const void *y,
                          const void *z, void *out, int *outtri, const ssdf_query_opts *opts);
/* Adds the z-planes z0 .. z0 + nz_slab - 1 of the node grid nx*ny*nz over [lo, hi] as one job: the
 * nodes keep the whole grid's coordinates (origin and spacing from the whole grid), so the slab's
 * results are bit for bit those of the same planes in a whole-grid job; out / outtri hold the slab's
 * nx*ny*nz_slab values. Lets a large grid be split into jobs that share batches with others. */
int ssdf_batch_add_grid_slab(ssdf_batch *batch, ssdf_mesh *mesh, ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz,
                             const double lo[3], const double hi[3], ptrdiff_t z0, ptrdiff_t nz_slab, void *out,
                             int *outtri, const ssdf_query_opts *opts);
/* Runs every job in one persistent launch (plus the fix-up window stage) on `stream`, asynchronously.
 * use_graph = 1: the launch sequence is captured into a CUDA graph on the first run and replayed
 * afterwards for any composition of jobs (the job table is device-resident). */
int ssdf_batch_run(ssdf_batch *batch, int use_graph, void *stream);
/* 128-query work items of the last run. */
long long ssdf_batch_last_blocks(const ssdf_batch *batch);

/* ---- autotuner (no reference counterpart) ------------------------------------------------------ */

typedef struct {
    int leaf_size; /* BVH leaf size: 2, 4 or 8                                               */
    int traversal; /* 1 warp packets, 2 thread per query                                      */
    int arity;     /* 2 binary, 4 four-wide                                                   */
    double ms;     /* measured time of the winner on the sample grid                         */
} ssdf_tuning;

/* Times leaf sizes {2, 4, 8} x traversal {warp, thread} x arity {2, 4} for this mesh (host double
 * arrays) on a sample of the grid -- the same box at up to 2^21 nodes -- in the given arithmetic,
 * and returns the fastest. With cache_path (a JSON file) the winner is stored per size class
 * (log2 triangles, log2 nodes, arithmetic) and later calls of that class return it untimed. */
int ssdf_autotune_grid(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints,
                       const double *sx, const double *sy, const double *sz, ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz,
                       const double lo[3], const double hi[3], int precision, const char *cache_path,
                       ssdf_tuning *best);

/* ---- pedf_update's selection steps on the device (distributed/psdf.hpp:327-470) -------------- */
/* The box of npoints device points grown by their distances out: box6 (device, coord_type) =
 * min(x - r), min(y - r), min(z - r), max(x + r), max(y + r), max(z + r), r = out in coord_type
 * (psdf.hpp:327-361); (max, max, max, lowest, lowest, lowest) for no points. Asynchronous. */
int ssdf_grown_box(ptrdiff_t npoints, const void *x, const void *y, const void *z, const void *out, int coord_type,
                   int out_type, void *box6, void *stream);
/* For each of nboxes boxes (device, 6 values of coord_type each, in ssdf_grown_box's order), the
 * triangles whose corner box meets it (closed intervals, psdf.hpp:378-452), in triangle order: their
 * corners (x0 y0 z0 x1 y1 z1 x2 y2 z2) into the device array corners, box after box, and their count
 * per box into the HOST array counts[nboxes]. With corners NULL only the counts are computed; a
 * total above capacity (triangles) is an error. Returns when done. */
int ssdf_triangles_meeting_boxes(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                 ptrdiff_t nspoints, const void *sx, const void *sy, const void *sz, int coord_type,
                                 int nboxes, const void *boxes, void *corners, long long capacity, long long *counts,
                                 void *stream);

/* ---- ssdf::pedf / ssdf::pedf_update (distributed/psdf.hpp:149-302, 304-482) over NCCL --------
 * One process per GPU, every rank of the communicator calls it (collective). comm is an ncclComm_t;
 * this rank's points (x, y, z), its part of the surface (s0, s1, s2 over its own nspoints vertices)
 * and out are DEVICE arrays; the exchanges run on `stream` and the call returns when out holds
 * min(out, distance to the union of every rank's part) -- bitwise what the single-process edf_bvh
 * gives on the whole surface. coord_type / out_type: <F64, F64>, <F32, F64> or <F32, F32>.
 * ssdf_pedf_nccl gathers the whole surface (SSDF_USE_ALLGATHER=1, default) or broadcasts the parts one
 * after the other (0), as the reference; ssdf_pedf_update_nccl exchanges only the triangles meeting
 * each rank's points' box grown by their current out (which must hold upper bounds). NCCL is opened
 * at the first call (libnccl.so.2); without it these return SSDF_ERR_NOT_SUPPORTED. */
int ssdf_pedf_nccl(void *comm, ptrdiff_t npoints, const void *x, const void *y, const void *z, ptrdiff_t nselements,
                   const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints, const void *sx, const void *sy,
                   const void *sz, int coord_type, int out_type, void *out, void *stream);
int ssdf_pedf_update_nccl(void *comm, ptrdiff_t npoints, const void *x, const void *y, const void *z,
                          ptrdiff_t nselements, const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints,
                          const void *sx, const void *sy, const void *sz, int coord_type, int out_type, void *out,
                          void *stream);

/* ---- serving loop: continuous batching over resident meshes (no reference counterpart) ------- */

typedef struct ssdf_server ssdf_server;

typedef struct {
    size_t memory_budget;  /* bytes of device-resident mesh data; LRU eviction beyond it        */
    int max_batch_queries; /* queries packed into one batch (also the largest request)         */
    int max_batch_jobs;    /* requests packed into one batch                                   */
    int precision;         /* SSDF_PREC_F32_FIXUP or SSDF_PREC_F64                             */
    int leaf_size;         /* BVH leaf size of resident meshes (0: default)                    */
    int slots;             /* batches in flight at once, 1..16 (0: 8); each holds its buffers  */
    long long max_queued_queries; /* admission limit: a request that would bring the queries waiting
                                     to be packed above it is refused with SSDF_ERR_BUSY (0: none) */
    int split_queries;     /* requests larger than this are answered as parts (z-slabs of a grid,
                              runs of a point list) packed round-robin with the other waiting
                              requests (0: 262144; must not exceed max_batch_queries)              */
} ssdf_server_opts;

typedef struct {
    long long completed;                  /* requests finished since the last reset            */
    double p50_ms, p99_ms, max_ms;        /* submit -> result-in-caller-buffer latency          */
    long long queries, batches, evictions, builds;
    long long resident_bytes, resident_meshes;
    double seconds;                       /* first submit -> last completion                   */
    long long rejected;                   /* requests refused by the admission limit           */
} ssdf_server_report;

/* A scheduler thread packs waiting requests into one persistent batch launch per free slot (several
 * slots, so one batch's upload, kernels and download overlap the others' and a batch's slow tail
 * leaves the SMs to the next); one completer thread per slot delivers its results. Results are
 * signed distances (double) and closest triangles written to the caller's HOST buffers. */
int ssdf_server_create(ssdf_server **server, const ssdf_server_opts *opts);
int ssdf_server_destroy(ssdf_server *server);
/* Registers a mesh (host arrays, copied); it is built on the device when first queried. */
int ssdf_server_add_mesh(ssdf_server *server, ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                         ptrdiff_t nspoints, const double *sx, const double *sy, const double *sz, int *mesh_id);
/* Asynchronous requests; the host arrays must stay valid until ssdf_server_wait returns. A request
 * over the admission limit returns SSDF_ERR_BUSY at once (nothing is queued). */
int ssdf_server_submit_points(ssdf_server *server, int mesh_id, ptrdiff_t npoints, const double *x, const double *y,
                              const double *z, double *out, int *outtri, long long *ticket);
int ssdf_server_submit_grid(ssdf_server *server, int mesh_id, ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz,
                            const double lo[3], const double hi[3], double *out, int *outtri, long long *ticket);
int ssdf_server_wait(ssdf_server *server, long long ticket, double timeout_s);
int ssdf_server_stats(ssdf_server *server, ssdf_server_report *stats);
int ssdf_server_reset_stats(ssdf_server *server);

/* ---- allocation-free grid query (no counterpart in the reference) ----------------------------
 * ssdf_query_grid with SSDF_PREC_F32_FIXUP, for callers that must not allocate device memory while
 * they query: loops that reserve all memory up front, hosts that forbid the CUDA allocator or own
 * every allocation. It allocates nothing: the fix-up overflow list lives in a fixed 8 MiB array
 * inside the library, held by every GPU that loads the library until the process exits. Limits:
 * at most ssdf_query_grid_noalloc_max() (1,048,576) nodes per call, larger grids are rejected with
 * SSDF_ERR_NOT_SUPPORTED (query them slab by slab); SSDF_PREC_F32_FIXUP only. The mesh is built
 * beforehand with ssdf_mesh_create. The first call on a device looks up the array's device address
 * (once per device): make that first call before any stream capture. All calls share the array and
 * each one resets it, so calls whose kernels overlap on the GPU (concurrent streams) race: order
 * them on one stream. */
int ssdf_query_grid_noalloc(ssdf_mesh *mesh, ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz, const double lo[3],
                            const double hi[3], void *out, int *outtri, const ssdf_query_opts *opts, void *stream);
long long ssdf_query_grid_noalloc_max(void);

/* Diagnostics for measurement: per-query triangle and box test counts of the last query on this
 * thread when SSDF_B200_COUNT=1 was set at its launch (an untimed, instrumented launch). */
int ssdf_last_query_counts(int64_t *triangle_tests, int64_t *box_tests, int64_t *fixup_queries,
                           int64_t *fallback_queries);

/* Measured fused multiply-add throughput of the current GPU in TFLOP/s (f64 = 0: float, 1: double),
 * the denominator of the traversal kernels' roofline. */
int ssdf_b200_fma_peak(int f64, double *tflops);

#ifdef __cplusplus
}
#endif

#endif /* SSDF_B200_H */
