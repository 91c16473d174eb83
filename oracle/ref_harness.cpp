// ref_harness.cpp -- C entry points over the reference's own templates (serial/ssdf.hpp,
// serial/edf/edf.hpp), compiled from the sources where they lie by oracle/Makefile into
// oracle/_ref/libssdf_ref.so.
//
// TEST INFRASTRUCTURE ONLY: used to pin the oracle and as the timed CPU baseline
// (bench.py --impl reference); the product never loads it. The reference's own exports
// ssdf_edf_f / ssdf_edf_d (serial/ssdf.cpp:36-66) come from serial/ssdf.cpp in the same link.
#include <iostream>
#include <streambuf>

#include "ssdf.hpp"

namespace {
    // The reference prints "<name> took X ms" from inside edf / edf_celllist (SSDF_TIMER,
    // serial/ssdf.hpp:25-46); a timed caller can route std::cout to this sink.
    struct NullBuf : std::streambuf {
        int overflow(int c) override { return c; }
    };
    NullBuf null_buf;
    std::streambuf *saved_buf = nullptr;
}  // namespace

#define REF_ARGS(G)                                                                                       \
    const ptrdiff_t npoints, const G *x, const G *y, const G *z, const ptrdiff_t nselements, const int *s0, \
        const int *s1, const int *s2, const ptrdiff_t nspoints, const G *sx, const G *sy, const G *sz, G *out
#define REF_PASS npoints, x, y, z, nselements, s0, s1, s2, nspoints, sx, sy, sz, out

extern "C" {

void ref_set_quiet(const int quiet) {
    if (quiet && !saved_buf) {
        saved_buf = std::cout.rdbuf(&null_buf);
    } else if (!quiet && saved_buf) {
        std::cout.rdbuf(saved_buf);
        saved_buf = nullptr;
    }
}

int ref_edf_d(REF_ARGS(double)) { return ssdf::edf<double, double, int>(REF_PASS); }
int ref_edf_f(REF_ARGS(float)) { return ssdf::edf<float, float, int>(REF_PASS); }
int ref_edf_celllist_d(REF_ARGS(double)) { return ssdf::edf_celllist<double, double, int>(REF_PASS); }
int ref_edf_celllist_f(REF_ARGS(float)) { return ssdf::edf_celllist<float, float, int>(REF_PASS); }

double ref_point_triangle_dist_sq_d(double px, double py, double pz, double ax, double ay, double az, double bx,
                                    double by, double bz, double cx, double cy, double cz) {
    return ssdf::point_triangle_dist_sq<double>(px, py, pz, ax, ay, az, bx, by, bz, cx, cy, cz);
}
float ref_point_triangle_dist_sq_f(float px, float py, float pz, float ax, float ay, float az, float bx, float by,
                                   float bz, float cx, float cy, float cz) {
    return ssdf::point_triangle_dist_sq<float>(px, py, pz, ax, ay, az, bx, by, bz, cx, cy, cz);
}
void ref_point_triangle_closest_point_d(double px, double py, double pz, double ax, double ay, double az, double bx,
                                        double by, double bz, double cx, double cy, double cz, double *ox, double *oy,
                                        double *oz) {
    ssdf::point_triangle_closest_point<double>(px, py, pz, ax, ay, az, bx, by, bz, cx, cy, cz, ox, oy, oz);
}
double ref_point_aabb_distance_squared_d(double px, double py, double pz, double minx, double maxx, double miny,
                                         double maxy, double minz, double maxz) {
    return ssdf::point_aabb_distance_squared<double>(px, py, pz, minx, maxx, miny, maxy, minz, maxz);
}
double ref_point_aabb_signed_distance_d(double px, double py, double pz, double minx, double maxx, double miny,
                                        double maxy, double minz, double maxz) {
    return ssdf::point_aabb_signed_distance<double>(px, py, pz, minx, maxx, miny, maxy, minz, maxz);
}

#define REF_BOX(T, SUF)                                                                                       \
    void ref_compute_aabb##SUF(const ptrdiff_t n, const T *x, const T *y, const T *z, T *b) {                 \
        ssdf::compute_aabb<T, T>(n, x, y, z, b, b + 1, b + 2, b + 3, b + 4, b + 5);                           \
    }                                                                                                         \
    void ref_all_points_aabb_signed_distance##SUF(const ptrdiff_t n, const T *x, const T *y, const T *z,      \
                                                 const T *b, T *out) {                                        \
        ssdf::all_points_aabb_signed_distance<T, T>(n, x, y, z, b[0], b[1], b[2], b[3], b[4], b[5], out);      \
    }
REF_BOX(double, _d)
REF_BOX(float, _f)

// point_triangle_barycentric / point_to_quad_closest_point (serial/edf/edf.hpp:251-489), the
// primitives of the closest-within-radius queries.
#define REF_QUAD(T, SUF)                                                                                      \
    T ref_point_triangle_barycentric##SUF(T qx, T qy, T qz, T ax, T ay, T az, T bx, T by, T bz, T cx, T cy,    \
                                          T cz, T *w) {                                                       \
        return ssdf::point_triangle_barycentric<T>(qx, qy, qz, ax, ay, az, bx, by, bz, cx, cy, cz, w, w + 1,   \
                                                   w + 2);                                                    \
    }                                                                                                         \
    void ref_point_to_quad_closest_point##SUF(const T *p, const T *v, T *st) {                                \
        ssdf::point_to_quad_closest_point<T>(p[0], p[1], p[2], v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7],  \
                                             v[8], v[9], v[10], v[11], st, st + 1);                           \
    }
REF_QUAD(double, _d)
REF_QUAD(float, _f)
}
