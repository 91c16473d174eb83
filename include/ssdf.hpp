// ssdf.hpp -- the reference's C++ template API (namespace ssdf), served by the B200 library.
//
// A drop-in for zulianp/ssdf's serial/ssdf.hpp (edf, edf_celllist, edf_select) and
// serial/bvh/bvh.hpp (edf_bvh, closest_point_bvh, sample_sqedf_bvh, sample_sdf_bvh, inside flags,
// closest_within_radius_*, potential_contact_*) and the grid
// helpers of serial/edf/edf.hpp (compute_aabb, all_points_aabb_signed_distance): same names,
// template parameters <G coordinates, T outputs, I indices>, argument order, in/out semantics and
// int return (0 on success). Each instantiation the reference provides maps onto one C symbol of
// libssdf_b200.so (include/ssdf_b200.h); other type combinations do not compile.
// Link with -lssdf_b200. Unlike the reference, a failure returns a non-zero status
// (SSDF_ERR_*) instead of aborting; ssdf_last_error() describes it.
#ifndef SSDF_B200_SSDF_HPP
#define SSDF_B200_SSDF_HPP

#include <stddef.h>

#include <type_traits>
#include <vector>

#include "ssdf_b200.h"

#ifndef SSDF_RESTRICT
#define SSDF_RESTRICT __restrict__
#endif

namespace ssdf {

namespace detail {
template <typename...>
struct always_false : std::false_type {};
}  // namespace detail

#define SSDF_B200_EDF_SIG(G, T)                                                                                   \
    const ptrdiff_t npoints, const G *const SSDF_RESTRICT x, const G *const SSDF_RESTRICT y,                      \
        const G *const SSDF_RESTRICT z, const ptrdiff_t nselements, const I *const SSDF_RESTRICT s0,               \
        const I *const SSDF_RESTRICT s1, const I *const SSDF_RESTRICT s2, const ptrdiff_t nspoints,               \
        const G *const SSDF_RESTRICT sx, const G *const SSDF_RESTRICT sy, const G *const SSDF_RESTRICT sz,         \
        T *const SSDF_RESTRICT out
#define SSDF_B200_EDF_PASS npoints, x, y, z, nselements, s0, s1, s2, nspoints, sx, sy, sz, out

// serial/ssdf.hpp:447-619
template <typename G, typename T, typename I>
int edf(SSDF_B200_EDF_SIG(G, T)) {
    static_assert(std::is_same<I, int>::value, "ssdf_b200 indices are int");
    if constexpr (std::is_same<G, float>::value && std::is_same<T, float>::value)
        return ssdf_b200_edf_ff(SSDF_B200_EDF_PASS);
    else if constexpr (std::is_same<G, double>::value && std::is_same<T, double>::value)
        return ssdf_b200_edf_dd(SSDF_B200_EDF_PASS);
    else
        static_assert(detail::always_false<G, T>::value, "edf is instantiated for <float,float> and <double,double>");
}

// serial/ssdf.hpp:642-963
template <typename G, typename T, typename I>
int edf_celllist(SSDF_B200_EDF_SIG(G, T)) {
    static_assert(std::is_same<I, int>::value, "ssdf_b200 indices are int");
    if constexpr (std::is_same<G, float>::value && std::is_same<T, float>::value)
        return ssdf_b200_edf_celllist_ff(SSDF_B200_EDF_PASS);
    else if constexpr (std::is_same<G, double>::value && std::is_same<T, double>::value)
        return ssdf_b200_edf_celllist_dd(SSDF_B200_EDF_PASS);
    else
        static_assert(detail::always_false<G, T>::value,
                      "edf_celllist is instantiated for <float,float> and <double,double>");
}

// serial/ssdf.hpp:965-1016 (SSDF_USE_BVH / SSDF_CELL_VALIDATE / SSDF_USE_CELL_LIST)
template <typename G, typename T, typename I>
int edf_select(SSDF_B200_EDF_SIG(G, T)) {
    static_assert(std::is_same<I, int>::value, "ssdf_b200 indices are int");
    if constexpr (std::is_same<G, float>::value && std::is_same<T, float>::value)
        return ssdf_edf_f(SSDF_B200_EDF_PASS);
    else if constexpr (std::is_same<G, double>::value && std::is_same<T, double>::value)
        return ssdf_edf_d(SSDF_B200_EDF_PASS);
    else
        static_assert(detail::always_false<G, T>::value,
                      "edf_select is instantiated for <float,float> and <double,double>");
}

// serial/bvh/bvh.hpp:19-32 (instantiations serial/bvh/bvh.cpp:1216-1256)
template <typename G, typename T, typename I>
int edf_bvh(SSDF_B200_EDF_SIG(G, T)) {
    static_assert(std::is_same<I, int>::value, "ssdf_b200 indices are int");
    if constexpr (std::is_same<G, float>::value && std::is_same<T, float>::value)
        return ssdf_b200_edf_bvh_ff(SSDF_B200_EDF_PASS);
    else if constexpr (std::is_same<G, float>::value && std::is_same<T, double>::value)
        return ssdf_b200_edf_bvh_fd(SSDF_B200_EDF_PASS);
    else if constexpr (std::is_same<G, double>::value && std::is_same<T, double>::value)
        return ssdf_b200_edf_bvh_dd(SSDF_B200_EDF_PASS);
    else
        static_assert(detail::always_false<G, T>::value, "edf_bvh: <float,float>, <float,double>, <double,double>");
}

// serial/bvh/bvh.hpp:34-51
template <typename G, typename T, typename I>
int closest_point_bvh(const ptrdiff_t npoints, const G *const SSDF_RESTRICT x, const G *const SSDF_RESTRICT y,
                      const G *const SSDF_RESTRICT z, const ptrdiff_t nselements, const I *const SSDF_RESTRICT s0,
                      const I *const SSDF_RESTRICT s1, const I *const SSDF_RESTRICT s2, const ptrdiff_t nspoints,
                      const G *const SSDF_RESTRICT sx, const G *const SSDF_RESTRICT sy,
                      const G *const SSDF_RESTRICT sz, T *const SSDF_RESTRICT outd, G *const SSDF_RESTRICT outx,
                      G *const SSDF_RESTRICT outy, G *const SSDF_RESTRICT outz, I *const SSDF_RESTRICT outtri) {
    static_assert(std::is_same<I, int>::value, "ssdf_b200 indices are int");
    if constexpr (std::is_same<G, float>::value && std::is_same<T, float>::value)
        return ssdf_b200_closest_point_bvh_ff(npoints, x, y, z, nselements, s0, s1, s2, nspoints, sx, sy, sz, outd,
                                              outx, outy, outz, outtri);
    else if constexpr (std::is_same<G, float>::value && std::is_same<T, double>::value)
        return ssdf_b200_closest_point_bvh_fd(npoints, x, y, z, nselements, s0, s1, s2, nspoints, sx, sy, sz, outd,
                                              outx, outy, outz, outtri);
    else if constexpr (std::is_same<G, double>::value && std::is_same<T, double>::value)
        return ssdf_b200_closest_point_bvh_dd(npoints, x, y, z, nselements, s0, s1, s2, nspoints, sx, sy, sz, outd,
                                              outx, outy, outz, outtri);
    else
        static_assert(detail::always_false<G, T>::value,
                      "closest_point_bvh: <float,float>, <float,double>, <double,double>");
}

#define SSDF_B200_GRID_SIG(G, T)                                                                                  \
    const ptrdiff_t nselements, const I *const SSDF_RESTRICT s0, const I *const SSDF_RESTRICT s1,                 \
        const I *const SSDF_RESTRICT s2, const ptrdiff_t nspoints, const G *const SSDF_RESTRICT sx,                \
        const G *const SSDF_RESTRICT sy, const G *const SSDF_RESTRICT sz, const ptrdiff_t nx, const ptrdiff_t ny,  \
        const ptrdiff_t nz, const G xmin, const G ymin, const G zmin, const G xmax, const G ymax, const G zmax,    \
        T *const SSDF_RESTRICT out
#define SSDF_B200_GRID_PASS nselements, s0, s1, s2, nspoints, sx, sy, sz, nx, ny, nz, xmin, ymin, zmin, xmax, ymax, zmax, out

// serial/bvh/bvh.hpp:183-201
template <typename G, typename T, typename I>
int sample_sqedf_bvh(SSDF_B200_GRID_SIG(G, T)) {
    static_assert(std::is_same<I, int>::value, "ssdf_b200 indices are int");
    if constexpr (std::is_same<G, float>::value && std::is_same<T, float>::value)
        return ssdf_b200_sample_sqedf_bvh_ff(SSDF_B200_GRID_PASS);
    else if constexpr (std::is_same<G, double>::value && std::is_same<T, double>::value)
        return ssdf_b200_sample_sqedf_bvh_dd(SSDF_B200_GRID_PASS);
    else
        static_assert(detail::always_false<G, T>::value, "sample_sqedf_bvh: <float,float>, <double,double>");
}

// serial/bvh/bvh.hpp:203-227: positive on the side the right-handed normals point to
template <typename G, typename T, typename I>
int sample_sdf_bvh(SSDF_B200_GRID_SIG(G, T)) {
    static_assert(std::is_same<I, int>::value, "ssdf_b200 indices are int");
    if constexpr (std::is_same<G, float>::value && std::is_same<T, float>::value)
        return ssdf_b200_sample_sdf_bvh_ff(SSDF_B200_GRID_PASS);
    else if constexpr (std::is_same<G, double>::value && std::is_same<T, double>::value)
        return ssdf_b200_sample_sdf_bvh_dd(SSDF_B200_GRID_PASS);
    else
        static_assert(detail::always_false<G, T>::value, "sample_sdf_bvh: <float,float>, <double,double>");
}

#undef SSDF_B200_EDF_SIG
#undef SSDF_B200_EDF_PASS
#undef SSDF_B200_GRID_SIG
#undef SSDF_B200_GRID_PASS

// serial/edf/edf.hpp:500-539. The reference returns void; this returns the status (a discarded
// int return compiles at the same call sites).
template <typename G, typename T>
int compute_aabb(const ptrdiff_t npoints, const G *const SSDF_RESTRICT x, const G *const SSDF_RESTRICT y,
                 const G *const SSDF_RESTRICT z, T *const SSDF_RESTRICT xmin, T *const SSDF_RESTRICT xmax,
                 T *const SSDF_RESTRICT ymin, T *const SSDF_RESTRICT ymax, T *const SSDF_RESTRICT zmin,
                 T *const SSDF_RESTRICT zmax) {
    if constexpr (std::is_same<G, float>::value && std::is_same<T, float>::value)
        return ssdf_b200_compute_aabb_ff(npoints, x, y, z, xmin, xmax, ymin, ymax, zmin, zmax);
    else if constexpr (std::is_same<G, float>::value && std::is_same<T, double>::value)
        return ssdf_b200_compute_aabb_fd(npoints, x, y, z, xmin, xmax, ymin, ymax, zmin, zmax);
    else if constexpr (std::is_same<G, double>::value && std::is_same<T, float>::value)
        return ssdf_b200_compute_aabb_df(npoints, x, y, z, xmin, xmax, ymin, ymax, zmin, zmax);
    else if constexpr (std::is_same<G, double>::value && std::is_same<T, double>::value)
        return ssdf_b200_compute_aabb_dd(npoints, x, y, z, xmin, xmax, ymin, ymax, zmin, zmax);
    else
        static_assert(detail::always_false<G, T>::value, "compute_aabb: G and T are float or double");
}

// serial/edf/edf.hpp:541-557 (void in the reference; the status here, as compute_aabb).
template <typename G, typename T>
int all_points_aabb_signed_distance(const ptrdiff_t npoints, const G *const SSDF_RESTRICT x,
                                    const G *const SSDF_RESTRICT y, const G *const SSDF_RESTRICT z, const T minx,
                                    const T maxx, const T miny, const T maxy, const T minz, const T maxz,
                                    T *const SSDF_RESTRICT out) {
    if constexpr (std::is_same<G, float>::value && std::is_same<T, float>::value)
        return ssdf_b200_all_points_aabb_signed_distance_ff(npoints, x, y, z, minx, maxx, miny, maxy, minz, maxz, out);
    else if constexpr (std::is_same<G, float>::value && std::is_same<T, double>::value)
        return ssdf_b200_all_points_aabb_signed_distance_fd(npoints, x, y, z, minx, maxx, miny, maxy, minz, maxz, out);
    else if constexpr (std::is_same<G, double>::value && std::is_same<T, float>::value)
        return ssdf_b200_all_points_aabb_signed_distance_df(npoints, x, y, z, minx, maxx, miny, maxy, minz, maxz, out);
    else if constexpr (std::is_same<G, double>::value && std::is_same<T, double>::value)
        return ssdf_b200_all_points_aabb_signed_distance_dd(npoints, x, y, z, minx, maxx, miny, maxy, minz, maxz, out);
    else
        static_assert(detail::always_false<G, T>::value,
                      "all_points_aabb_signed_distance: G and T are float or double");
}

// serial/bvh/bvh.hpp:54-66
template <typename G, typename I>
int points_inside_bvh(const ptrdiff_t npoints, const G *const SSDF_RESTRICT x, const G *const SSDF_RESTRICT y,
                      const G *const SSDF_RESTRICT z, const ptrdiff_t nselements, const I *const SSDF_RESTRICT s0,
                      const I *const SSDF_RESTRICT s1, const I *const SSDF_RESTRICT s2, const ptrdiff_t nspoints,
                      const G *const SSDF_RESTRICT sx, const G *const SSDF_RESTRICT sy,
                      const G *const SSDF_RESTRICT sz, uint8_t *const SSDF_RESTRICT out) {
    static_assert(std::is_same<I, int>::value, "ssdf_b200 indices are int");
    if constexpr (std::is_same<G, float>::value)
        return ssdf_b200_points_inside_bvh_f(npoints, x, y, z, nselements, s0, s1, s2, nspoints, sx, sy, sz, out);
    else if constexpr (std::is_same<G, double>::value)
        return ssdf_b200_points_inside_bvh_d(npoints, x, y, z, nselements, s0, s1, s2, nspoints, sx, sy, sz, out);
    else
        static_assert(detail::always_false<G>::value, "points_inside_bvh: G is float or double");
}

// serial/bvh/bvh.hpp:230-247
template <typename G, typename I>
int sample_inside_bvh(const ptrdiff_t nselements, const I *const SSDF_RESTRICT s0, const I *const SSDF_RESTRICT s1,
                      const I *const SSDF_RESTRICT s2, const ptrdiff_t nspoints, const G *const SSDF_RESTRICT sx,
                      const G *const SSDF_RESTRICT sy, const G *const SSDF_RESTRICT sz, const ptrdiff_t nx,
                      const ptrdiff_t ny, const ptrdiff_t nz, const G xmin, const G ymin, const G zmin, const G xmax,
                      const G ymax, const G zmax, uint8_t *const SSDF_RESTRICT out) {
    static_assert(std::is_same<I, int>::value, "ssdf_b200 indices are int");
    if constexpr (std::is_same<G, float>::value)
        return ssdf_b200_sample_inside_bvh_f(nselements, s0, s1, s2, nspoints, sx, sy, sz, nx, ny, nz, xmin, ymin,
                                             zmin, xmax, ymax, zmax, out);
    else if constexpr (std::is_same<G, double>::value)
        return ssdf_b200_sample_inside_bvh_d(nselements, s0, s1, s2, nspoints, sx, sy, sz, nx, ny, nz, xmin, ymin,
                                             zmin, xmax, ymax, zmax, out);
    else
        static_assert(detail::always_false<G>::value, "sample_inside_bvh: G is float or double");
}

// ---- level sets and field rebuilds (serial/bvh/sdf_rebuild.hpp) ----------------------------------

// serial/bvh/sdf_rebuild.hpp:10-21: n[d] samples along axis d at o[d] + i h[d], x fastest.
template <typename G>
struct GridGeometry {
    ptrdiff_t n[3];
    G o[3];
    G h[3];

    ptrdiff_t size() const { return n[0] * n[1] * n[2]; }
    GridGeometry strided(const ptrdiff_t stride) const {
        GridGeometry s = *this;
        for (int d = 0; d < 3; ++d) {
            s.n[d] = (n[d] - 1) / stride + 1;
            s.h[d] = h[d] * G(stride);
        }
        return s;
    }
    GridGeometry refined(const ptrdiff_t factor) const {
        GridGeometry r = *this;
        for (int d = 0; d < 3; ++d) {
            r.n[d] = (n[d] - 1) * factor + 1;
            r.h[d] = G(double(h[d]) / double(factor));
        }
        return r;
    }
};

// serial/bvh/sdf_rebuild.hpp:23-37: appends the soup to x, y, z; returns the triangle count (or a
// negative status).
template <typename G, typename T>
ptrdiff_t level_set_triangles(const GridGeometry<G> &grid, const T *const f, const T level, std::vector<G> &x,
                              std::vector<G> &y, std::vector<G> &z) {
    static_assert(std::is_same<G, T>::value && (std::is_same<G, float>::value || std::is_same<G, double>::value),
                  "level_set_triangles is instantiated for <float,float> and <double,double>");
    ptrdiff_t nt = 0;
    auto call = [&](ptrdiff_t cap, G *px, G *py, G *pz) {
        if constexpr (std::is_same<G, float>::value)
            return ssdf_b200_level_set_triangles_ff(grid.n, grid.o, grid.h, f, level, cap, px, py, pz, &nt);
        else
            return ssdf_b200_level_set_triangles_dd(grid.n, grid.o, grid.h, f, level, cap, px, py, pz, &nt);
    };
    int st = call(0, nullptr, nullptr, nullptr);
    if (st != SSDF_OK) return -ptrdiff_t(st);
    const size_t first = x.size();
    x.resize(first + 3 * size_t(nt));
    y.resize(first + 3 * size_t(nt));
    z.resize(first + 3 * size_t(nt));
    if (nt > 0) st = call(nt, x.data() + first, y.data() + first, z.data() + first);
    return st == SSDF_OK ? nt : -ptrdiff_t(st);
}

// serial/bvh/sdf_rebuild.hpp:38-50
template <typename G, typename T>
int rebuild_sdf(const GridGeometry<G> &grid, const T *const f, const T level, const T band, const ptrdiff_t stride,
                T *const out) {
    if constexpr (std::is_same<G, float>::value && std::is_same<T, float>::value)
        return ssdf_b200_rebuild_sdf_ff(grid.n, grid.o, grid.h, f, level, band, stride, out);
    else if constexpr (std::is_same<G, double>::value && std::is_same<T, double>::value)
        return ssdf_b200_rebuild_sdf_dd(grid.n, grid.o, grid.h, f, level, band, stride, out);
    else
        static_assert(detail::always_false<G, T>::value, "rebuild_sdf is instantiated for <float,float> and <double,double>");
}

// serial/bvh/sdf_rebuild.hpp:52-56 (void in the reference; the status here)
template <typename G, typename T>
int refine_field(const GridGeometry<G> &grid, const T *const f, const ptrdiff_t factor, T *const fine) {
    if constexpr (std::is_same<G, float>::value && std::is_same<T, float>::value)
        return ssdf_b200_refine_field_ff(grid.n, grid.o, grid.h, f, factor, fine);
    else if constexpr (std::is_same<G, double>::value && std::is_same<T, double>::value)
        return ssdf_b200_refine_field_dd(grid.n, grid.o, grid.h, f, factor, fine);
    else
        static_assert(detail::always_false<G, T>::value, "refine_field is instantiated for <float,float> and <double,double>");
}

// serial/bvh/sdf_rebuild.hpp:57-78
template <typename G, typename T>
int round_sdf(const GridGeometry<G> &grid, const T *const f, const T radius, const T band, const bool open,
              const bool close, const ptrdiff_t stride, T *const out, T *const f0) {
    if constexpr (std::is_same<G, float>::value && std::is_same<T, float>::value)
        return ssdf_b200_round_sdf_ff(grid.n, grid.o, grid.h, f, radius, band, open, close, stride, out, f0);
    else if constexpr (std::is_same<G, double>::value && std::is_same<T, double>::value)
        return ssdf_b200_round_sdf_dd(grid.n, grid.o, grid.h, f, radius, band, open, close, stride, out, f0);
    else
        static_assert(detail::always_false<G, T>::value, "round_sdf is instantiated for <float,float> and <double,double>");
}

// serial/bvh/bvh.hpp:68-154: the closest primitive within a radius. Instantiations
// <float, float>, <float, double>, <double, double> (serial/bvh/bvh.cpp:1272-1521).
#define SSDF_B200_RADIUS_SIG(G, T)                                                                                \
    const ptrdiff_t npoints, const G *const SSDF_RESTRICT x, const G *const SSDF_RESTRICT y,                      \
        const G *const SSDF_RESTRICT z, const ptrdiff_t nselements, const I *const SSDF_RESTRICT s0,               \
        const I *const SSDF_RESTRICT s1, const I *const SSDF_RESTRICT s2
#define SSDF_B200_RADIUS_TAIL(G, T)                                                                               \
    const ptrdiff_t nspoints, const G *const SSDF_RESTRICT sx, const G *const SSDF_RESTRICT sy,                   \
        const G *const SSDF_RESTRICT sz, const ptrdiff_t radius_stride, const T *const SSDF_RESTRICT radius_squared, \
        I *const SSDF_RESTRICT outtri, T *const SSDF_RESTRICT out_sqr_dist
#define SSDF_B200_RADIUS_DISPATCH(NAME, ...)                                                                      \
    static_assert(std::is_same<I, int>::value, "ssdf_b200 indices are int");                                     \
    if constexpr (std::is_same<G, float>::value && std::is_same<T, float>::value)                                 \
        return ssdf_b200_##NAME##_ff(__VA_ARGS__);                                                                \
    else if constexpr (std::is_same<G, float>::value && std::is_same<T, double>::value)                           \
        return ssdf_b200_##NAME##_fd(__VA_ARGS__);                                                                \
    else if constexpr (std::is_same<G, double>::value && std::is_same<T, double>::value)                          \
        return ssdf_b200_##NAME##_dd(__VA_ARGS__);                                                                \
    else                                                                                                          \
        static_assert(detail::always_false<G, T>::value, #NAME ": <float,float>, <float,double>, <double,double>")

template <typename G, typename T, typename I>
int closest_within_radius_bvh(SSDF_B200_RADIUS_SIG(G, T), SSDF_B200_RADIUS_TAIL(G, T),
                              T *const SSDF_RESTRICT closest_x, T *const SSDF_RESTRICT closest_y,
                              T *const SSDF_RESTRICT closest_z, const bool skip_self = false) {
    SSDF_B200_RADIUS_DISPATCH(closest_within_radius_bvh, npoints, x, y, z, nselements, s0, s1, s2, nspoints, sx, sy,
                              sz, radius_stride, radius_squared, outtri, out_sqr_dist, closest_x, closest_y, closest_z,
                              skip_self ? 1 : 0);
}

template <typename G, typename T, typename I>
int closest_within_radius_local_bvh(SSDF_B200_RADIUS_SIG(G, T), SSDF_B200_RADIUS_TAIL(G, T),
                                    T *const SSDF_RESTRICT closest_s, T *const SSDF_RESTRICT closest_t,
                                    const bool skip_self = false) {
    SSDF_B200_RADIUS_DISPATCH(closest_within_radius_local_bvh, npoints, x, y, z, nselements, s0, s1, s2, nspoints, sx,
                              sy, sz, radius_stride, radius_squared, outtri, out_sqr_dist, closest_s, closest_t,
                              skip_self ? 1 : 0);
}

template <typename G, typename T, typename I>
int closest_within_radius_quads_bvh(SSDF_B200_RADIUS_SIG(G, T), const I *const SSDF_RESTRICT s3,
                                    SSDF_B200_RADIUS_TAIL(G, T), T *const SSDF_RESTRICT closest_x,
                                    T *const SSDF_RESTRICT closest_y, T *const SSDF_RESTRICT closest_z,
                                    const bool skip_self = false) {
    SSDF_B200_RADIUS_DISPATCH(closest_within_radius_quads_bvh, npoints, x, y, z, nselements, s0, s1, s2, s3, nspoints,
                              sx, sy, sz, radius_stride, radius_squared, outtri, out_sqr_dist, closest_x, closest_y,
                              closest_z, skip_self ? 1 : 0);
}

template <typename G, typename T, typename I>
int closest_within_radius_quads_local_bvh(SSDF_B200_RADIUS_SIG(G, T), const I *const SSDF_RESTRICT s3,
                                          SSDF_B200_RADIUS_TAIL(G, T), T *const SSDF_RESTRICT closest_s,
                                          T *const SSDF_RESTRICT closest_t, const bool skip_self = false) {
    SSDF_B200_RADIUS_DISPATCH(closest_within_radius_quads_local_bvh, npoints, x, y, z, nselements, s0, s1, s2, s3,
                              nspoints, sx, sy, sz, radius_stride, radius_squared, outtri, out_sqr_dist, closest_s,
                              closest_t, skip_self ? 1 : 0);
}

// serial/bvh/bvh.hpp:156-181: candidate contact pairs, CSR with a malloc'd index array.
// Instantiations <float, float, int, int>, <double, double, int, int> (serial/bvh/bvh.cpp:1524-1572).
template <typename G, typename T, typename I, typename F>
int potential_contact_triangles_bvh(const ptrdiff_t nselements, const I *const SSDF_RESTRICT s0,
                                    const I *const SSDF_RESTRICT s1, const I *const SSDF_RESTRICT s2,
                                    const ptrdiff_t nspoints, const G *const SSDF_RESTRICT sx,
                                    const G *const SSDF_RESTRICT sy, const G *const SSDF_RESTRICT sz, const T extrusion,
                                    ptrdiff_t *const SSDF_RESTRICT pc_ptr, F **const SSDF_RESTRICT out_pc_idx) {
    static_assert(std::is_same<I, int>::value && std::is_same<F, int>::value, "ssdf_b200 indices are int");
    if constexpr (std::is_same<G, float>::value && std::is_same<T, float>::value)
        return ssdf_b200_potential_contact_triangles_bvh_ff(nselements, s0, s1, s2, nspoints, sx, sy, sz, extrusion,
                                                            pc_ptr, out_pc_idx);
    else if constexpr (std::is_same<G, double>::value && std::is_same<T, double>::value)
        return ssdf_b200_potential_contact_triangles_bvh_dd(nselements, s0, s1, s2, nspoints, sx, sy, sz, extrusion,
                                                            pc_ptr, out_pc_idx);
    else
        static_assert(detail::always_false<G, T>::value, "potential_contact_triangles_bvh: <float,float>, <double,double>");
}

template <typename G, typename T, typename I, typename F>
int potential_contact_quads_bvh(const ptrdiff_t nselements, const I *const SSDF_RESTRICT s0,
                                const I *const SSDF_RESTRICT s1, const I *const SSDF_RESTRICT s2,
                                const I *const SSDF_RESTRICT s3, const ptrdiff_t nspoints,
                                const G *const SSDF_RESTRICT sx, const G *const SSDF_RESTRICT sy,
                                const G *const SSDF_RESTRICT sz, const T extrusion, ptrdiff_t *const SSDF_RESTRICT pc_ptr,
                                F **const SSDF_RESTRICT out_pc_idx) {
    static_assert(std::is_same<I, int>::value && std::is_same<F, int>::value, "ssdf_b200 indices are int");
    if constexpr (std::is_same<G, float>::value && std::is_same<T, float>::value)
        return ssdf_b200_potential_contact_quads_bvh_ff(nselements, s0, s1, s2, s3, nspoints, sx, sy, sz, extrusion,
                                                        pc_ptr, out_pc_idx);
    else if constexpr (std::is_same<G, double>::value && std::is_same<T, double>::value)
        return ssdf_b200_potential_contact_quads_bvh_dd(nselements, s0, s1, s2, s3, nspoints, sx, sy, sz, extrusion,
                                                        pc_ptr, out_pc_idx);
    else
        static_assert(detail::always_false<G, T>::value, "potential_contact_quads_bvh: <float,float>, <double,double>");
}

}  // namespace ssdf

#endif  // SSDF_B200_SSDF_HPP
