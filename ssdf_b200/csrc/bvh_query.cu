// bvh_query.cu -- closest-triangle queries over the device BVH.
//
// Stands in for the reference's device query (serial/bvh/bvh.cu:60-76 + cuBQL CPAT) and its CPU
// grid samplers (serial/bvh/bvh.cpp:1574-1798). Three arithmetics (SSDF_PREC_*):
//   F64   double nodes and triangles, the reference's exact double expression; lexicographic
//         (d^2, triangle index) minimum: bitwise the reference's double value;
//   F32   the same over float nodes/triangles with the reference's float expression (its
//         edf<float> value);
//   F32X  float traversal with fused multiply-adds keeps the K smallest float d^2 inside a
//         window (sqrt(best) + tau)^2; the window's members are re-evaluated in double and the
//         lexicographic minimum taken. tau bounds twice the float error of one distance, so the
//         double winner is always in the window; a query whose window overflowed the K slots is
//         walked again with the window fixed, re-evaluating every member in double (k_window, a
//         warp per query).
//         Result: bitwise the F64 result.
// Traversal: nearest child first, the farther one pushed with its box distance on a per-lane stack
// and culled on pop against the current thresholds. Each lane answers kQ queries (a build option;
// 1 by default, 2 measured no faster: it shares each node and triangle load between two chains of
// arithmetic but costs the registers of the second). Grid queries map a
// warp to a 4 x 4 x 2kQ brick of nodes, so the warp's traversals stay coherent; by default a grid
// warp walks the tree as one packet.
// Outputs (SSDF_OUT_*): in/out distance (edf), in/out squared distance (sqedf), signed distance
// with the pseudo-normal rule of serial/bvh/bvh.cpp:1751-1792, closest point + triangle
// (closest_point_bvh, serial/bvh/bvh.cpp:178-194).
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>

#include "device_geom.cuh"
#include "internal.h"

namespace ssdf_b200 {

namespace {

constexpr int kThreads = 128;
// F32X window slots: candidates kept per query in shared memory. A window that overflows them sends
// its query to the second stage (k_window). On the torus-knot 256^3 grid: 8 slots overflow 0.72% of
// the queries (22.9 ms), 12 slots 0.01% (21.6 ms), 16 slots none (23.2 ms: the longer insertion).
#ifndef SSDF_B200_WINDOW_SLOTS
#define SSDF_B200_WINDOW_SLOTS 12
#endif
constexpr int kCand = SSDF_B200_WINDOW_SLOTS;

// Minimum resident blocks per SM the float query kernels are compiled for: 10 blocks of 128 cap
// them at 48 registers (the fix-up window lives in shared memory). The traversal is issue-latency
// bound, so the occupancy this buys outweighs the spills (measured on the torus-knot grid with the
// packed box test: 16.79 ms against 17.22 ms for 9 blocks at 56 registers, 17.72 ms for 8 at 64 and
// 16.77 ms for 11 at 40); the double kernel keeps its registers.
#ifndef SSDF_B200_QUERY_MIN_BLOCKS
#define SSDF_B200_QUERY_MIN_BLOCKS 10
#endif

// The double kernel keeps 5 resident blocks per SM (at most 102 registers), its occupancy before the
// seeded column walk added a few live values.
constexpr int kF64MinBlocks = 5;

struct Counters {
    unsigned long long tri = 0, box = 0, fix = 0;
};

__device__ __forceinline__ double dinf() { return __longlong_as_double(0x7ff0000000000000ll); }
__device__ __forceinline__ float finf() { return __int_as_float(0x7f800000); }

// ---- query mapping ------------------------------------------------------------------------------

// Each lane answers kQ queries. Grid: a block covers an 8 (x) x 4 (y) column of nodes and, at step
// `step`, the 4 kQ z-planes from (column * grid_steps + step) * 4 kQ on; a warp takes a 4 x 4 x 2kQ
// brick of them, lane (lx, ly, lz) kQ consecutive z nodes. Point lists: query
// (block * kQ + s) * 128 + thread, so each of a lane's queries is a coalesced load.
__device__ __forceinline__ bool map_query(const QueryArgs &a, long long b, int step, int s, long long &q,
                                          long long &i, long long &j, long long &k) {
    if (!a.is_grid) {
        const long long slot = (b * kQ + s) * kThreads + threadIdx.x;
        if (slot >= a.npoints) return false;
        q = a.order ? (long long)__ldg(a.order + slot) : slot;
        return true;
    }
    const long long bxn = grid_blocks_x(a.nx), byn = grid_blocks_y(a.ny);
    const long long bx = b % bxn, r = b / bxn;
    const long long by = r % byn, bz = r / byn;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    i = bx * 8 + (warp & 1) * 4 + (lane & 3);
    j = by * 4 + ((lane >> 2) & 3);
    k = (((bz * a.grid_steps + step) * 4 + (warp >> 1) * 2) + (lane >> 4)) * kQ + s;
    q = i + a.nx * (j + a.ny * k);
    return i < a.nx && j < a.ny && k < a.nz;
}

__device__ __forceinline__ void grid_ijk(const QueryArgs &a, long long q, long long &i, long long &j, long long &k) {
    i = q % a.nx;
    const long long r = q / a.nx;
    j = r % a.ny;
    k = r / a.ny;
}

__device__ __forceinline__ void query_point(const QueryArgs &a, long long q, long long i, long long j, long long k,
                                            double &x, double &y, double &z) {
    if (a.is_grid) {
        if (a.coord_f64) {
            x = grid_coord<double>(a.lo64[0], a.h64[0], i);
            y = grid_coord<double>(a.lo64[1], a.h64[1], j);
            z = grid_coord<double>(a.lo64[2], a.h64[2], k + a.z0);
        } else {
            x = grid_coord<float>(a.lo32[0], a.h32[0], i);
            y = grid_coord<float>(a.lo32[1], a.h32[1], j);
            z = grid_coord<float>(a.lo32[2], a.h32[2], k + a.z0);
        }
    } else if (a.coord_f64) {
        x = __ldg((const double *)a.x + q);
        y = __ldg((const double *)a.y + q);
        z = __ldg((const double *)a.z + q);
    } else {
        x = double(__ldg((const float *)a.x + q));
        y = double(__ldg((const float *)a.y + q));
        z = double(__ldg((const float *)a.z + q));
    }
}

__device__ __forceinline__ double load_out(const QueryArgs &a, long long q) {
    return a.out_f64 ? ((const double *)a.out)[q] : double(((const float *)a.out)[q]);
}
__device__ __forceinline__ void store_out(const QueryArgs &a, long long q, double v) {
    if (a.out_f64)
        ((double *)a.out)[q] = v;
    else
        ((float *)a.out)[q] = float(v);
}

// ---- node and triangle loads ----------------------------------------------------------------------

struct Node32 {
    float4 a, b, c;
    int r0, r1;
};
__device__ __forceinline__ Node32 load_node32(const float4 *__restrict__ nodes, int n) {
    Node32 o;
    o.a = __ldg(nodes + 4 * n);
    o.b = __ldg(nodes + 4 * n + 1);
    o.c = __ldg(nodes + 4 * n + 2);
    const float4 d = __ldg(nodes + 4 * n + 3);
    o.r0 = __float_as_int(d.x);
    o.r1 = __float_as_int(d.y);
    return o;
}

struct Node64 {
    double2 x0, y0, z0, x1, y1, z1;
    int r0, r1;
};
__device__ __forceinline__ Node64 load_node64(const double2 *__restrict__ nodes, int n) {
    Node64 o;
    const double2 *p = nodes + 8 * n;
    o.x0 = __ldg(p);
    o.y0 = __ldg(p + 1);
    o.z0 = __ldg(p + 2);
    o.x1 = __ldg(p + 3);
    o.y1 = __ldg(p + 4);
    o.z1 = __ldg(p + 5);
    const double2 r = __ldg(p + 6);
    o.r0 = int((unsigned)__double_as_longlong(r.x));
    o.r1 = int((unsigned)__double_as_longlong(r.y));
    return o;
}

// 4-wide node: per child c, box (lox, hix, loy, hiy, loz, hiz)[c] and reference r[c].
template <typename T>
__device__ __forceinline__ void boxes4_exact(const DeviceMesh &m, int node, T px, T py, T pz, T (&d)[4], int (&r)[4]);

template <>
__device__ __forceinline__ void boxes4_exact<float>(const DeviceMesh &m, int node, float px, float py, float pz,
                                                    float (&d)[4], int (&r)[4]) {
    const float4 *p = m.nodes4_32 + 8 * node;
    const float4 lx = __ldg(p), hx = __ldg(p + 1), ly = __ldg(p + 2), hy = __ldg(p + 3), lz = __ldg(p + 4),
                 hz = __ldg(p + 5), rr = __ldg(p + 6);
    d[0] = box_dist_sq<float>(px, py, pz, lx.x, hx.x, ly.x, hy.x, lz.x, hz.x);
    d[1] = box_dist_sq<float>(px, py, pz, lx.y, hx.y, ly.y, hy.y, lz.y, hz.y);
    d[2] = box_dist_sq<float>(px, py, pz, lx.z, hx.z, ly.z, hy.z, lz.z, hz.z);
    d[3] = box_dist_sq<float>(px, py, pz, lx.w, hx.w, ly.w, hy.w, lz.w, hz.w);
    r[0] = __float_as_int(rr.x), r[1] = __float_as_int(rr.y), r[2] = __float_as_int(rr.z), r[3] = __float_as_int(rr.w);
}

template <>
__device__ __forceinline__ void boxes4_exact<double>(const DeviceMesh &m, int node, double px, double py, double pz,
                                                     double (&d)[4], int (&r)[4]) {
    const double2 *p = m.nodes4_64 + 14 * node;
    double2 row[12];
#pragma unroll
    for (int k = 0; k < 12; k++) row[k] = __ldg(p + k);
    const double2 rr = __ldg(p + 12);
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int h = c >> 1;
        auto pick = [&](int rw) { return (c & 1) ? row[2 * rw + h].y : row[2 * rw + h].x; };
        d[c] = box_dist_sq<double>(px, py, pz, pick(0), pick(1), pick(2), pick(3), pick(4), pick(5));
    }
    const unsigned long long a = (unsigned long long)__double_as_longlong(rr.x);
    const unsigned long long b = (unsigned long long)__double_as_longlong(rr.y);
    r[0] = int(unsigned(a)), r[1] = int(unsigned(a >> 32)), r[2] = int(unsigned(b)), r[3] = int(unsigned(b >> 32));
}

// box_dist_sq_fast of both children of a node at once, bit for bit: the clamps per child, the
// differences and the squared norms as packed FP32 pairs (child 0, child 1) of sm_100's
// two-wide FP32 instructions (__fadd2_rn, __fmul2_rn and __ffma2_rn round each half as the scalar
// operation does). One node visit issues 18 instructions for the two boxes instead of 24.
__device__ __forceinline__ float2 box_dist_sq_pair(const float px, const float py, const float pz, const Node32 &n) {
    const float2 dx = __fadd2_rn(make_float2(px, px), make_float2(-fminf(fmaxf(px, n.a.x), n.a.y),
                                                                  -fminf(fmaxf(px, n.b.x), n.b.y)));
    const float2 dy = __fadd2_rn(make_float2(py, py), make_float2(-fminf(fmaxf(py, n.a.z), n.a.w),
                                                                  -fminf(fmaxf(py, n.b.z), n.b.w)));
    const float2 dz = __fadd2_rn(make_float2(pz, pz), make_float2(-fminf(fmaxf(pz, n.c.x), n.c.y),
                                                                  -fminf(fmaxf(pz, n.c.z), n.c.w)));
    return __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
}

// The 4-wide node's child-box distances (box_dist_sq_fast's, bit for bit), children (0, 1) and (2, 3)
// as packed FP32 pairs.
__device__ __forceinline__ void boxes4_pair(const DeviceMesh &m, int node, float px, float py, float pz,
                                            float (&d)[4], int (&r)[4]) {
    const float4 *p = m.nodes4_32 + 8 * node;
    const float4 lx = __ldg(p), hx = __ldg(p + 1), ly = __ldg(p + 2), hy = __ldg(p + 3), lz = __ldg(p + 4),
                 hz = __ldg(p + 5), rr = __ldg(p + 6);
    const float2 x2 = make_float2(px, px), y2 = make_float2(py, py), z2 = make_float2(pz, pz);
    const float2 dx01 = __fadd2_rn(x2, make_float2(-fminf(fmaxf(px, lx.x), hx.x), -fminf(fmaxf(px, lx.y), hx.y)));
    const float2 dy01 = __fadd2_rn(y2, make_float2(-fminf(fmaxf(py, ly.x), hy.x), -fminf(fmaxf(py, ly.y), hy.y)));
    const float2 dz01 = __fadd2_rn(z2, make_float2(-fminf(fmaxf(pz, lz.x), hz.x), -fminf(fmaxf(pz, lz.y), hz.y)));
    const float2 dx23 = __fadd2_rn(x2, make_float2(-fminf(fmaxf(px, lx.z), hx.z), -fminf(fmaxf(px, lx.w), hx.w)));
    const float2 dy23 = __fadd2_rn(y2, make_float2(-fminf(fmaxf(py, ly.z), hy.z), -fminf(fmaxf(py, ly.w), hy.w)));
    const float2 dz23 = __fadd2_rn(z2, make_float2(-fminf(fmaxf(pz, lz.z), hz.z), -fminf(fmaxf(pz, lz.w), hz.w)));
    const float2 s01 = __ffma2_rn(dx01, dx01, __ffma2_rn(dy01, dy01, __fmul2_rn(dz01, dz01)));
    const float2 s23 = __ffma2_rn(dx23, dx23, __ffma2_rn(dy23, dy23, __fmul2_rn(dz23, dz23)));
    d[0] = s01.x, d[1] = s01.y, d[2] = s23.x, d[3] = s23.y;
    r[0] = __float_as_int(rr.x), r[1] = __float_as_int(rr.y), r[2] = __float_as_int(rr.z), r[3] = __float_as_int(rr.w);
}

struct Tri32 {
    float ax, ay, az, bx, by, bz, cx, cy, cz;
    int id;
};

// The fix-up filter's record of leaf position p (DeviceMesh::filt32, 3 x float4): the precomputed
// triangle (or proxy, the sign bit of its ab.ab set).
__device__ __forceinline__ FiltRec load_filt(const float4 *__restrict__ f, int p) {
    const float4 u = __ldg(f + 3 * p), v = __ldg(f + 3 * p + 1), w = __ldg(f + 3 * p + 2);
    const float pen = (__float_as_uint(u.w) >> 31) ? __int_as_float(0x7f800000) : 0.f;
    return FiltRec{u.x, u.y, u.z, v.x, v.y, v.z, w.x, w.y, w.z, fabsf(u.w), v.w, w.w, pen};
}
__device__ __forceinline__ Tri32 load_tri32(const float4 *__restrict__ t, int p) {
    const float4 u = __ldg(t + 3 * p), v = __ldg(t + 3 * p + 1), w = __ldg(t + 3 * p + 2);
    return Tri32{u.x, u.y, u.z, u.w, v.x, v.y, v.z, v.w, w.x, __float_as_int(w.y)};
}

struct Tri64 {
    double ax, ay, az, bx, by, bz, cx, cy, cz;
    int id;
};
__device__ __forceinline__ Tri64 load_tri64(const double2 *__restrict__ t, int p) {
    const double2 *r = t + 5 * p;
    const double2 u = __ldg(r), v = __ldg(r + 1), w = __ldg(r + 2), x = __ldg(r + 3), y = __ldg(r + 4);
    return Tri64{u.x, u.y, v.x, v.y, w.x, w.y, x.x, x.y, y.x, int(y.y)};
}

// ---- traversal policies ---------------------------------------------------------------------------
//
// A policy owns a lane's kQ queries (points, incumbents, prune thresholds `thr`) and knows how to
// test a node's child boxes and a leaf's triangles in its arithmetic. A node or leaf is wanted by a
// lane when any of its queries wants it (`want` returns the per-query mask); a pushed node keeps the
// smallest of its queries' box distances and is entered on pop while that is below the largest
// threshold (conservative for every query of the lane).

template <typename T>
struct ExactData;
template <>
struct ExactData<double> {
    using Tri = Tri64;
    static constexpr double rel = 1.0 + 1.0 / 65536.0;
    static __device__ __forceinline__ double abs_margin(float scale) {
        const double s = double(scale) * 0x1p-40;
        return s * s;
    }
    static __device__ __forceinline__ Node64 node(const DeviceMesh &m, int n) { return load_node64(m.nodes64, n); }
    static __device__ __forceinline__ void boxes(const Node64 &n, double px, double py, double pz, double &d0,
                                                 double &d1) {
        d0 = box_dist_sq<double>(px, py, pz, n.x0.x, n.x0.y, n.y0.x, n.y0.y, n.z0.x, n.z0.y);
        d1 = box_dist_sq<double>(px, py, pz, n.x1.x, n.x1.y, n.y1.x, n.y1.y, n.z1.x, n.z1.y);
    }
    static __device__ __forceinline__ Tri tri(const DeviceMesh &m, int pos) { return load_tri64(m.tris64, pos); }
};
template <>
struct ExactData<float> {
    using Tri = Tri32;
    static constexpr float rel = 1.0f + 1.0f / 65536.0f;
    static __device__ __forceinline__ float abs_margin(float scale) {
        const float s = scale * 0x1p-16f;
        return s * s;
    }
    static __device__ __forceinline__ Node32 node(const DeviceMesh &m, int n) { return load_node32(m.nodes32, n); }
    static __device__ __forceinline__ void boxes(const Node32 &n, float px, float py, float pz, float &d0, float &d1) {
        d0 = box_dist_sq<float>(px, py, pz, n.a.x, n.a.y, n.a.z, n.a.w, n.c.x, n.c.y);
        d1 = box_dist_sq<float>(px, py, pz, n.b.x, n.b.y, n.b.z, n.b.w, n.c.z, n.c.w);
    }
    static __device__ __forceinline__ Tri tri(const DeviceMesh &m, int pos) { return load_tri32(m.tris32, pos); }
};

// Lexicographic (d^2, id) minimum over all triangles, starting from (best, -1): a triangle replaces
// the incumbent if strictly closer, or equally close with a lower index (never the initial bound on
// a tie). Boxes are kept while their distance is below best * (1 + 2^-16) + margin, so rounding in
// box distances never drops a tie.
template <typename T, int Q>
struct ExactPolicy {
    using R = T;
    static constexpr int kQn = Q;
    const DeviceMesh &m;
    T px[Q], py[Q], pz[Q], best[Q], thr[Q];
    int bid[Q], bpos[Q];
    T margin;
    __device__ explicit ExactPolicy(const DeviceMesh &mesh) : m(mesh) {
        margin = ExactData<T>::abs_margin(m.coord_scale);
    }
    __device__ __forceinline__ void set(int q, T x, T y, T z, T init) {
        px[q] = x, py[q] = y, pz[q] = z, best[q] = init, bid[q] = -1, bpos[q] = -1;
        thr[q] = init * ExactData<T>::rel + margin;
    }
    __device__ __forceinline__ void disable(int q) {
        px[q] = py[q] = pz[q] = T(0), best[q] = T(0), bid[q] = -1, bpos[q] = -1;
        thr[q] = T(-1);
    }
    // Starts query q from the triangle at leaf position pos, as if the walk had tested it first (it
    // replaces the incoming bound only when strictly closer; the walk meets it again without effect).
    __device__ __forceinline__ void seed(int q, int pos) {
        const auto t = ExactData<T>::tri(m, pos);
        const T d2 = tri_dist_sq_exact<T>(px[q], py[q], pz[q], t.ax, t.ay, t.az, t.bx, t.by, t.bz, t.cx, t.cy, t.cz);
        if (d2 < best[q]) {
            best[q] = d2;
            bid[q] = t.id;
            bpos[q] = pos;
            thr[q] = best[q] * ExactData<T>::rel + margin;
        }
    }
    __device__ __forceinline__ void boxes(int node, T (&d0)[Q], T (&d1)[Q], int &r0, int &r1) const {
        const auto n = ExactData<T>::node(m, node);
#pragma unroll
        for (int q = 0; q < Q; q++) ExactData<T>::boxes(n, px[q], py[q], pz[q], d0[q], d1[q]);
        r0 = n.r0;
        r1 = n.r1;
    }
    __device__ __forceinline__ void boxes4(int node, T (&d)[4][Q], int (&r)[4]) const {
#pragma unroll
        for (int q = 0; q < Q; q++) {
            T dq[4];
            boxes4_exact<T>(m, node, px[q], py[q], pz[q], dq, r);
#pragma unroll
            for (int c = 0; c < 4; c++) d[c][q] = dq[c];
        }
    }
    __device__ __forceinline__ T max_thr() const {
        T t = thr[0];
#pragma unroll
        for (int q = 1; q < Q; q++) t = t > thr[q] ? t : thr[q];
        return t;
    }
    template <bool COUNT>
    __device__ __forceinline__ void leaf(int first, int n, unsigned mask, Counters &cnt) {
        for (int k = 0; k < n; k++) {
            const auto t = ExactData<T>::tri(m, first + k);
#pragma unroll
            for (int q = 0; q < Q; q++) {
                if (!((mask >> q) & 1u)) continue;
                const T d2 = tri_dist_sq_exact<T>(px[q], py[q], pz[q], t.ax, t.ay, t.az, t.bx, t.by, t.bz, t.cx,
                                                  t.cy, t.cz);
                if (COUNT) cnt.tri++;
                if (d2 < best[q] || (d2 == best[q] && bid[q] >= 0 && t.id < bid[q])) {
                    best[q] = d2;
                    bid[q] = t.id;
                    bpos[q] = first + k;
                    thr[q] = best[q] * ExactData<T>::rel + margin;
                }
            }
        }
    }
};

// F32X: float filter. Per query, the kCand smallest float d^2 inside the window
// (sqrt(best) + tau)^2 are kept, unordered, in shared memory (slot (q, s) of thread t at
// [(q * kCand + s) * kThreads + t]: consecutive threads, consecutive banks), with the smallest d^2
// pushed out of the slots. A candidate is appended to the used slots; only when they are full are
// the entries the shrinking window has left behind dropped (their d^2 is at or above the final
// window, so dropping them loses nothing), and if every slot is still inside the window the largest
// of the kCand + 1 is pushed out. The slots hold the same inside-the-window set as a sorted list
// would, for an append instead of a sorted insertion.
//
// The float filter's error is second order in its error along the triangle's plane, which stays
// small unless the triangle is ill-conditioned (a needle or a
// sliver: the face-region solve divides by its area). Such a triangle is filtered through a
// well-conditioned proxy that contains it (DeviceMesh::filt32): a lower bound of its distance,
// within the float filter's error, which may enter the window but, with its +inf penalty, never
// moves its centre; the member is re-evaluated in double like any other, so the double winner,
// whose key is at most its distance plus that error, stays inside the window.
__device__ __forceinline__ float window_thr(float best, float tau_rel, float scale) {
    if (!(best < finf())) return finf();
    const float d = sqrtf(best);
    const float w = d + tau_rel * (scale + d);
    return w * w * (1.0f + 1.0f / 65536.0f);
}

template <int Q>
struct FastPolicy {
    using R = float;
    static constexpr int kQn = Q;
    static constexpr bool kBudgeted = true;
    const DeviceMesh &m;
    float px[Q], py[Q], pz[Q], best[Q], thr[Q], evicted[Q];
    int used[Q];  // window slots in use
    float tau_rel;
    float *wd;
    int *wp;
    __device__ FastPolicy(const DeviceMesh &mesh, float tau, float *sd, int *sp)
        : m(mesh), tau_rel(tau), wd(sd + threadIdx.x), wp(sp + threadIdx.x) {}
    __device__ __forceinline__ int slot(int q, int s) const { return (q * kCand + s) * kThreads; }
    __device__ __forceinline__ void set(int q, float x, float y, float z, float init) {
        px[q] = x, py[q] = y, pz[q] = z, best[q] = init, evicted[q] = finf(), used[q] = 0;
        thr[q] = window_thr(init, tau_rel, m.coord_scale);
    }
    __device__ __forceinline__ void disable(int q) {
        set(q, 0.f, 0.f, 0.f, finf());
        thr[q] = -1.f;
    }
    // Starts query q's window from the key of the triangle at leaf position pos (not a proxy), as the
    // walk would on meeting it: best is then still the key of a tested triangle, and the walk inserts
    // the triangle when it meets it.
    __device__ __forceinline__ void seed(int q, int pos) {
        const FiltRec t = load_filt(m.filt32, pos);
        const float d2 = tri_dist_sq_filter(px[q], py[q], pz[q], t);
        if (t.pen == 0.f && d2 < best[q]) {
            best[q] = d2;
            thr[q] = window_thr(best[q], tau_rel, m.coord_scale);
        }
    }
    // the walk stops early: every live query goes to the second stage with its current window
    __device__ __forceinline__ void abandon() {
#pragma unroll
        for (int q = 0; q < Q; q++)
            if (thr[q] > 0.f) evicted[q] = 0.f;
    }
    __device__ __forceinline__ void boxes(int node, float (&d0)[Q], float (&d1)[Q], int &r0, int &r1) const {
        const Node32 n = load_node32(m.nodes32, node);
#pragma unroll
        for (int q = 0; q < Q; q++) {
            const float2 d = box_dist_sq_pair(px[q], py[q], pz[q], n);
            d0[q] = d.x;
            d1[q] = d.y;
        }
        r0 = n.r0;
        r1 = n.r1;
    }
    __device__ __forceinline__ void boxes4(int node, float (&d)[4][Q], int (&r)[4]) const {
#pragma unroll
        for (int q = 0; q < Q; q++) {
            float dq[4];
            boxes4_pair(m, node, px[q], py[q], pz[q], dq, r);
#pragma unroll
            for (int c = 0; c < 4; c++) d[c][q] = dq[c];
        }
    }
    __device__ __forceinline__ float max_thr() const {
        float t = thr[0];
#pragma unroll
        for (int q = 1; q < Q; q++) t = fmaxf(t, thr[q]);
        return t;
    }
    __device__ __forceinline__ void insert(int q, float d, int p) {
        if (used[q] < kCand) {
            wd[slot(q, used[q])] = d;
            wp[slot(q, used[q])] = p;
            used[q]++;
            return;
        }
        // full: keep the entries still inside the window, in place
        int w = 0, imax = 0;
        float vmax = -1.f;
        for (int s = 0; s < kCand; s++) {
            const float cur = wd[slot(q, s)];
            if (cur < thr[q]) {
                const int cp = wp[slot(q, s)];
                wd[slot(q, w)] = cur;
                wp[slot(q, w)] = cp;
                if (cur > vmax) vmax = cur, imax = w;
                w++;
            }
        }
        if (w < kCand) {
            wd[slot(q, w)] = d;
            wp[slot(q, w)] = p;
            used[q] = w + 1;
        } else if (d < vmax) {  // every slot inside the window: the largest of the kCand + 1 goes
            evicted[q] = fminf(evicted[q], vmax);
            wd[slot(q, imax)] = d;
            wp[slot(q, imax)] = p;
        } else {
            evicted[q] = fminf(evicted[q], d);
        }
    }
    template <bool COUNT>
    __device__ __forceinline__ void leaf(int first, int n, unsigned mask, Counters &cnt) {
        for (int k = 0; k < n; k++) {
            const FiltRec t = load_filt(m.filt32, first + k);
            const float pen = t.pen;
#pragma unroll
            for (int q = 0; q < Q; q++) {
                if (!((mask >> q) & 1u)) continue;
                const float d2 = tri_dist_sq_filter(px[q], py[q], pz[q], t);
                if (COUNT) cnt.tri++;
                if (d2 < thr[q]) {
                    insert(q, d2, first + k);
                    if (d2 + pen < best[q]) {
                        best[q] = d2;
                        thr[q] = window_thr(best[q], tau_rel, m.coord_scale);
                    }
                }
            }
        }
    }
};

template <class P, int Q = P::kQn>
__device__ __forceinline__ unsigned want_mask(const P &p, const typename P::R (&d)[Q]) {
    unsigned m = 0;
#pragma unroll
    for (int q = 0; q < Q; q++) m |= (d[q] < p.thr[q]) ? (1u << q) : 0u;
    return m;
}

template <typename R, int Q>
__device__ __forceinline__ R min_of(const R (&d)[Q]) {
    R v = d[0];
#pragma unroll
    for (int q = 1; q < Q; q++) v = d[q] < v ? d[q] : v;
    return v;
}

// Stack entries of a packet walk hold a float: distances round down and thresholds up, so the
// float comparison never culls what the exact one would keep.
__device__ __forceinline__ float stack_key_lo(float d) { return d; }
__device__ __forceinline__ float stack_key_lo(double d) { return __double2float_rd(d); }
__device__ __forceinline__ float stack_key_hi(float t) { return t; }
__device__ __forceinline__ float stack_key_hi(double t) { return __double2float_ru(t); }

// Policies that can hand their queries to a second stage (P::kBudgeted) stop a packet's walk after a
// work budget; the others always finish it.
template <class P, class = void>
struct HasBudget : std::false_type {};
template <class P>
struct HasBudget<P, std::void_t<decltype(P::kBudgeted)>> : std::bool_constant<P::kBudgeted> {};
template <class P>
constexpr bool budgeted() {
    return HasBudget<P>::value;
}

constexpr int kRepLane = 21;  // (1, 1, 1) of the 4 x 4 x 2 brick

// Packet walk (a grid warp as one packet): the node ids on the stack are the same in every lane, so
// the warp keeps one stack in shared memory instead of 32 copies in local memory. An entry keeps
// the smallest box distance over the warp's lanes (one redux.sync on the float bits, which order
// like the values for non-negative floats) and is entered on pop while that is below the largest
// lane threshold: a superset of "some lane's distance below its own threshold", so never a miss.
template <bool COUNT, bool BUDGET, class P>
__device__ __forceinline__ void traverse_packet(P &p, Counters &cnt, int budget) {
    using R = typename P::R;
    constexpr int Q = P::kQn;
    constexpr unsigned kAll = 0xffffffffu;
    int work = 0;  // triangle records the packet has tested (the same in every lane; BUDGET only)
    if (budget <= 0) budget = 0x7fffffff;
    __shared__ int s_node[kThreads / 32][kStackSize];
    __shared__ float s_dist[kThreads / 32][kStackSize];
    int *snode = s_node[threadIdx.x >> 5];
    float *sdist = s_dist[threadIdx.x >> 5];
    const bool live = p.max_thr() >= R(0);  // lanes without a query take no part in the keys
    int sp = 0;
    int node = 0;
    while (true) {
        R d0[Q], d1[Q];
        int r0, r1;
        p.boxes(node, d0, d1, r0, r1);
        if (COUNT) cnt.box += 2 * Q;
        R k0 = min_of<R, Q>(d0), k1 = min_of<R, Q>(d1);
        if (__shfl_sync(kAll, k1 < k0, kRepLane)) {  // the nearer child for the brick's centre lane
#pragma unroll
            for (int q = 0; q < Q; q++) {
                const R t = d0[q];
                d0[q] = d1[q];
                d1[q] = t;
            }
            const R tk = k0;
            k0 = k1;
            k1 = tk;
            const int tr = r0;
            r0 = r1;
            r1 = tr;
        }
        int next = -1;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int rc = h ? r1 : r0;
            const unsigned m = rc == kEmptyRef ? 0u : (h ? want_mask(p, d1) : want_mask(p, d0));
            if (!__any_sync(kAll, m != 0u)) continue;
            if (rc < 0) {
                p.template leaf<COUNT>(leaf_first(rc), leaf_count(rc), m, cnt);
                if constexpr (BUDGET && budgeted<P>()) work += leaf_count(rc);
            } else if (next < 0) {
                next = rc;
            } else if (sp < kStackSize) {
                const float key = live ? stack_key_lo(h ? k1 : k0) : finf();
                snode[sp] = rc;  // every lane stores the same values
                sdist[sp] = __uint_as_float(__reduce_min_sync(kAll, __float_as_uint(key)));
                sp++;
            }
        }
        if (next < 0) {
            if constexpr (BUDGET && budgeted<P>()) {
                if (work > budget) {  // warp-uniform; checked where a path ends
                    p.abandon();
                    break;
                }
            }
            const float tl = live ? stack_key_hi(p.max_thr()) : 0.f;
            const float tmax = __uint_as_float(__reduce_max_sync(kAll, __float_as_uint(tl)));
            while (sp > 0) {
                sp--;
                if (sdist[sp] < tmax) {
                    next = snode[sp];
                    break;
                }
            }
            if (next < 0) break;
        }
        node = next;
    }
}

// Nearest-child-first traversal with a per-lane stack of (node, smallest box distance), culled on
// pop. WARP = false: every thread walks its own queries. WARP = true (packet): the 32 lanes of a
// warp walk one path together -- a child is entered if any lane wants it, the nearer child is the
// one the brick's centre lane ranks first (traverse_packet) -- so node and triangle loads are
// warp-uniform (broadcast) and leaf work does not diverge. Every lane must call it
// (warp-synchronous when WARP).
template <bool WARP, bool COUNT, bool BUDGET, class P>
__device__ __forceinline__ void traverse(P &p, Counters &cnt, int budget) {
    if constexpr (WARP) {
        traverse_packet<COUNT, BUDGET>(p, cnt, budget);
        return;
    }
    using R = typename P::R;
    constexpr int Q = P::kQn;
    int snode[kStackSize];
    R sdist[kStackSize];
    int sp = 0;
    int node = 0;
    while (true) {
        R d0[Q], d1[Q];
        int r0, r1;
        p.boxes(node, d0, d1, r0, r1);
        if (COUNT) cnt.box += 2 * Q;
        R k0 = min_of<R, Q>(d0), k1 = min_of<R, Q>(d1);
        const bool swap = WARP ? (__popc(__ballot_sync(0xffffffffu, k1 < k0)) > 16) : (k1 < k0);
        if (swap) {
#pragma unroll
            for (int q = 0; q < Q; q++) {
                const R t = d0[q];
                d0[q] = d1[q];
                d1[q] = t;
            }
            const R tk = k0;
            k0 = k1;
            k1 = tk;
            const int tr = r0;
            r0 = r1;
            r1 = tr;
        }
        int next = -1;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int rc = h ? r1 : r0;
            const unsigned m = rc == kEmptyRef ? 0u : (h ? want_mask(p, d1) : want_mask(p, d0));
            if (WARP ? !__any_sync(0xffffffffu, m != 0u) : m == 0u) continue;
            if (rc < 0) {
                p.template leaf<COUNT>(leaf_first(rc), leaf_count(rc), m, cnt);
            } else if (next < 0) {
                next = rc;
            } else if (sp < kStackSize) {
                snode[sp] = rc;
                sdist[sp] = h ? k1 : k0;
                sp++;
            }
        }
        if (next < 0) {
            const R tmax = p.max_thr();
            while (sp > 0) {
                sp--;
                const bool w = sdist[sp] < tmax;
                if (WARP ? __any_sync(0xffffffffu, w) : w) {
                    next = snode[sp];
                    break;
                }
            }
            if (next < 0) break;
        }
        node = next;
    }
}

// The same over the 4-wide BVH. Children are visited in ascending box distance -- the lane's own
// smallest in thread mode, a representative lane's (the brick centre) in warp mode -- leaves first
// in that order, then the nearest wanted internal child is entered and the others pushed
// farthest-first.

template <typename R, int Q>
__device__ __forceinline__ void cswap4(float (&k)[4], R (&d)[4][Q], int (&r)[4], int i, int j) {
    if (k[j] < k[i]) {
        const float tk = k[i];
        k[i] = k[j];
        k[j] = tk;
#pragma unroll
        for (int q = 0; q < Q; q++) {
            const R td = d[i][q];
            d[i][q] = d[j][q];
            d[j][q] = td;
        }
        const int tr = r[i];
        r[i] = r[j];
        r[j] = tr;
    }
}

template <bool WARP, bool COUNT, class P>
__device__ __forceinline__ void traverse4(P &p, Counters &cnt) {
    using R = typename P::R;
    constexpr int Q = P::kQn;
    int snode[kStackSize];
    R sdist[kStackSize];
    int sp = 0;
    int node = 0;
    while (true) {
        R d[4][Q];
        int r[4];
        p.boxes4(node, d, r);
        if (COUNT) cnt.box += 4 * Q;
        float key[4];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const float own = float(min_of<R, Q>(d[c]));
            key[c] = WARP ? __shfl_sync(0xffffffffu, own, kRepLane) : own;
        }
        cswap4<R, Q>(key, d, r, 0, 1);
        cswap4<R, Q>(key, d, r, 2, 3);
        cswap4<R, Q>(key, d, r, 0, 2);
        cswap4<R, Q>(key, d, r, 1, 3);
        cswap4<R, Q>(key, d, r, 1, 2);
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if (r[c] >= 0 || r[c] == kEmptyRef) continue;
            const unsigned m = want_mask(p, d[c]);
            if (WARP ? !__any_sync(0xffffffffu, m != 0u) : m == 0u) continue;
            p.template leaf<COUNT>(leaf_first(r[c]), leaf_count(r[c]), m, cnt);
        }
        int next = -1;
        R next_d = R(0);
#pragma unroll
        for (int c = 3; c >= 0; c--) {
            if (r[c] < 0) continue;
            const unsigned m = want_mask(p, d[c]);
            if (WARP ? !__any_sync(0xffffffffu, m != 0u) : m == 0u) continue;
            if (next >= 0 && sp < kStackSize) {
                snode[sp] = next;
                sdist[sp] = next_d;
                sp++;
            }
            next = r[c];
            next_d = min_of<R, Q>(d[c]);
        }
        if (next < 0) {
            const R tmax = p.max_thr();
            while (sp > 0) {
                sp--;
                const bool w = sdist[sp] < tmax;
                if (WARP ? __any_sync(0xffffffffu, w) : w) {
                    next = snode[sp];
                    break;
                }
            }
            if (next < 0) break;
        }
        node = next;
    }
}

// Packet walk of the 4-wide BVH, the binary packet walk's rules over four children: a child is
// wanted when any lane wants it; wanted leaves are tested at once; of the wanted internal children
// the one nearest the brick's centre lane is entered and the others go on the warp's shared stack
// with the warp's smallest box distance, entered on pop while that is below the largest lane
// threshold. At most 3 entries a level: the build keeps 3 x (4-wide depth) below kStackSize.
template <bool COUNT, bool BUDGET, class P>
__device__ __forceinline__ void traverse4_packet(P &p, Counters &cnt, int budget) {
    using R = typename P::R;
    constexpr int Q = P::kQn;
    constexpr unsigned kAll = 0xffffffffu;
    int work = 0;
    if (budget <= 0) budget = 0x7fffffff;
    __shared__ int s_node[kThreads / 32][kStackSize];
    __shared__ float s_dist[kThreads / 32][kStackSize];
    int *snode = s_node[threadIdx.x >> 5];
    float *sdist = s_dist[threadIdx.x >> 5];
    const bool live = p.max_thr() >= R(0);
    int sp = 0;
    int node = 0;
    while (true) {
        R d[4][Q];
        int r[4];
        p.boxes4(node, d, r);
        if (COUNT) cnt.box += 4 * Q;
        int next = -1;
        float next_rank = 0.f, next_key = 0.f;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int rc = r[c];
            const unsigned m = rc == kEmptyRef ? 0u : want_mask(p, d[c]);
            if (!__any_sync(kAll, m != 0u)) continue;
            if (rc < 0) {
                p.template leaf<COUNT>(leaf_first(rc), leaf_count(rc), m, cnt);
                if constexpr (BUDGET && budgeted<P>()) work += leaf_count(rc);
                continue;
            }
            const R own = min_of<R, Q>(d[c]);
            const float key =
                __uint_as_float(__reduce_min_sync(kAll, __float_as_uint(live ? stack_key_lo(own) : finf())));
            const float rank = __shfl_sync(kAll, float(own), kRepLane);
            int push = rc;
            float push_key = key;
            if (next < 0 || rank < next_rank) {
                push = next;
                push_key = next_key;
                next = rc;
                next_rank = rank;
                next_key = key;
            }
            if (push >= 0 && sp < kStackSize) {
                snode[sp] = push;  // every lane stores the same values
                sdist[sp] = push_key;
                sp++;
            }
        }
        if (next < 0) {
            if constexpr (BUDGET && budgeted<P>()) {
                if (work > budget) {
                    p.abandon();
                    break;
                }
            }
            const float tl = live ? stack_key_hi(p.max_thr()) : 0.f;
            const float tmax = __uint_as_float(__reduce_max_sync(kAll, __float_as_uint(tl)));
            while (sp > 0) {
                sp--;
                if (sdist[sp] < tmax) {
                    next = snode[sp];
                    break;
                }
            }
            if (next < 0) break;
        }
        node = next;
    }
}

template <bool WARP, bool WIDE, bool COUNT, bool BUDGET = false, class P>
__device__ __forceinline__ void walk(P &p, Counters &cnt, int budget = 0) {
    if constexpr (WIDE && WARP)
        traverse4_packet<COUNT, BUDGET>(p, cnt, budget);
    else if constexpr (WIDE)
        traverse4<WARP, COUNT>(p, cnt);
    else
        traverse<WARP, COUNT, BUDGET>(p, cnt, budget);
}

// ---- outputs ----------------------------------------------------------------------------------------

// Signed distance from the closest triangle (caller's index t, leaf position pos) and d^2, in
// double: the closest point, its barycentric coordinates, the pseudo-normal they select and the
// sign of (q - c) . n (serial/bvh/bvh.cpp:1751-1792, tolerance 1e-4 from bvh.cpp:1738).
__device__ double signed_distance(const DeviceMesh &m, int pos, int t, double qx, double qy, double qz, double d2,
                                  double &cx, double &cy, double &cz) {
    const Tri64 tr = load_tri64(m.tris64, pos);
    tri_closest_point_exact<double>(qx, qy, qz, tr.ax, tr.ay, tr.az, tr.bx, tr.by, tr.bz, tr.cx, tr.cy, tr.cz, cx, cy,
                                    cz);
    const double e1[3] = {tr.bx - tr.ax, tr.by - tr.ay, tr.bz - tr.az};
    const double e2[3] = {tr.cx - tr.ax, tr.cy - tr.ay, tr.cz - tr.az};
    const double r[3] = {cx - tr.ax, cy - tr.ay, cz - tr.az};
    const double d11 = e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2];
    const double d12 = e1[0] * e2[0] + e1[1] * e2[1] + e1[2] * e2[2];
    const double d22 = e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2];
    const double r1 = r[0] * e1[0] + r[1] * e1[1] + r[2] * e1[2];
    const double r2 = r[0] * e2[0] + r[1] * e2[1] + r[2] * e2[2];
    const double det = d11 * d22 - d12 * d12;
    const double l1 = det > 0 ? (d22 * r1 - d12 * r2) / det : 0;
    const double l2 = det > 0 ? (d11 * r2 - d12 * r1) / det : 0;
    const double l[3] = {1 - l1 - l2, l1, l2};
    const double tol = 1e-4;
    int small = 0, last_small = -1, last_large = -1;
#pragma unroll
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
        n = m.face_n + 3 * (size_t)t;
    } else if (small == 1) {
        n = m.edge_n + 9 * (size_t)t + 3 * ((last_small + 1) % 3);
    } else {
        const int *s = last_large == 0 ? m.s0 : (last_large == 1 ? m.s1 : m.s2);
        n = m.vertex_n + 3 * (size_t)__ldg(s + t);
    }
    const double dot = (qx - cx) * __ldg(n) + (qy - cy) * __ldg(n + 1) + (qz - cz) * __ldg(n + 2);
    const double dist = sqrt(d2);
    return dot < 0 ? -dist : dist;
}

// Writes one query's outputs from its double result (best, bid, bpos); `init` is the bound the
// search started from (incoming value for the in/out outputs).
__device__ void write_result(const QueryArgs &a, long long q, double qx, double qy, double qz, double best, int bid,
                             int bpos) {
    switch (a.output) {
        case SSDF_OUT_EDF:
            store_out(a, q, sqrt(best));
            if (a.outtri && bid >= 0) a.outtri[q] = bid;
            break;
        case SSDF_OUT_SQEDF:
            store_out(a, q, best);
            break;
        case SSDF_OUT_SDF: {
            double cx, cy, cz;
            const double v = bid >= 0 ? signed_distance(a.m, bpos, bid, qx, qy, qz, best, cx, cy, cz) : sqrt(best);
            store_out(a, q, v);
            if (a.outtri) a.outtri[q] = bid;
            break;
        }
        case SSDF_OUT_CLOSEST: {
            if (bid < 0) break;
            const double dist = sqrt(best);
            const double din = load_out(a, q);
            const double dist_t = a.out_f64 ? dist : double(float(dist));
            if (din > dist_t) {
                const Tri64 tr = load_tri64(a.m.tris64, bpos);
                double cx, cy, cz;
                tri_closest_point_exact<double>(qx, qy, qz, tr.ax, tr.ay, tr.az, tr.bx, tr.by, tr.bz, tr.cx, tr.cy,
                                                tr.cz, cx, cy, cz);
                store_out(a, q, dist);
                if (a.coord_f64) {
                    ((double *)a.outx)[q] = cx, ((double *)a.outy)[q] = cy, ((double *)a.outz)[q] = cz;
                } else {
                    ((float *)a.outx)[q] = float(cx), ((float *)a.outy)[q] = float(cy), ((float *)a.outz)[q] = float(cz);
                }
                a.outtri[q] = bid;
            }
            break;
        }
        default:
            break;
    }
}

// Incoming bound of the search, as a squared distance in double.
__device__ __forceinline__ double initial_bound(const QueryArgs &a, long long q) {
    switch (a.output) {
        case SSDF_OUT_EDF:
        case SSDF_OUT_CLOSEST: {
            const double o = load_out(a, q);
            return o * o;
        }
        case SSDF_OUT_SQEDF:
            return load_out(a, q);
        default:
            return dinf();
    }
}

__device__ __forceinline__ void flush_counters(const QueryArgs &a, const Counters &c) {
    unsigned long long t = c.tri, b = c.box, f = c.fix;
    for (int o = 16; o > 0; o >>= 1) {
        t += __shfl_xor_sync(0xffffffffu, t, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
        f += __shfl_xor_sync(0xffffffffu, f, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(a.counters + 0, t);
        atomicAdd(a.counters + 1, b);
        atomicAdd(a.counters + 2, f);
    }
}

// ---- kernels ----------------------------------------------------------------------------------------

// Streamed download: the block's results are stored; the last block of its chunk to finish tells the
// host, which copies the chunk out while the launch goes on. Every thread fences its own stores
// before the block counts itself, and the last block fences at system scope before the flag.
__device__ __forceinline__ void signal_chunk(const QueryArgs &a) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned c = blockIdx.x / unsigned(a.chunk_blocks);
        const unsigned members = min(unsigned(a.chunk_blocks), gridDim.x - c * unsigned(a.chunk_blocks));
        if (atomicAdd(a.chunk_counts + c, 1) == int(members) - 1) {
            __threadfence_system();
            *(volatile int *)(a.chunk_flags + c) = 1;
        }
    }
}

// One block of 128 lanes x kQ queries: a point-list block, or one step of a grid block's column.
// Lanes without a query (the edge of a grid brick, the tail of a point list) take part in warp-mode
// traversal with a negative threshold, so they never ask for a node. seed[s] is the leaf position of
// the closest triangle the lane's query s found one step below (-1: none); it is updated here.
template <int PREC, bool WARP, bool WIDE, bool COUNT, bool BUDGET>
__device__ __forceinline__ void query_step(const QueryArgs &a, int step, const bool (&valid)[kQ],
                                           const long long (&qid)[kQ], const long long (&gi)[kQ],
                                           const long long (&gj)[kQ], const long long (&gk)[kQ], bool any,
                                           int (&seed)[kQ], Counters &cnt) {
    constexpr int Q = kQ;
    const bool seeded = a.seed != 0 && step > 0;
    if (PREC == SSDF_PREC_F64) {
        ExactPolicy<double, Q> p(a.m);
#pragma unroll
        for (int s = 0; s < Q; s++) {
            if (valid[s]) {
                double x, y, z;
                query_point(a, qid[s], gi[s], gj[s], gk[s], x, y, z);
                p.set(s, x, y, z, initial_bound(a, qid[s]));
                if (seeded && seed[s] >= 0) p.seed(s, seed[s]);
            } else {
                p.disable(s);
            }
        }
        if (WARP || any) walk<WARP, WIDE, COUNT>(p, cnt);
#pragma unroll
        for (int s = 0; s < Q; s++) {
            if (!valid[s]) continue;
            write_result(a, qid[s], p.px[s], p.py[s], p.pz[s], p.best[s], p.bid[s], p.bpos[s]);
            if (p.bpos[s] >= 0) seed[s] = p.bpos[s];
        }
    } else if (PREC == SSDF_PREC_F32) {
        // the reference's float arithmetic end to end (edf<float>'s value); edf and sqedf outputs
        ExactPolicy<float, Q> p(a.m);
#pragma unroll
        for (int s = 0; s < Q; s++) {
            if (valid[s]) {
                double x, y, z;
                query_point(a, qid[s], gi[s], gj[s], gk[s], x, y, z);
                const long long q = qid[s];
                const float o = a.out_f64 ? float(((const double *)a.out)[q]) : ((const float *)a.out)[q];
                p.set(s, float(x), float(y), float(z), a.output == SSDF_OUT_SQEDF ? o : o * o);
                if (seeded && seed[s] >= 0) p.seed(s, seed[s]);
            } else {
                p.disable(s);
            }
        }
        if (WARP || any) walk<WARP, WIDE, COUNT>(p, cnt);
#pragma unroll
        for (int s = 0; s < Q; s++) {
            if (!valid[s]) continue;
            const long long q = qid[s];
            if (a.output == SSDF_OUT_SQEDF) {
                store_out(a, q, double(p.best[s]));
            } else {
                store_out(a, q, double(sqrtf(p.best[s])));
                if (a.outtri && p.bid[s] >= 0) a.outtri[q] = p.bid[s];
            }
            if (p.bpos[s] >= 0) seed[s] = p.bpos[s];
        }
    } else {
        __shared__ float s_wd[kQ * kCand * kThreads];
        __shared__ int s_wp[kQ * kCand * kThreads];
        FastPolicy<Q> p(a.m, a.tau_rel, s_wd, s_wp);
        bool exact[Q];  // a finite point beyond the float filter's range: the second stage, exactly
#pragma unroll
        for (int s = 0; s < Q; s++) {
            exact[s] = false;
            if (valid[s]) {
                double x, y, z;
                query_point(a, qid[s], gi[s], gj[s], gk[s], x, y, z);
                const double ax = fabs(x), ay = fabs(y), az = fabs(z);
                exact[s] = (ax > kFilterMaxCoord || ay > kFilterMaxCoord || az > kFilterMaxCoord) &&
                           ax < dinf() && ay < dinf() && az < dinf();
                const double init = initial_bound(a, qid[s]);
                // float start bound rounded up, so no triangle closer in double is cut off
                if (exact[s]) {
                    p.disable(s);
                } else {
                    p.set(s, float(x), float(y), float(z), init < dinf() ? __double2float_ru(init) : finf());
                    if (seeded && seed[s] >= 0) p.seed(s, seed[s]);
                }
            } else {
                p.disable(s);
            }
        }
        if (WARP || any) walk<WARP, WIDE, COUNT, BUDGET>(p, cnt, a.warp_budget);
#pragma unroll
        for (int s = 0; s < Q; s++) {
            if (!valid[s]) continue;
            const long long q = qid[s];
            if (exact[s] || p.evicted[s] < p.thr[s]) {
                const int slot = atomicAdd(a.fallback_count, 1);
                a.fallback_ids[slot] = int(q);  // q < 2^31 is checked on the host
                a.fallback_thr[slot] = exact[s] ? finf() : p.thr[s];
                continue;
            }
            // the double point and bound are recomputed here rather than kept live through the walk
            double rx, ry, rz;
            query_point(a, q, gi[s], gj[s], gk[s], rx, ry, rz);
            double b = initial_bound(a, q);
            int bid = -1, bpos = -1;
            for (int c = 0; c < p.used[s]; c++) {
                const int ix = p.slot(s, c);
                if (p.wd[ix] < p.thr[s]) {
                    const int pos = p.wp[ix];
                    const Tri64 t = load_tri64(a.m.tris64, pos);
                    const double d2 =
                        tri_dist_sq_exact<double>(rx, ry, rz, t.ax, t.ay, t.az, t.bx, t.by, t.bz, t.cx, t.cy, t.cz);
                    if (COUNT) cnt.fix++;
                    if (d2 < b || (d2 == b && bid >= 0 && t.id < bid)) {
                        b = d2;
                        bid = t.id;
                        bpos = pos;
                    }
                }
            }
            write_result(a, q, rx, ry, rz, b, bid, bpos);
            if (bpos >= 0) seed[s] = bpos;
        }
    }
}

// A point-list block, or a grid block's column step by step (each step seeded from the one below).
template <int PREC, bool WARP, bool WIDE, bool COUNT, bool BUDGET>
__device__ __forceinline__ void query_block(const QueryArgs &a, long long block, Counters &cnt) {
    constexpr int Q = kQ;
    int seed[Q];
#pragma unroll
    for (int s = 0; s < Q; s++) seed[s] = -1;
    const int steps = a.is_grid ? a.grid_steps : 1;
    for (int step = 0; step < steps; step++) {
        long long qid[Q], gi[Q], gj[Q], gk[Q];
        bool valid[Q];
        bool any = false;
#pragma unroll
        for (int s = 0; s < Q; s++) {
            gi[s] = gj[s] = gk[s] = 0;
            valid[s] = map_query(a, block, step, s, qid[s], gi[s], gj[s], gk[s]);
            any |= valid[s];
        }
        // this warp's part of the column has left the grid (higher steps have no node either); a warp
        // decision, not a block one: the warps share nothing, and a block barrier per step made every
        // warp wait for the block's slowest (17 % on the torus knot)
        if (step > 0 && !__any_sync(0xffffffffu, any)) break;
        query_step<PREC, WARP, WIDE, COUNT, BUDGET>(a, step, valid, qid, gi, gj, gk, any, seed, cnt);
    }
}

// BUDGET: the fix-up kernel's packets stop after QueryArgs::warp_budget triangle records (a separate
// instantiation, so the kernels without it compile as if it did not exist).
// SIGNAL: the streamed grid download's instantiation, whose blocks count themselves done per chunk
// (a separate instantiation: the dormant signal code cost the fix-up kernel 3 % where it was merely
// compiled in).
template <int PREC, bool WARP, bool WIDE, bool COUNT, bool BUDGET = false, bool SIGNAL = false>
__global__ void __launch_bounds__(kThreads, PREC == SSDF_PREC_F64 ? kF64MinBlocks : SSDF_B200_QUERY_MIN_BLOCKS)
    k_query(const QueryArgs a) {
    Counters cnt;
    query_block<PREC, WARP, WIDE, COUNT, BUDGET>(a, blockIdx.x, cnt);
    if (COUNT) flush_counters(a, cnt);
    if constexpr (SIGNAL) signal_chunk(a);
}

// ---- second fix-up stage: one warp per overflowed query --------------------------------------------
//
// A query whose window overflowed its slots is walked again from its final window, and a query whose
// packet ran out of budget from the window it had then: every triangle whose float distance is
// inside the window is re-evaluated in double. The window only shrinks (after each step, to what the
// warp's smallest non-proxy key allows, by the first stage's rule), so the visiting order is free,
// and the warp walks the tree breadth-parallel: each step
// the 32 lanes take up to 32 nodes from the warp's shared stack, test their children, run the
// wanted leaves, and push the wanted internal children (ballot-compacted). A lane keeps the
// lexicographic (d^2, index) minimum of the triangles it evaluated (the incoming bound ranks -1, so
// it wins ties, as in the sequential rule) and a warp reduction takes the minimum of those: the
// same value as the sequential walk, since each triangle's double distance does not depend on the
// order. The boxes and the float test are the first stage's, on the binary tree: the double winner
// lies inside the window by the margin tau, so its boxes pass under either arity.
constexpr int kWinStack = 1024;  // node slots of a warp's shared stack
// Blocks per SM of the second stage's grid. Its kernel keeps its registers (116: capping them at 64 or
// 40 spilled the double evaluation and lost 10-100 %), so 4 blocks are resident per SM; a grid of 12
// per SM queues the rest behind them, so a warp takes one query where 4 per SM had each take two or
// three, and blocks that finish early make room. Measured: 64^3 icosphere step 0.487 -> 0.447 ms,
// 20,480-triangle sphere 96^3 1.58 -> 1.44 ms, the serving leg's heaviest grid 8.22 -> 8.03 ms, the
// torus knot unchanged.
#ifndef SSDF_B200_WINDOW_BLOCKS_PER_SM
#define SSDF_B200_WINDOW_BLOCKS_PER_SM 12
#endif
constexpr int kWindowBlocksPerSm = SSDF_B200_WINDOW_BLOCKS_PER_SM;

struct WindowBest {
    double d2;
    int id, pos;
};

// A window of +inf takes every node and triangle, whatever its float key (a query point beyond the
// float filter's range, whose keys may have overflowed, is answered this way: exactly, in double).
__device__ __forceinline__ bool in_window(float key, float thr) { return key < thr || thr == finf(); }

// kbest: the smallest key of a non-proxy triangle the lane has met (the window may shrink to it, as in
// the first stage: any such key bounds the window from below, so the double winner stays inside).
__device__ __forceinline__ void window_leaf(const DeviceMesh &m, int ref, float px, float py, float pz, float thr,
                                            double qx, double qy, double qz, WindowBest &b, Counters &cnt,
                                            bool count, float &kbest) {
    const int first = leaf_first(ref), n = leaf_count(ref);
    for (int k = 0; k < n; k++) {
        const FiltRec r = load_filt(m.filt32, first + k);
        const float f = tri_dist_sq_filter(px, py, pz, r);  // the first stage's key
        if (r.pen == 0.f && f < kbest) kbest = f;
        if (count) cnt.tri++;
        if (in_window(f, thr)) {
            const Tri64 u = load_tri64(m.tris64, first + k);
            const double e2 =
                tri_dist_sq_exact<double>(qx, qy, qz, u.ax, u.ay, u.az, u.bx, u.by, u.bz, u.cx, u.cy, u.cz);
            if (count) cnt.fix++;
            if (e2 < b.d2 || (e2 == b.d2 && u.id < b.id)) b = WindowBest{e2, u.id, first + k};
        }
    }
}

// A lane's own depth-first walk of the subtree under `root` (when the warp's stack is full). Depth
// below kStackSize is checked when the mesh is built, and a depth-first walk that pushes both
// children holds at most depth + 1 entries.
__device__ __noinline__ void window_subtree(const DeviceMesh &m, int root, float px, float py, float pz, float thr,
                                            double qx, double qy, double qz, WindowBest &b, Counters &cnt,
                                            bool count, float &kbest) {
    int st[kStackSize];
    int sp = 0;
    st[sp++] = root;
    while (sp > 0) {
        const Node32 n = load_node32(m.nodes32, st[--sp]);
        const float d0 = box_dist_sq_fast(px, py, pz, n.a.x, n.a.y, n.a.z, n.a.w, n.c.x, n.c.y);
        const float d1 = box_dist_sq_fast(px, py, pz, n.b.x, n.b.y, n.b.z, n.b.w, n.c.z, n.c.w);
        if (count) cnt.box += 2;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int c = h ? n.r1 : n.r0;
            if (c == kEmptyRef || !in_window(h ? d1 : d0, thr)) continue;
            if (c < 0)
                window_leaf(m, c, px, py, pz, thr, qx, qy, qz, b, cnt, count, kbest);
            else if (sp < kStackSize)
                st[sp++] = c;
        }
    }
}

// The whole warp answers overflowed query `idx` of job `a`; lane 0 writes the result.
template <bool COUNT>
__device__ void window_warp(const QueryArgs &a, int idx, int *__restrict__ stack, int cap, Counters &cnt) {
    const unsigned kAll = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const long long q = a.fallback_ids[idx];
    long long i = 0, j = 0, k = 0;
    if (a.is_grid) grid_ijk(a, q, i, j, k);
    double qx, qy, qz;
    query_point(a, q, i, j, k, qx, qy, qz);
    const float px = float(qx), py = float(qy), pz = float(qz);
    float thr = a.fallback_thr[idx];
    const bool shrink = thr < finf();  // an infinite window (a point beyond the float range) stays
    float kbest = finf();
    const DeviceMesh &m = a.m;
    WindowBest b{initial_bound(a, q), -1, -1};
    if (lane == 0) stack[0] = 0;
    int sp = 1;  // warp-uniform
    __syncwarp();
    while (sp > 0) {
        const int take = sp < 32 ? sp : 32;
        const int node = lane < take ? stack[sp - take + lane] : -1;
        sp -= take;
        __syncwarp();  // the slots just read are free for the pushes below
        int c0 = kEmptyRef, c1 = kEmptyRef;
        bool w0 = false, w1 = false;
        if (node >= 0) {
            const Node32 n = load_node32(m.nodes32, node);
            const float d0 = box_dist_sq_fast(px, py, pz, n.a.x, n.a.y, n.a.z, n.a.w, n.c.x, n.c.y);
            const float d1 = box_dist_sq_fast(px, py, pz, n.b.x, n.b.y, n.b.z, n.b.w, n.c.z, n.c.w);
            if (COUNT) cnt.box += 2;
            c0 = n.r0, c1 = n.r1;
            w0 = c0 != kEmptyRef && in_window(d0, thr);
            w1 = c1 != kEmptyRef && in_window(d1, thr);
            if (w0 && c0 < 0) {
                window_leaf(m, c0, px, py, pz, thr, qx, qy, qz, b, cnt, COUNT, kbest);
                w0 = false;
            }
            if (w1 && c1 < 0) {
                window_leaf(m, c1, px, py, pz, thr, qx, qy, qz, b, cnt, COUNT, kbest);
                w1 = false;
            }
        }
        if (shrink) {  // the window the warp's smallest key allows, as the first stage computes it
            const float wb = __uint_as_float(__reduce_min_sync(kAll, __float_as_uint(kbest)));
            thr = fminf(thr, window_thr(wb, a.tau_rel, m.coord_scale));
        }
        const unsigned m0 = __ballot_sync(kAll, w0), m1 = __ballot_sync(kAll, w1);
        const int n0 = __popc(m0), total = n0 + __popc(m1);
        if (sp + total <= cap) {
            const unsigned below = (1u << lane) - 1u;
            if (w0) stack[sp + __popc(m0 & below)] = c0;
            if (w1) stack[sp + n0 + __popc(m1 & below)] = c1;
            sp += total;
        } else {
            if (w0) window_subtree(m, c0, px, py, pz, thr, qx, qy, qz, b, cnt, COUNT, kbest);
            if (w1) window_subtree(m, c1, px, py, pz, thr, qx, qy, qz, b, cnt, COUNT, kbest);
        }
        __syncwarp();
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double od = __shfl_xor_sync(kAll, b.d2, o);
        const int oid = __shfl_xor_sync(kAll, b.id, o), opos = __shfl_xor_sync(kAll, b.pos, o);
        if (od < b.d2 || (od == b.d2 && oid < b.id)) b = WindowBest{od, oid, opos};
    }
    if (lane == 0) write_result(a, q, qx, qy, qz, b.d2, b.id, b.pos);
}

// Overflowed queries of one launch, a warp each. `cap` (<= kWinStack) is the shared stack's usable
// depth: kWinStack, lowered only to test the per-lane subtree walk.
template <bool COUNT>
__global__ void __launch_bounds__(kThreads) k_window(const QueryArgs a, int cap) {
    __shared__ int s_stack[kThreads / 32][kWinStack];
    const int n = *a.fallback_count;
    const int w = (blockIdx.x * kThreads + threadIdx.x) >> 5, nw = (gridDim.x * kThreads) >> 5;
    Counters cnt;
    for (int idx = w; idx < n; idx += nw) window_warp<COUNT>(a, idx, s_stack[threadIdx.x >> 5], cap, cnt);
    if (COUNT) flush_counters(a, cnt);
}

// ---- batches: many (mesh, query set) jobs in one persistent launch -----------------------------------
//
// The job table lives in device memory (BatchHeader + QueryArgs[] + first block of each job), so a
// captured CUDA graph of these two kernels replays for any batch composition without being
// re-instantiated: only the table is rewritten before each replay. Blocks pull work items (one
// 128-query block of one job) from an atomic counter, largest jobs first (the host orders them).

template <int PREC, bool WARP, bool WIDE, bool COUNT, bool BUDGET = false>
__global__ void __launch_bounds__(kThreads, PREC == SSDF_PREC_F64 ? kF64MinBlocks : SSDF_B200_QUERY_MIN_BLOCKS)
    k_query_batch(const BatchHeader *__restrict__ hdr, const QueryArgs *__restrict__ jobs,
                  const long long *__restrict__ first_block, unsigned long long *__restrict__ next_item) {
    __shared__ long long s_item;
    const int njobs = hdr->njobs;
    const long long total = hdr->total_blocks;
    Counters cnt;
    while (true) {
        if (threadIdx.x == 0) s_item = (long long)atomicAdd(next_item, 1ull);
        __syncthreads();
        const long long it = s_item;
        __syncthreads();
        if (it >= total) break;
        int lo = 0, hi = njobs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(first_block + mid) <= it) lo = mid; else hi = mid - 1;
        }
        query_block<PREC, WARP, WIDE, COUNT, BUDGET>(jobs[lo], it - __ldg(first_block + lo), cnt);
    }
    if (COUNT && njobs > 0) flush_counters(jobs[0], cnt);
}

// Overflowed queries of every job: the jobs' lists laid end to end and dealt to the warps in turn,
// so no warp takes the same position of every list.
template <bool COUNT>
__global__ void __launch_bounds__(kThreads) k_window_batch(const BatchHeader *__restrict__ hdr,
                                                           const QueryArgs *__restrict__ jobs, int cap) {
    __shared__ int s_stack[kThreads / 32][kWinStack];
    const int njobs = hdr->njobs;
    const long long w = (blockIdx.x * kThreads + threadIdx.x) >> 5, nw = (gridDim.x * kThreads) >> 5;
    Counters cnt;
    long long base = 0;  // overflowed queries of the jobs before jb
    for (int jb = 0; jb < njobs; jb++) {
        const QueryArgs &a = jobs[jb];
        if (!a.fallback_count) continue;
        const int n = *a.fallback_count;
        for (long long idx = ((w - base) % nw + nw) % nw; idx < n; idx += nw)
            window_warp<COUNT>(a, int(idx), s_stack[threadIdx.x >> 5], cap, cnt);
        base += n;
    }
    if (COUNT && njobs > 0) flush_counters(jobs[0], cnt);
}

// Usable depth of the second stage's shared stack: kWinStack, or SSDF_B200_WINDOW_STACK (1 ..
// kWinStack) to exercise the per-lane subtree walk in tests.
int window_stack_cap() {
    const int v = env_int("SSDF_B200_WINDOW_STACK", kWinStack);
    return v < 1 ? 1 : (v > kWinStack ? kWinStack : v);
}

template <int PREC, bool WARP, bool WIDE>
cudaError_t launch_batch_main(const BatchLaunch &b, bool count, cudaStream_t stream) {
    constexpr bool kCanBudget = PREC == SSDF_PREC_F32_FIXUP && WARP;
    if constexpr (kCanBudget) {
        if (b.budget) {
            if (count)
                k_query_batch<PREC, WARP, WIDE, true, true><<<b.grid, kThreads, 0, stream>>>(b.hdr, b.jobs, b.first_block,
                                                                                            b.next_item);
            else
                k_query_batch<PREC, WARP, WIDE, false, true><<<b.grid, kThreads, 0, stream>>>(b.hdr, b.jobs, b.first_block,
                                                                                             b.next_item);
        }
    }
    if (!kCanBudget || !b.budget) {
        if (count)
            k_query_batch<PREC, WARP, WIDE, true><<<b.grid, kThreads, 0, stream>>>(b.hdr, b.jobs, b.first_block, b.next_item);
        else
            k_query_batch<PREC, WARP, WIDE, false><<<b.grid, kThreads, 0, stream>>>(b.hdr, b.jobs, b.first_block, b.next_item);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || PREC != SSDF_PREC_F32_FIXUP) return e;
    if (count)
        k_window_batch<true><<<kWindowBlocksPerSm * b.sms, kThreads, 0, stream>>>(b.hdr, b.jobs, window_stack_cap());
    else
        k_window_batch<false><<<kWindowBlocksPerSm * b.sms, kThreads, 0, stream>>>(b.hdr, b.jobs, window_stack_cap());
    return cudaGetLastError();
}

template <int PREC>
cudaError_t launch_batch_prec(const BatchLaunch &b, bool count, cudaStream_t stream) {
    if (b.wide)
        return b.warp ? launch_batch_main<PREC, true, true>(b, count, stream)
                      : launch_batch_main<PREC, false, true>(b, count, stream);
    return b.warp ? launch_batch_main<PREC, true, false>(b, count, stream)
                  : launch_batch_main<PREC, false, false>(b, count, stream);
}

template <int PREC, bool WARP, bool WIDE>
int batch_occupancy() {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_query_batch<PREC, WARP, WIDE, false>, kThreads, 0);
    return nb > 0 ? nb : 1;
}

thread_local unsigned long long t_last_counts[4] = {0, 0, 0, 0};

template <int PREC, bool WARP, bool WIDE>
cudaError_t launch_main(const QueryArgs &a, bool count, unsigned nblocks, cudaStream_t stream) {
    if constexpr (PREC == SSDF_PREC_F32_FIXUP && WARP) {
        if (a.warp_budget > 0) {
            if (count)
                k_query<PREC, WARP, WIDE, true, true><<<nblocks, kThreads, 0, stream>>>(a);
            else
                k_query<PREC, WARP, WIDE, false, true><<<nblocks, kThreads, 0, stream>>>(a);
            return cudaGetLastError();
        }
    }
    // a counting or budgeted launch raises no chunk flags: its streamed download copies every chunk
    // once the launch has ended
    if (count)
        k_query<PREC, WARP, WIDE, true><<<nblocks, kThreads, 0, stream>>>(a);
    else if (a.chunk_flags)
        k_query<PREC, WARP, WIDE, false, false, true><<<nblocks, kThreads, 0, stream>>>(a);
    else
        k_query<PREC, WARP, WIDE, false><<<nblocks, kThreads, 0, stream>>>(a);
    return cudaGetLastError();
}

template <int PREC>
cudaError_t launch_prec(const QueryArgs &a, bool warp, bool wide, bool count, unsigned nblocks, cudaStream_t stream) {
    if (wide)
        return warp ? launch_main<PREC, true, true>(a, count, nblocks, stream)
                    : launch_main<PREC, false, true>(a, count, nblocks, stream);
    return warp ? launch_main<PREC, true, false>(a, count, nblocks, stream)
                : launch_main<PREC, false, false>(a, count, nblocks, stream);
}

}  // namespace

void set_last_counts(unsigned long long tri, unsigned long long box, unsigned long long fix,
                     unsigned long long fallback) {
    t_last_counts[0] = tri, t_last_counts[1] = box, t_last_counts[2] = fix, t_last_counts[3] = fallback;
}

int query_counts(int64_t *tri, int64_t *box, int64_t *fix, int64_t *fallback) {
    if (tri) *tri = (int64_t)t_last_counts[0];
    if (box) *box = (int64_t)t_last_counts[1];
    if (fix) *fix = (int64_t)t_last_counts[2];
    if (fallback) *fallback = (int64_t)t_last_counts[3];
    return SSDF_OK;
}

// Traversal mode: SSDF_B200_TRAVERSAL=warp|thread overrides; by default grids (coherent bricks) walk
// in warp packets and point lists thread by thread.
// BVH arity: SSDF_B200_ARITY=2|4; binary by default (measured as fast as 4-wide on the torus knot).
static bool use_wide(const QueryArgs &a) {
    if (a.force_arity) return a.force_arity == 4;
    return env_int("SSDF_B200_ARITY", 2) == 4;
}

static bool use_warp(const QueryArgs &a) {
    if (a.force_traversal) return a.force_traversal == 1;
    const char *v = env_str("SSDF_B200_TRAVERSAL");
    if (v && !strcmp(v, "warp")) return true;
    if (v && !strcmp(v, "thread")) return false;
    return a.is_grid != 0 || a.order != nullptr;  // sorted point lists are coherent enough for packets
}

// Point lists in Morton order: a warp's 32 slots then hold neighbouring points, which the packet walk
// needs (in input order a warp of scattered queries keeps about 5 of its lanes busy). Keys are 30-bit
// Morton codes of the points in the mesh's bounding box (the union of the root's two child boxes),
// points outside it clamped to its faces; the stable radix sort makes the order deterministic.
__global__ void k_point_keys(long long n, const void *__restrict__ x, const void *__restrict__ y,
                             const void *__restrict__ z, int f64, const float4 *__restrict__ root,
                             uint32_t *__restrict__ keys, int *__restrict__ vals) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 c0 = __ldg(root), c1 = __ldg(root + 1), c2 = __ldg(root + 2);
    // child boxes: (lox, hix, loy, hiy) of each, then (loz, hiz) of both; an empty child is inverted
    const float lo[3] = {fminf(c0.x, c1.x), fminf(c0.z, c1.z), fminf(c2.x, c2.z)};
    const float hi[3] = {fmaxf(c0.y, c1.y), fmaxf(c0.w, c1.w), fmaxf(c2.y, c2.w)};
    const float p[3] = {f64 ? float(((const double *)x)[i]) : ((const float *)x)[i],
                        f64 ? float(((const double *)y)[i]) : ((const float *)y)[i],
                        f64 ? float(((const double *)z)[i]) : ((const float *)z)[i]};
    uint32_t key = 0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const float ext = hi[d] - lo[d];
        float u = ext > 0.f ? (p[d] - lo[d]) / ext : 0.5f;
        u = fminf(fmaxf(u, 0.f), 1.f);  // NaN -> 0
        uint32_t v = uint32_t(fminf(u * 1024.f, 1023.f));
        v = (v * 0x00010001u) & 0xFF0000FFu;
        v = (v * 0x00000101u) & 0x0F00F00Fu;
        v = (v * 0x00000011u) & 0xC30C30C3u;
        v = (v * 0x00000005u) & 0x49249249u;
        key |= v << (2 - d);
    }
    keys[i] = key;
    vals[i] = int(i);
}

int grid_steps_for(long long one_step_blocks) {
    const int forced = env_int("SSDF_B200_GRID_STEPS", 0);
    if (forced > 0) return forced < kMaxGridSteps ? forced : kMaxGridSteps;
    static int slots[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    int &r = slots[dev & 63];
    if (r == 0) {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        r = std::max(1, sms) * SSDF_B200_QUERY_MIN_BLOCKS;
    }
    int steps = kDefaultGridSteps;
    while (steps > 1 && one_step_blocks / steps < 4ll * r) steps >>= 1;
    return steps;
}

void set_grid_steps(QueryArgs *a) {
    if (!a->is_grid) return;
    a->grid_steps = grid_steps_for(grid_blocks_x(a->nx) * grid_blocks_y(a->ny) * grid_blocks_z(a->nz, 1));
}

// Measured on B200: the torus knot with 29 % of its triangles slivers still runs 1.4x faster on the
// fix-up path than on FP64; the beam lattice (64 % slivers, in parallel bundles) runs 5x slower.
constexpr double kIllMaxFraction = 0.5;

// The fix-up path hands a mesh to the FP64 kernel when more than this fraction of its triangles are
// ill-conditioned (SSDF_B200_ILL_MAX overrides; above 1 never).
bool sliver_heavy(const DeviceMesh &m) {
    const char *v = env_str("SSDF_B200_ILL_MAX");
    const double f = v ? atof(v) : kIllMaxFraction;
    return m.nt > 0 && double(m.nill) > f * double(m.nt);
}

// A fix-up request on this mesh runs the FP64 kernel (the same bits): a mesh made mostly of slivers,
// or one outside the float filter's preconditions (coordinates beyond 2^28, a record that rounding to
// float made degenerate or too small, or a window wider than 2^-8).
bool fixup_runs_f64(const DeviceMesh &m) { return sliver_heavy(m) || !m.filter_ok; }


int morton_point_order(long long n, const void *x, const void *y, const void *z, int f64, const float4 *nodes32,
                       int **order, cudaStream_t stream) {
    *order = nullptr;
    if (n <= 0 || n >= 0x7fffffffll) return fail(SSDF_ERR_INVALID_ARGUMENT, "point count out of range for sorting");
    uint32_t *keys = nullptr;
    SSDF_CUDA(cudaMallocAsync(&keys, sizeof(uint32_t) * size_t(n), stream));
    cudaError_t e = cudaMallocAsync(order, sizeof(int) * size_t(n), stream);
    int st = e == cudaSuccess ? SSDF_OK : cuda_fail(e, "sort order", __FILE__, __LINE__);
    if (st == SSDF_OK) {
        k_point_keys<<<unsigned((n + 255) / 256), 256, 0, stream>>>(n, x, y, z, f64, nodes32, keys, *order);
        e = cudaGetLastError();
        st = e == cudaSuccess ? radix_sort_pairs_u32(keys, *order, int(n), 30, stream)
                              : cuda_fail(e, "point keys", __FILE__, __LINE__);
    }
    cudaFreeAsync(keys, stream);
    if (st != SSDF_OK && *order) {
        cudaFreeAsync(*order, stream);
        *order = nullptr;
    }
    return st;
}

// Blocks of the second fix-up stage (kWindowBlocksPerSm per SM, four warps each; more than fit at
// once). The warps stride over the overflow count, which is only known on the device.
unsigned window_grid() {
    static int cached[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    int &g = cached[dev & 63];
    if (g == 0) {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        g = kWindowBlocksPerSm * std::max(1, sms);
    }
    return unsigned(g);
}

int launch_query(const QueryArgs &args_in, int precision, cudaStream_t stream) {
    return launch_query_keep(args_in, precision, stream, nullptr);
}

int launch_query_keep(const QueryArgs &args_in, int precision, cudaStream_t stream, int **fallback_list) {
    if (fallback_list) *fallback_list = nullptr;
    retain_pool_memory();
    QueryArgs a = args_in;
    const long long n = a.is_grid ? a.nx * a.ny * a.nz : a.npoints;
    if (n <= 0) return SSDF_OK;
    if (precision == SSDF_PREC_F64 && !a.m.nodes64)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "mesh built without double data (keep_fp64=0)");
    if (precision == SSDF_PREC_F32_FIXUP && (!a.m.tris64 || !a.m.nodes64 || !a.m.filt32))
        return fail(SSDF_ERR_INVALID_ARGUMENT, "fix-up queries need the double triangles and BVH (keep_fp64=1)");
    if (a.output == SSDF_OUT_SDF && !a.m.face_n)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "signed queries need a mesh built with normals=1");
    if (a.output == SSDF_OUT_SDF && !a.m.tris64)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "signed queries need the double triangles (keep_fp64=1)");
    // A mesh made mostly of ill-conditioned triangles (needles, slivers) is answered faster by the
    // plain FP64 kernel: the fix-up filter sees each such triangle through a wide proxy, whose keys
    // crowd the window. Both give the same bits.
    if (precision == SSDF_PREC_F32_FIXUP && fixup_runs_f64(a.m)) precision = SSDF_PREC_F64;
    a.warp_budget = resolve_warp_budget(a.warp_budget, n, a.m.nt);
    if (a.output == SSDF_OUT_CLOSEST && (!a.m.tris64 || !a.outx || !a.outy || !a.outz || !a.outtri))
        return fail(SSDF_ERR_INVALID_ARGUMENT, "closest-point queries need outx/outy/outz/outtri and double data");
    if (precision == SSDF_PREC_F32 && (a.output == SSDF_OUT_SDF || a.output == SSDF_OUT_CLOSEST))
        return fail(SSDF_ERR_INVALID_ARGUMENT, "SSDF_PREC_F32 serves the edf and sqedf outputs");
    const bool count = env_int("SSDF_B200_COUNT", 0) != 0;
    // large point lists: visit them in Morton order, as warp packets (results are per query, so the
    // order changes nothing but the time); the order array is freed behind the launches
    struct StreamFree {  // stream-ordered free when the launch returns, on every path
        int *p;
        cudaStream_t s;
        ~StreamFree() {
            if (p) cudaFreeAsync(p, s);
        }
    } sorted{nullptr, stream};
    if (!a.is_grid && !a.force_traversal && n >= kSortMinPoints && n < 0x7fffffffll &&
        env_int("SSDF_B200_SORT_POINTS", 1) != 0) {
        SSDF_CHECK(morton_point_order(n, a.x, a.y, a.z, a.coord_f64, a.m.nodes32, &sorted.p, stream));
        a.order = sorted.p;
    }
    const bool warp = use_warp(a);
    const bool wide = use_wide(a);
    const long long nblocks = query_blocks(a);
    if (nblocks > 0x7fffffffll) return fail(SSDF_ERR_NOT_SUPPORTED, "too many queries in one launch");
    unsigned long long *counters = nullptr;
    int *fb = nullptr;
    int st = SSDF_OK;
    if (count) {
        SSDF_CUDA(cudaMallocAsync(&counters, 4 * sizeof(unsigned long long), stream));
        SSDF_CUDA(cudaMemsetAsync(counters, 0, 4 * sizeof(unsigned long long), stream));
    }
    a.counters = counters;
    cudaError_t e = cudaSuccess;
    if (precision == SSDF_PREC_F32_FIXUP) {
        if (n >= 0x7fffffffll) {
            st = fail(SSDF_ERR_NOT_SUPPORTED, "more than 2^31 - 1 queries in one fix-up launch");
        } else if (cudaMallocAsync(&fb, sizeof(int) * size_t(2 * n + 1), stream) != cudaSuccess) {
            st = fail(SSDF_ERR_OUT_OF_MEMORY, "fix-up overflow list");
        } else {
            a.fallback_count = fb;
            a.fallback_ids = fb + 1;
            a.fallback_thr = reinterpret_cast<float *>(fb + 1 + n);
            e = cudaMemsetAsync(fb, 0, sizeof(int), stream);
            if (e == cudaSuccess) e = launch_prec<SSDF_PREC_F32_FIXUP>(a, warp, wide, count, unsigned(nblocks), stream);
            if (e == cudaSuccess) {
                const unsigned wg = window_grid();
                const int cap = window_stack_cap();
                count ? k_window<true><<<wg, kThreads, 0, stream>>>(a, cap)
                      : k_window<false><<<wg, kThreads, 0, stream>>>(a, cap);
                e = cudaGetLastError();
            }
        }
    } else if (precision == SSDF_PREC_F64) {
        e = launch_prec<SSDF_PREC_F64>(a, warp, wide, count, unsigned(nblocks), stream);
    } else {
        e = launch_prec<SSDF_PREC_F32>(a, warp, wide, count, unsigned(nblocks), stream);
    }
    if (e != cudaSuccess && st == SSDF_OK) st = cuda_fail(e, "query launch", __FILE__, __LINE__);
    if (count && st == SSDF_OK) {
        unsigned long long h[4] = {0, 0, 0, 0};
        int nfb = 0;
        cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, stream);
        if (fb) cudaMemcpyAsync(&nfb, fb, sizeof(int), cudaMemcpyDeviceToHost, stream);
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) st = cuda_fail(e, "query counters", __FILE__, __LINE__);
        h[3] = (unsigned long long)nfb;
        memcpy(t_last_counts, h, sizeof(h));
    }
    if (fb && fallback_list && st == SSDF_OK)
        *fallback_list = fb;  // [count, ids...]; the caller frees it (stream-ordered)
    else if (fb)
        cudaFreeAsync(fb, stream);
    if (counters) cudaFreeAsync(counters, stream);
    return st;
}

// Resident blocks per SM of the batch kernel for this arithmetic / traversal.
int batch_blocks_per_sm(int precision, bool warp, bool wide) {
    if (precision == SSDF_PREC_F64)
        return warp ? (wide ? batch_occupancy<SSDF_PREC_F64, true, true>() : batch_occupancy<SSDF_PREC_F64, true, false>())
                    : (wide ? batch_occupancy<SSDF_PREC_F64, false, true>() : batch_occupancy<SSDF_PREC_F64, false, false>());
    if (precision == SSDF_PREC_F32)
        return warp ? (wide ? batch_occupancy<SSDF_PREC_F32, true, true>() : batch_occupancy<SSDF_PREC_F32, true, false>())
                    : (wide ? batch_occupancy<SSDF_PREC_F32, false, true>() : batch_occupancy<SSDF_PREC_F32, false, false>());
    return warp ? (wide ? batch_occupancy<SSDF_PREC_F32_FIXUP, true, true>()
                        : batch_occupancy<SSDF_PREC_F32_FIXUP, true, false>())
                : (wide ? batch_occupancy<SSDF_PREC_F32_FIXUP, false, true>()
                        : batch_occupancy<SSDF_PREC_F32_FIXUP, false, false>());
}

// Enqueues the persistent batch kernel (and the fix-up window stage) on `stream`; the job table and
// counters in `b` must already be in device memory. Capturable in a CUDA graph. Batch jobs carry no
// counter buffer (QueryArgs::counters is null), so batch launches never take the counting
// instantiations, whatever SSDF_B200_COUNT says.
int launch_batch(const BatchLaunch &b, int precision, cudaStream_t stream) {
    const bool count = false;
    cudaError_t e;
    if (precision == SSDF_PREC_F64)
        e = launch_batch_prec<SSDF_PREC_F64>(b, count, stream);
    else if (precision == SSDF_PREC_F32)
        e = launch_batch_prec<SSDF_PREC_F32>(b, count, stream);
    else
        e = launch_batch_prec<SSDF_PREC_F32_FIXUP>(b, count, stream);
    if (e != cudaSuccess) return cuda_fail(e, "batch launch", __FILE__, __LINE__);
    return SSDF_OK;
}

bool default_warp(int is_grid) {
    const char *v = env_str("SSDF_B200_TRAVERSAL");
    if (v && !strcmp(v, "warp")) return true;
    if (v && !strcmp(v, "thread")) return false;
    return is_grid != 0;
}

bool default_wide() { return env_int("SSDF_B200_ARITY", 2) == 4; }

// ---- allocation-free variant of the fix-up grid query ------------------------------------------------
//
// For callers that cannot allocate device memory while they query (a real-time loop whose memory is
// reserved up front, an application that runs under a custom allocator and forbids the CUDA one, a
// plugin host that owns all allocations): the FP32 + FP64 fix-up query keeps its overflow list
// (count, query ids, window thresholds) in this fixed array instead of stream-ordered scratch. The
// array is part of the library image, so every GPU that loads the library holds it (8 MiB) until
// the process exits. All calls share it: each call clears the count it starts from, and two calls
// whose kernels overlap on the GPU (different streams, no ordering between them) race on it.
constexpr long long kNoAllocMaxQueries = 1ll << 20;  // queries per call
static __device__ __align__(256) int g_noalloc_scratch[2 * kNoAllocMaxQueries + 1];

static std::mutex g_noalloc_mutex;
static int *g_noalloc_ptr[256];

// Device address of g_noalloc_scratch on the current device, looked up once per device (the host
// symbol is only a stand-in for it). The address belongs to the device's context: a process that calls
// cudaDeviceReset on a device must not use the allocation-free query on that device afterwards.
static int noalloc_scratch(int **ptr) {
    int dev = 0;
    SSDF_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) return fail(SSDF_ERR_NOT_SUPPORTED, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
        g_noalloc_ptr[dev] = static_cast<int *>(p);
    }
    *ptr = g_noalloc_ptr[dev];
    return SSDF_OK;
}

long long noalloc_max_queries() { return kNoAllocMaxQueries; }

// The fix-up query of `args` with its overflow list in g_noalloc_scratch: no allocation. It takes the
// same launch decisions as launch_query_keep: the packet work budget of a launch this size, and the
// FP64 kernel (which needs no scratch) for a mesh made mostly of ill-conditioned triangles.
int launch_query_noalloc(const QueryArgs &args_in, cudaStream_t stream) {
    QueryArgs a = args_in;
    const long long n = a.is_grid ? a.nx * a.ny * a.nz : a.npoints;
    if (n <= 0) return SSDF_OK;
    if (n > kNoAllocMaxQueries)
        return fail(SSDF_ERR_NOT_SUPPORTED, "the allocation-free query takes at most " +
                                                std::to_string(kNoAllocMaxQueries) + " queries per call, got " +
                                                std::to_string(n) + ": split the grid into slabs");
    if (!a.m.tris64 || !a.m.nodes64 || !a.m.filt32)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "fix-up queries need the double triangles and BVH (keep_fp64=1)");
    if (a.output == SSDF_OUT_SDF && !a.m.face_n)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "signed queries need a mesh built with normals=1");
    a.counters = nullptr;
    const bool warp = use_warp(a), wide = use_wide(a);
    const long long nblocks = query_blocks(a);
    if (fixup_runs_f64(a.m)) {  // the same bits from the FP64 kernel, which has no overflow list
        const cudaError_t e = launch_prec<SSDF_PREC_F64>(a, warp, wide, false, unsigned(nblocks), stream);
        if (e != cudaSuccess) return cuda_fail(e, "allocation-free query launch", __FILE__, __LINE__);
        return SSDF_OK;
    }
    a.warp_budget = resolve_warp_budget(a.warp_budget, n, a.m.nt);
    int *scratch = nullptr;
    SSDF_CHECK(noalloc_scratch(&scratch));
    a.fallback_count = scratch;
    a.fallback_ids = scratch + 1;
    a.fallback_thr = reinterpret_cast<float *>(scratch + 1 + n);
    cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(int), stream);  // the count starts at zero
    if (e == cudaSuccess) e = launch_prec<SSDF_PREC_F32_FIXUP>(a, warp, wide, false, unsigned(nblocks), stream);
    if (e == cudaSuccess) {
        k_window<false><<<window_grid(), kThreads, 0, stream>>>(a, kWinStack);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return cuda_fail(e, "allocation-free query launch", __FILE__, __LINE__);
    return SSDF_OK;
}

}  // namespace ssdf_b200

