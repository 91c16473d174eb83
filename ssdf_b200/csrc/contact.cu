// contact.cu -- the closest primitive within a radius of each point: ssdf::closest_within_radius_bvh,
// _local_bvh, _quads_bvh and _quads_local_bvh (serial/bvh/bvh.cpp:367-832, declared at
// serial/bvh/bvh.hpp:68-154), on the device BVH.
//
// The reference builds a cuBQL BVH over the primitives' boxes on the host and, per point, visits
// every primitive whose box lies within the radius (cuBQL::fixedRadiusQuery), keeping the closest
// with `sqrDist <= closest`, everything in float. Here the BVH is the library's own, built on the
// device; a quad enters it as its two halves (0, 1, 2) and (0, 2, 3), whose boxes together cover the
// quad's. Each point walks the tree with the radius shrunk to the best squared distance found so
// far (a box farther than that cannot hold a better primitive), nearer child first, and keeps the
// lexicographic minimum of (float squared distance, primitive index) among primitives at most the
// incoming radius away. Large point sets are visited in Morton order so that a warp's points share
// their paths.
//
// Primitive arithmetic, float, one rounding per operation in the written order (the library is
// compiled with -fmad=false):
//   triangles: the closest point of serial/ssdf.hpp:143-239 (tri_closest_point_exact<float>), standing
//              in for cuBQL's triangles::computeClosestPoint, which is not available to this build;
//   quads:     point_to_quad_closest_point (serial/edf/edf.hpp:388-489) with its helpers
//              point_triangle_barycentric and point_segment_parameter (edf.hpp:222-386), then the
//              bilinear point of serial/bvh/bvh.cpp:663-667;
//   the squared distance is |q - closest|^2 summed x, y, z.
// The local variants add, for triangles, triangle_local_coordinates_st (serial/bvh/bvh.cpp:60-83) in
// the output type on the float closest point, and for quads the clamped bilinear (s, t).
#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>
#include <stdlib.h>

#include <vector>

#include "device_geom.cuh"
#include "internal.h"

namespace ssdf_b200 {
namespace {

constexpr int kRadiusThreads = 128;
constexpr float kEps32 = 1.1920928955078125e-7f;  // 2^-23, std::numeric_limits<float>::epsilon()

struct RadiusArgs {
    long long n;
    const void *x, *y, *z;  // points, G
    int g64;                // G == double
    const void *r2;         // radius_squared, T, read at pid * stride
    long long stride;
    int *outtri;
    void *outd, *o0, *o1, *o2;          // T outputs (o2 unused by the local variants)
    const int *e0, *e1, *e2, *e3;       // the caller's element indices (e3 for quads)
    const void *sx, *sy, *sz;           // the caller's vertices, G (local triangle coordinates)
    const float4 *quads;                // [3 * nq]: the quads' float corners, caller's order
    const float4 *nodes;                // binary FP32 BVH
    const float4 *tris;                 // FP32 leaf records
    const int *order;                   // visiting order, or null
    float scale;                        // max |coordinate| over the primitives
    int skip_self;
};

__device__ __forceinline__ float ld_f(const void *p, long long i, int f64) {
    return f64 ? float(__ldg(static_cast<const double *>(p) + i)) : __ldg(static_cast<const float *>(p) + i);
}

template <typename T>
__device__ __forceinline__ T ld_t(const void *p, long long i, int f64) {
    return f64 ? T(__ldg(static_cast<const double *>(p) + i)) : T(__ldg(static_cast<const float *>(p) + i));
}

// std::clamp(v, 0, 1): a NaN stays NaN.
__device__ __forceinline__ float clamp01(float v) { return v < 0.f ? 0.f : (1.f < v ? 1.f : v); }

// serial/edf/edf.hpp:222-249: squared distance to segment ab, parameter of the closest point.
__device__ __forceinline__ float segment_f(float qx, float qy, float qz, float ax, float ay, float az, float bx,
                                           float by, float bz, float &u) {
    const float ex = bx - ax, ey = by - ay, ez = bz - az;
    const float fx = qx - ax, fy = qy - ay, fz = qz - az;
    const float len2 = ex * ex + ey * ey + ez * ez;
    u = len2 > 0.f ? clamp01((fx * ex + fy * ey + fz * ez) / len2) : 0.f;
    const float dx = qx - (ax + u * ex), dy = qy - (ay + u * ey), dz = qz - (az + u * ez);
    return dx * dx + dy * dy + dz * dz;
}

// serial/edf/edf.hpp:251-386: squared distance to triangle abc and the barycentric weights of the
// closest point. Near-degenerate triangles (squared normal at most 64 eps times the longest squared
// edge, squared) are their three edges; otherwise Ericson's regions.
__device__ float barycentric_f(float qx, float qy, float qz, float ax, float ay, float az, float bx, float by,
                               float bz, float cx, float cy, float cz, float &wa, float &wb, float &wc) {
    const float abx = bx - ax, aby = by - ay, abz = bz - az;
    const float acx = cx - ax, acy = cy - ay, acz = cz - az;
    const float bcx = cx - bx, bcy = cy - by, bcz = cz - bz;
    const float lab = abx * abx + aby * aby + abz * abz;
    const float lac = acx * acx + acy * acy + acz * acz;
    const float lbc = bcx * bcx + bcy * bcy + bcz * bcz;
    const float nx = aby * acz - abz * acy, ny = abz * acx - abx * acz, nz = abx * acy - aby * acx;
    const float inner = lac < lbc ? lbc : lac;
    const float lmax = lab < inner ? inner : lab;
    const float n2 = nx * nx + ny * ny + nz * nz;
    if (lmax <= 0.f || n2 <= kEps32 * 64.f * lmax * lmax) {
        float u;
        float best = segment_f(qx, qy, qz, ax, ay, az, bx, by, bz, u);
        wa = 1.f - u, wb = u, wc = 0.f;
        float d = segment_f(qx, qy, qz, bx, by, bz, cx, cy, cz, u);
        if (d < best) best = d, wa = 0.f, wb = 1.f - u, wc = u;
        d = segment_f(qx, qy, qz, cx, cy, cz, ax, ay, az, u);
        if (d < best) best = d, wa = u, wb = 0.f, wc = 1.f - u;
        return best;
    }
    const float aqx = qx - ax, aqy = qy - ay, aqz = qz - az;
    const float d1 = abx * aqx + aby * aqy + abz * aqz;
    const float d2 = acx * aqx + acy * aqy + acz * aqz;
    if (d1 <= 0.f && d2 <= 0.f) {
        wa = 1.f, wb = 0.f, wc = 0.f;
        return aqx * aqx + aqy * aqy + aqz * aqz;
    }
    const float bqx = qx - bx, bqy = qy - by, bqz = qz - bz;
    const float d3 = abx * bqx + aby * bqy + abz * bqz;
    const float d4 = acx * bqx + acy * bqy + acz * bqz;
    if (d3 >= 0.f && d4 <= d3) {
        wa = 0.f, wb = 1.f, wc = 0.f;
        return bqx * bqx + bqy * bqy + bqz * bqz;
    }
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
        const float v = d1 / (d1 - d3);
        const float dx = qx - (ax + v * abx), dy = qy - (ay + v * aby), dz = qz - (az + v * abz);
        wa = 1.f - v, wb = v, wc = 0.f;
        return dx * dx + dy * dy + dz * dz;
    }
    const float cqx = qx - cx, cqy = qy - cy, cqz = qz - cz;
    const float d5 = abx * cqx + aby * cqy + abz * cqz;
    const float d6 = acx * cqx + acy * cqy + acz * cqz;
    if (d6 >= 0.f && d5 <= d6) {
        wa = 0.f, wb = 0.f, wc = 1.f;
        return cqx * cqx + cqy * cqy + cqz * cqz;
    }
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
        const float w = d2 / (d2 - d6);
        const float dx = qx - (ax + w * acx), dy = qy - (ay + w * acy), dz = qz - (az + w * acz);
        wa = 1.f - w, wb = 0.f, wc = w;
        return dx * dx + dy * dy + dz * dz;
    }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
        const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        const float dx = qx - (bx + w * bcx), dy = qy - (by + w * bcy), dz = qz - (bz + w * bcz);
        wa = 0.f, wb = 1.f - w, wc = w;
        return dx * dx + dy * dy + dz * dz;
    }
    const float inv = 1.f / (va + vb + vc);
    const float v = vb * inv, w = vc * inv;
    const float dx = qx - (ax + abx * v + acx * w);
    const float dy = qy - (ay + aby * v + acy * w);
    const float dz = qz - (az + abz * v + acz * w);
    wa = 1.f - v - w, wb = v, wc = w;
    return dx * dx + dy * dy + dz * dz;
}

// serial/edf/edf.hpp:388-489: clamped bilinear (s, t) of the point of quad v0 v1 v2 v3 closest to p.
// The split diagonal is 0-2 when the quad is convex in the projection dropping the dominant axis of
// its Newell normal (or, with that projected area within 64 eps of zero, when 0-2 is the shorter
// diagonal), else 1-3; the strictly closer half wins.
__device__ void quad_st_f(float px, float py, float pz, const float (&v)[4][3], float &s, float &t) {
    const float gx = (v[0][1] - v[1][1]) * (v[0][2] + v[1][2]) + (v[1][1] - v[2][1]) * (v[1][2] + v[2][2]) +
                     (v[2][1] - v[3][1]) * (v[2][2] + v[3][2]) + (v[3][1] - v[0][1]) * (v[3][2] + v[0][2]);
    const float gy = (v[0][2] - v[1][2]) * (v[0][0] + v[1][0]) + (v[1][2] - v[2][2]) * (v[1][0] + v[2][0]) +
                     (v[2][2] - v[3][2]) * (v[2][0] + v[3][0]) + (v[3][2] - v[0][2]) * (v[3][0] + v[0][0]);
    const float gz = (v[0][0] - v[1][0]) * (v[0][1] + v[1][1]) + (v[1][0] - v[2][0]) * (v[1][1] + v[2][1]) +
                     (v[2][0] - v[3][0]) * (v[2][1] + v[3][1]) + (v[3][0] - v[0][0]) * (v[3][1] + v[0][1]);
    const float ax = fabsf(gx), ay = fabsf(gy), az = fabsf(gz);
    const int iu = (ax >= ay && ax >= az) ? 1 : 0;            // drop x: (y, z); else (x, z) or (x, y)
    const int iv = (ax >= ay && ax >= az) ? 2 : (ay >= az ? 2 : 1);
    float u[4], w[4];
#pragma unroll
    for (int k = 0; k < 4; k++) u[k] = v[k][iu], w[k] = v[k][iv];
    const float area2 = u[0] * w[1] - w[0] * u[1] + u[1] * w[2] - w[1] * u[2] + u[2] * w[3] - w[2] * u[3] +
                        u[3] * w[0] - w[3] * u[0];
    const float turn1 = (u[1] - u[0]) * (w[2] - w[0]) - (w[1] - w[0]) * (u[2] - u[0]);
    const float turn3 = (u[3] - u[2]) * (w[0] - w[2]) - (w[3] - w[2]) * (u[0] - u[2]);
    bool split02;
    if (fabsf(area2) > kEps32 * 64.f) {
        const float sgn = area2 > 0.f ? 1.f : -1.f;
        split02 = !(turn1 * sgn < 0.f || turn3 * sgn < 0.f);
    } else {
        const float ex = v[2][0] - v[0][0], ey = v[2][1] - v[0][1], ez = v[2][2] - v[0][2];
        const float fx = v[3][0] - v[1][0], fy = v[3][1] - v[1][1], fz = v[3][2] - v[1][2];
        split02 = (ex * ex + ey * ey + ez * ez) <= (fx * fx + fy * fy + fz * fz);
    }
    // halves (0, 1, 2) + (0, 2, 3), or (0, 1, 3) + (1, 2, 3)
    const int h0[3] = {0, 1, split02 ? 2 : 3};
    const int h1[3] = {split02 ? 0 : 1, 2, 3};
    float wa, wb, wc;
    const float d0 = barycentric_f(px, py, pz, v[h0[0]][0], v[h0[0]][1], v[h0[0]][2], v[h0[1]][0], v[h0[1]][1],
                                   v[h0[1]][2], v[h0[2]][0], v[h0[2]][1], v[h0[2]][2], wa, wb, wc);
    float s0 = split02 ? wb + wc : wb, t0 = wc;
    const float d1 = barycentric_f(px, py, pz, v[h1[0]][0], v[h1[0]][1], v[h1[0]][2], v[h1[1]][0], v[h1[1]][1],
                                   v[h1[1]][2], v[h1[2]][0], v[h1[2]][1], v[h1[2]][2], wa, wb, wc);
    if (d1 < d0) s0 = split02 ? wb : wa + wb, t0 = wb + wc;
    s = clamp01(s0);
    t = clamp01(t0);
}

// serial/bvh/bvh.cpp:60-83: p = a + s (b - a) + t (c - a) by the normal equations, in T.
template <typename T>
__device__ __forceinline__ void local_st(T px, T py, T pz, T ax, T ay, T az, T bx, T by, T bz, T cx, T cy, T cz,
                                         T &s, T &t) {
    const T ex = bx - ax, ey = by - ay, ez = bz - az;
    const T fx = cx - ax, fy = cy - ay, fz = cz - az;
    const T gx = px - ax, gy = py - ay, gz = pz - az;
    const T ee = ex * ex + ey * ey + ez * ez;
    const T ef = ex * fx + ey * fy + ez * fz;
    const T ff = fx * fx + fy * fy + fz * fz;
    const T ge = gx * ex + gy * ey + gz * ez;
    const T gf = gx * fx + gy * fy + gz * fz;
    const T inv = T(1) / (ee * ff - ef * ef);
    s = (ff * ge - ef * gf) * inv;
    t = (ee * gf - ef * ge) * inv;
}

template <typename T>
__device__ __forceinline__ void st_t(void *p, long long i, T v) {
    static_cast<T *>(p)[i] = v;
}

// Squared distance from q to box [lo, hi] shrunk by the margin e on every side (never below 0): a
// primitive's float closest point may round up to e outside its box, so the walk must not cut a box
// its primitives could still beat.
__device__ __forceinline__ float gap_sq(float qx, float qy, float qz, float lox, float hix, float loy, float hiy,
                                        float loz, float hiz, float e) {
    const float dx = fmaxf(fmaxf(lox - qx, qx - hix) - e, 0.f);
    const float dy = fmaxf(fmaxf(loy - qy, qy - hiy) - e, 0.f);
    const float dz = fmaxf(fmaxf(loz - qz, qz - hiz) - e, 0.f);
    return dx * dx + dy * dy + dz * dz;
}

template <bool QUAD, bool LOCAL, typename T>
__global__ void __launch_bounds__(kRadiusThreads) k_within_radius(const RadiusArgs a) {
    const long long slot = blockIdx.x * (long long)kRadiusThreads + threadIdx.x;
    if (slot >= a.n) return;
    const long long pid = a.order ? (long long)__ldg(a.order + slot) : slot;
    const float qx = ld_f(a.x, pid, a.g64), qy = ld_f(a.y, pid, a.g64), qz = ld_f(a.z, pid, a.g64);
    float best = float(ld_t<T>(a.r2, pid * a.stride, sizeof(T) == 8));
    int bt = -1;
    float cx = 0.f, cy = 0.f, cz = 0.f, bs = 0.f, btt = 0.f;
    // 2^-20 of the coordinates' magnitude: above the float closest point's rounding (a few ulps)
    const float e = 9.5367431640625e-7f * (a.scale + fmaxf(fabsf(qx), fmaxf(fabsf(qy), fabsf(qz))));
    int snode[kStackSize];
    float sdist[kStackSize];
    int sp = 0, node = 0;
    while (a.nodes != nullptr && best >= 0.f) {  // no primitives, or a negative or NaN radius: nothing
        const float4 n0 = __ldg(a.nodes + 4 * node), n1 = __ldg(a.nodes + 4 * node + 1);
        const float4 n2 = __ldg(a.nodes + 4 * node + 2), n3 = __ldg(a.nodes + 4 * node + 3);
        int r[2] = {__float_as_int(n3.x), __float_as_int(n3.y)};
        float d[2] = {gap_sq(qx, qy, qz, n0.x, n0.y, n0.z, n0.w, n2.x, n2.y, e),
                      gap_sq(qx, qy, qz, n1.x, n1.y, n1.z, n1.w, n2.z, n2.w, e)};
        if (d[1] < d[0]) {
            const float td = d[0];
            d[0] = d[1], d[1] = td;
            const int tr = r[0];
            r[0] = r[1], r[1] = tr;
        }
        int next = -1;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            if (r[h] == kEmptyRef || !(d[h] <= best)) continue;
            if (r[h] >= 0) {
                if (next < 0) next = r[h];
                else if (sp < kStackSize) snode[sp] = r[h], sdist[sp] = d[h], sp++;
                continue;
            }
            const int first = leaf_first(r[h]), count = leaf_count(r[h]);
            for (int k = first; k < first + count; k++) {
                const float4 t0 = __ldg(a.tris + 3 * k), t1 = __ldg(a.tris + 3 * k + 1);
                const float4 t2 = __ldg(a.tris + 3 * k + 2);
                const int rid = __float_as_int(t2.y);
                const int id = QUAD ? rid >> 1 : rid;
                if (a.skip_self) {
                    const long long i0 = __ldg(a.e0 + id), i1 = __ldg(a.e1 + id), i2 = __ldg(a.e2 + id);
                    const long long i3 = QUAD ? (long long)__ldg(a.e3 + id) : i2;
                    if (pid == i0 || pid == i1 || pid == i2 || pid == i3) continue;
                }
                float px, py, pz, ps = 0.f, pt = 0.f;
                if constexpr (QUAD) {
                    const float4 q0 = __ldg(a.quads + 3 * id), q1 = __ldg(a.quads + 3 * id + 1);
                    const float4 q2 = __ldg(a.quads + 3 * id + 2);
                    const float v[4][3] = {{q0.x, q0.y, q0.z}, {q0.w, q1.x, q1.y}, {q1.z, q1.w, q2.x},
                                           {q2.y, q2.z, q2.w}};
                    quad_st_f(qx, qy, qz, v, ps, pt);
                    const float ms = 1.f - ps, mt = 1.f - pt;
                    const float w0 = ms * mt, w1 = ps * mt, w2 = ps * pt, w3 = ms * pt;
                    px = v[0][0] * w0 + v[1][0] * w1 + v[2][0] * w2 + v[3][0] * w3;
                    py = v[0][1] * w0 + v[1][1] * w1 + v[2][1] * w2 + v[3][1] * w3;
                    pz = v[0][2] * w0 + v[1][2] * w1 + v[2][2] * w2 + v[3][2] * w3;
                } else {
                    tri_closest_point_exact<float>(qx, qy, qz, t0.x, t0.y, t0.z, t0.w, t1.x, t1.y, t1.z, t1.w, t2.x,
                                                   px, py, pz);
                }
                const float dx = qx - px, dy = qy - py, dz = qz - pz;
                const float d2 = dx * dx + dy * dy + dz * dz;
                if (d2 != __int_as_float(0x7f800000) &&
                    (d2 < best || (d2 == best && (bt < 0 || id < bt)))) {
                    best = d2, bt = id;
                    cx = px, cy = py, cz = pz, bs = ps, btt = pt;
                }
            }
        }
        if (next < 0) {
            while (sp > 0) {
                sp--;
                if (sdist[sp] <= best) {
                    next = snode[sp];
                    break;
                }
            }
            if (next < 0) break;
        }
        node = next;
    }
    a.outtri[pid] = bt;
    st_t<T>(a.outd, pid, T(best));
    if constexpr (!LOCAL) {
        st_t<T>(a.o0, pid, T(cx));
        st_t<T>(a.o1, pid, T(cy));
        st_t<T>(a.o2, pid, T(cz));
    } else if constexpr (QUAD) {
        st_t<T>(a.o0, pid, T(bs));
        st_t<T>(a.o1, pid, T(btt));
    } else {
        T s = T(0), t = T(0);
        if (bt >= 0) {
            const int i0 = __ldg(a.e0 + bt), i1 = __ldg(a.e1 + bt), i2 = __ldg(a.e2 + bt);
            const int g = a.g64;
            local_st<T>(T(cx), T(cy), T(cz), ld_t<T>(a.sx, i0, g), ld_t<T>(a.sy, i0, g), ld_t<T>(a.sz, i0, g),
                        ld_t<T>(a.sx, i1, g), ld_t<T>(a.sy, i1, g), ld_t<T>(a.sz, i1, g), ld_t<T>(a.sx, i2, g),
                        ld_t<T>(a.sy, i2, g), ld_t<T>(a.sz, i2, g), s, t);
        }
        st_t<T>(a.o0, pid, s);
        st_t<T>(a.o1, pid, t);
    }
}

// Float corners of each quad, caller's order: (x0, y0, z0, x1), (y1, z1, x2, y2), (z2, x3, y3, z3).
__global__ void k_quad_records(int nq, const int *__restrict__ e0, const int *__restrict__ e1,
                               const int *__restrict__ e2, const int *__restrict__ e3, const void *sx, const void *sy,
                               const void *sz, int g64, float4 *__restrict__ out) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const int i[4] = {e0[q], e1[q], e2[q], e3[q]};
    float c[12];
#pragma unroll
    for (int k = 0; k < 4; k++)
        c[3 * k] = ld_f(sx, i[k], g64), c[3 * k + 1] = ld_f(sy, i[k], g64), c[3 * k + 2] = ld_f(sz, i[k], g64);
    out[3 * q] = make_float4(c[0], c[1], c[2], c[3]);
    out[3 * q + 1] = make_float4(c[4], c[5], c[6], c[7]);
    out[3 * q + 2] = make_float4(c[8], c[9], c[10], c[11]);
}

// Device buffers freed (stream-ordered) when the call returns, after the stream has drained.
struct Buffers {
    cudaStream_t stream;
    std::vector<void *> ptrs;
    explicit Buffers(cudaStream_t s) : stream(s) {}
    ~Buffers() {
        for (void *p : ptrs) cudaFreeAsync(p, stream);
        cudaStreamSynchronize(stream);
    }
    int alloc(void **p, size_t bytes) {
        if (cudaMallocAsync(p, bytes ? bytes : 16, stream) != cudaSuccess)
            return fail(SSDF_ERR_OUT_OF_MEMORY, "device allocation of " + std::to_string(bytes) + " bytes");
        ptrs.push_back(*p);
        return SSDF_OK;
    }
    int upload(void **dst, const void *src, size_t bytes) {
        SSDF_CHECK(alloc(dst, bytes));
        SSDF_CUDA(cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, stream));
        return SSDF_OK;
    }
};

struct MeshHold {
    ssdf_mesh *mesh = nullptr;
    cudaStream_t stream = nullptr;
    ~MeshHold() {
        if (mesh) ssdf_mesh_destroy_async(mesh, stream);
    }
};

// The four reference functions over host arrays: validate, build the BVH (a quad as two halves),
// upload, query, download. Blocking, like the reference.
template <typename G, typename T, bool QUAD, bool LOCAL>
int within_radius_host(ptrdiff_t npoints, const G *x, const G *y, const G *z, ptrdiff_t ne, const int *s0,
                       const int *s1, const int *s2, const int *s3, ptrdiff_t nv, const G *sx, const G *sy,
                       const G *sz, ptrdiff_t stride, const T *r2, int *outtri, T *outd, T *o0, T *o1, T *o2,
                       int skip_self) {
    if (npoints < 0 || ne < 0 || nv < 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "negative size");
    if (stride < 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "negative radius_stride");
    if (npoints == 0) return SSDF_OK;
    if (!x || !y || !z || !r2 || !outtri || !outd || !o0 || !o1 || (!LOCAL && !o2))
        return fail(SSDF_ERR_INVALID_ARGUMENT, "null point, radius or output array");
    if (ne > 0 && (!s0 || !s1 || !s2 || (QUAD && !s3))) return fail(SSDF_ERR_INVALID_ARGUMENT, "null index array");
    if (nv > 0 && (!sx || !sy || !sz)) return fail(SSDF_ERR_INVALID_ARGUMENT, "null vertex coordinate array");
    const int *s[4] = {s0, s1, s2, s3};
    for (int k = 0; k < (QUAD ? 4 : 3); k++)
        for (ptrdiff_t e = 0; e < ne; e++)
            if (s[k][e] < 0 || s[k][e] >= nv)
                return fail(SSDF_ERR_INVALID_ARGUMENT, "element " + std::to_string(e) + " has a vertex index outside [0, " +
                                                           std::to_string(nv) + ")");
    if (ne > (QUAD ? kMaxTriangles / 2 : kMaxTriangles))
        return fail(SSDF_ERR_NOT_SUPPORTED, "too many elements for one BVH");
    if (stride > 0 && npoints - 1 > (ptrdiff_t(1) << 60) / stride)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "radius_stride too large");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(SSDF_ERR_CUDA, "no usable CUDA device");
    cudaStream_t stream = library_stream();
    if (!stream) return fail(SSDF_ERR_CUDA, "could not create the library stream");

    RadiusArgs a{};
    a.n = npoints;
    a.g64 = sizeof(G) == 8;
    a.stride = stride;
    a.skip_self = skip_self ? 1 : 0;
    MeshHold mh;
    mh.stream = stream;
    Buffers buf(stream);
    const int cf = sizeof(G) == 8 ? SSDF_F64 : SSDF_F32;
    const bool have_mesh = ne > 0 && nv > 0;
    if (have_mesh) {
        ssdf_build_opts bo;
        bo.leaf_size = env_int("SSDF_B200_LEAF", 0), bo.keep_fp64 = 0, bo.normals = 0;
        bo.treelet_opt = call_treelet_rounds(npoints);
        if (QUAD) {  // halves (0, 1, 2) and (0, 2, 3): record 2e + h belongs to quad e
            std::vector<int> h0(size_t(2 * ne)), h1(size_t(2 * ne)), h2(size_t(2 * ne));
            for (ptrdiff_t e = 0; e < ne; e++) {
                h0[2 * e] = s0[e], h1[2 * e] = s1[e], h2[2 * e] = s2[e];
                h0[2 * e + 1] = s0[e], h1[2 * e + 1] = s2[e], h2[2 * e + 1] = s3[e];
            }
            SSDF_CHECK(ssdf_mesh_create(&mh.mesh, 2 * ne, h0.data(), h1.data(), h2.data(), nv, sx, sy, sz, cf, 0, &bo,
                                        stream));
        } else {
            SSDF_CHECK(ssdf_mesh_create(&mh.mesh, ne, s0, s1, s2, nv, sx, sy, sz, cf, 0, &bo, stream));
        }
        a.nodes = mh.mesh->m.nodes32;
        a.tris = mh.mesh->m.tris32;
        a.scale = mh.mesh->m.coord_scale;
        void *d[4] = {nullptr, nullptr, nullptr, nullptr};
        const bool need_idx = skip_self || QUAD || LOCAL;
        for (int k = 0; k < (QUAD ? 4 : 3) && need_idx; k++)
            SSDF_CHECK(buf.upload(&d[k], s[k], sizeof(int) * size_t(ne)));
        a.e0 = (const int *)d[0], a.e1 = (const int *)d[1], a.e2 = (const int *)d[2], a.e3 = (const int *)d[3];
        if (QUAD || LOCAL) {
            void *vx, *vy, *vz;
            SSDF_CHECK(buf.upload(&vx, sx, sizeof(G) * size_t(nv)));
            SSDF_CHECK(buf.upload(&vy, sy, sizeof(G) * size_t(nv)));
            SSDF_CHECK(buf.upload(&vz, sz, sizeof(G) * size_t(nv)));
            a.sx = vx, a.sy = vy, a.sz = vz;
        }
        if (QUAD) {
            void *qr;
            SSDF_CHECK(buf.alloc(&qr, sizeof(float4) * 3 * size_t(ne)));
            k_quad_records<<<unsigned((ne + 255) / 256), 256, 0, stream>>>(int(ne), a.e0, a.e1, a.e2, a.e3, a.sx, a.sy,
                                                                          a.sz, a.g64, (float4 *)qr);
            SSDF_CUDA(cudaGetLastError());
            a.quads = (const float4 *)qr;
        }
    }
    void *dx, *dy, *dz, *dr, *dt, *dd, *d0, *d1, *d2 = nullptr;
    const size_t gb = sizeof(G) * size_t(npoints), tb = sizeof(T) * size_t(npoints);
    SSDF_CHECK(buf.upload(&dx, x, gb));
    SSDF_CHECK(buf.upload(&dy, y, gb));
    SSDF_CHECK(buf.upload(&dz, z, gb));
    SSDF_CHECK(buf.upload(&dr, r2, sizeof(T) * size_t(stride * (npoints - 1) + 1)));
    SSDF_CHECK(buf.alloc(&dt, sizeof(int) * size_t(npoints)));
    SSDF_CHECK(buf.alloc(&dd, tb));
    SSDF_CHECK(buf.alloc(&d0, tb));
    SSDF_CHECK(buf.alloc(&d1, tb));
    if (!LOCAL) SSDF_CHECK(buf.alloc(&d2, tb));
    a.x = dx, a.y = dy, a.z = dz, a.r2 = dr, a.outtri = (int *)dt, a.outd = dd, a.o0 = d0, a.o1 = d1, a.o2 = d2;
    if (have_mesh && npoints >= 4096 && npoints < 0x7fffffffll && env_int("SSDF_B200_SORT_POINTS", 1) != 0) {
        int *order = nullptr;
        SSDF_CHECK(morton_point_order(npoints, dx, dy, dz, a.g64, a.nodes, &order, stream));
        buf.ptrs.push_back(order);
        a.order = order;
    }
    const long long blocks = (npoints + kRadiusThreads - 1) / kRadiusThreads;
    if (blocks > 0x7fffffffll) return fail(SSDF_ERR_NOT_SUPPORTED, "too many points in one launch");
    k_within_radius<QUAD, LOCAL, T><<<unsigned(blocks), kRadiusThreads, 0, stream>>>(a);
    SSDF_CUDA(cudaGetLastError());
    SSDF_CUDA(cudaMemcpyAsync(outtri, dt, sizeof(int) * size_t(npoints), cudaMemcpyDeviceToHost, stream));
    SSDF_CUDA(cudaMemcpyAsync(outd, dd, tb, cudaMemcpyDeviceToHost, stream));
    SSDF_CUDA(cudaMemcpyAsync(o0, d0, tb, cudaMemcpyDeviceToHost, stream));
    SSDF_CUDA(cudaMemcpyAsync(o1, d1, tb, cudaMemcpyDeviceToHost, stream));
    if (!LOCAL) SSDF_CUDA(cudaMemcpyAsync(o2, d2, tb, cudaMemcpyDeviceToHost, stream));
    SSDF_CUDA(cudaStreamSynchronize(stream));
    return SSDF_OK;
}


// ---- candidate contact pairs (serial/bvh/bvh.cpp:834-1196) -----------------------------------------
//
// ssdf::potential_contact_triangles_bvh / _quads_bvh: for each element, every other element whose
// tight box meets its box grown by `extrusion` along its normals and a tenth of that against them,
// sharing no corner with it; a CSR list whose index array the caller frees with free(). The BVH is
// built over each element's exact float box (a degenerate triangle from the box's low to its high
// corner), so a node is entered exactly when a box under it can meet the query box. A row lists its
// candidates in the order of the element's walk, the same for the same input (the reference's order
// within a row is that of its threads).

struct PairArgs {
    int ne, nk;                      // elements, corners per element (3 or 4)
    const int *e[4];                 // the caller's element indices
    const float4 *prims;             // [3 * ne] float corners (k_quad_records layout)
    const float4 *nodes, *boxes;     // BVH over the element boxes: nodes and leaf records
    float ext, inner;                // extrusion along the normals, and against them
    int *count;                      // [ne] candidates per element
    const int *offset;               // [ne] exclusive scan of count (fill pass)
    int *idx;                        // [total] (fill pass)
    unsigned long long *total;       // count pass
};

__device__ __forceinline__ void prim_corners(const float4 *__restrict__ prims, int e, float (&c)[4][3]) {
    const float4 q0 = __ldg(prims + 3 * e), q1 = __ldg(prims + 3 * e + 1), q2 = __ldg(prims + 3 * e + 2);
    c[0][0] = q0.x, c[0][1] = q0.y, c[0][2] = q0.z, c[1][0] = q0.w, c[1][1] = q1.x, c[1][2] = q1.y;
    c[2][0] = q1.z, c[2][1] = q1.w, c[2][2] = q2.x, c[3][0] = q2.y, c[3][1] = q2.z, c[3][2] = q2.w;
}

__device__ __forceinline__ void cross3(const float (&a)[3], const float (&b)[3], float (&o)[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

// v * (1 / sqrt(v . v)) (IEEE division and square root)
__device__ __forceinline__ void unit3(float (&v)[3]) {
    const float inv = 1.0f / sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    v[0] = v[0] * inv, v[1] = v[1] * inv, v[2] = v[2] * inv;
}

// The grown box of element e: its tight box, each corner moved ext along its normal and inner against
// it. Triangles: the unit normal of (b - a) x (c - a) (cuBQL's Triangle::normal()); quads: one normal
// per corner from its two edges (serial/bvh/bvh.cpp:1019-1030). min / max ignore NaN.
__device__ void grown_box(const float (&c)[4][3], int nk, float ext, float inner, float (&lo)[3], float (&hi)[3]) {
    float n[4][3];
    if (nk == 3) {
        const float u[3] = {c[1][0] - c[0][0], c[1][1] - c[0][1], c[1][2] - c[0][2]};
        const float v[3] = {c[2][0] - c[0][0], c[2][1] - c[0][1], c[2][2] - c[0][2]};
        cross3(u, v, n[0]);
        unit3(n[0]);
        for (int k = 1; k < 3; k++)
            for (int d = 0; d < 3; d++) n[k][d] = n[0][d];
    } else {
        float ab[3], dc[3], ad[3], bc[3];
        for (int d = 0; d < 3; d++) {
            ab[d] = c[1][d] - c[0][d], dc[d] = c[2][d] - c[3][d];
            ad[d] = c[3][d] - c[0][d], bc[d] = c[2][d] - c[1][d];
        }
        cross3(ab, ad, n[0]);
        cross3(ab, bc, n[1]);
        cross3(dc, bc, n[2]);
        cross3(dc, ad, n[3]);
        for (int k = 0; k < 4; k++) unit3(n[k]);
    }
    for (int d = 0; d < 3; d++) {
        lo[d] = c[0][d], hi[d] = c[0][d];
        for (int k = 1; k < nk; k++) lo[d] = fminf(lo[d], c[k][d]), hi[d] = fmaxf(hi[d], c[k][d]);
    }
    for (int k = 0; k < nk; k++)
        for (int d = 0; d < 3; d++) {
            const float out = c[k][d] + n[k][d] * ext, in = c[k][d] - n[k][d] * inner;
            lo[d] = fminf(lo[d], out), hi[d] = fmaxf(hi[d], out);
            lo[d] = fminf(lo[d], in), hi[d] = fmaxf(hi[d], in);
        }
}

// Box vertices of the BVH over the elements: element e is the degenerate triangle (2e, 2e+1, 2e+1)
// from the low to the high corner of its tight float box.
__global__ void k_box_vertices(int ne, int nk, const float4 *__restrict__ prims, float *__restrict__ vx,
                               float *__restrict__ vy, float *__restrict__ vz, int *__restrict__ t0,
                               int *__restrict__ t1) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    float c[4][3];
    prim_corners(prims, e, c);
    float lo[3], hi[3];
    for (int d = 0; d < 3; d++) {
        lo[d] = c[0][d], hi[d] = c[0][d];
        for (int k = 1; k < nk; k++) lo[d] = fminf(lo[d], c[k][d]), hi[d] = fmaxf(hi[d], c[k][d]);
    }
    vx[2 * e] = lo[0], vy[2 * e] = lo[1], vz[2 * e] = lo[2];
    vx[2 * e + 1] = hi[0], vy[2 * e + 1] = hi[1], vz[2 * e + 1] = hi[2];
    t0[e] = 2 * e;
    t1[e] = 2 * e + 1;
}

__device__ __forceinline__ bool meets(const float (&alo)[3], const float (&ahi)[3], float blox, float bhix,
                                      float bloy, float bhiy, float bloz, float bhiz) {
    return alo[0] <= bhix && blox <= ahi[0] && alo[1] <= bhiy && bloy <= ahi[1] && alo[2] <= bhiz && bloz <= ahi[2];
}

// One thread per element. FILL = false counts the candidates, true writes them in the same order.
template <bool FILL>
__global__ void __launch_bounds__(128) k_pairs(const PairArgs a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.ne) return;
    float c[4][3];
    prim_corners(a.prims, p, c);
    float lo[3], hi[3];
    grown_box(c, a.nk, a.ext, a.inner, lo, hi);
    int mine[4];
    for (int k = 0; k < 4; k++) mine[k] = k < a.nk ? __ldg(a.e[k] + p) : -1;
    int *row = FILL ? a.idx + a.offset[p] : nullptr;
    const int room = FILL ? a.count[p] : 0;  // the count pass's figure for this row (the walk repeats it)
    int n = 0;
    int stack[kStackSize];
    int sp = 0, node = 0;
    while (true) {
        const float4 n0 = __ldg(a.nodes + 4 * node), n1 = __ldg(a.nodes + 4 * node + 1);
        const float4 n2 = __ldg(a.nodes + 4 * node + 2), n3 = __ldg(a.nodes + 4 * node + 3);
        const int r[2] = {__float_as_int(n3.x), __float_as_int(n3.y)};
        const bool w[2] = {r[0] != kEmptyRef && meets(lo, hi, n0.x, n0.y, n0.z, n0.w, n2.x, n2.y),
                           r[1] != kEmptyRef && meets(lo, hi, n1.x, n1.y, n1.z, n1.w, n2.z, n2.w)};
        int next = -1;
        for (int h = 0; h < 2; h++) {
            if (!w[h]) continue;
            if (r[h] >= 0) {
                if (next < 0) next = r[h];
                else if (sp < kStackSize) stack[sp++] = r[h];
                continue;
            }
            const int first = leaf_first(r[h]), cnt = leaf_count(r[h]);
            for (int k = first; k < first + cnt; k++) {
                const float4 b0 = __ldg(a.boxes + 3 * k), b1 = __ldg(a.boxes + 3 * k + 1);
                const float4 b2 = __ldg(a.boxes + 3 * k + 2);
                // record: (lo.x, lo.y, lo.z, hi.x), (hi.y, hi.z, hi.x, hi.y), (hi.z, id, ...)
                if (!meets(lo, hi, b0.x, b0.w, b0.y, b1.x, b0.z, b1.y)) continue;
                const int t = __float_as_int(b2.y);
                bool shared = false;
                for (int j = 0; j < a.nk; j++) {
                    const int v = __ldg(a.e[j] + t);
                    for (int i = 0; i < a.nk; i++) shared |= mine[i] == v;
                }
                if (shared) continue;
                if (FILL && n < room) row[n] = t;
                n++;
            }
        }
        if (next < 0) {
            if (sp == 0) break;
            next = stack[--sp];
        }
        node = next;
    }
    if (!FILL) {
        a.count[p] = n;
        atomicAdd(a.total, (unsigned long long)n);
    }
}

template <typename G, typename T, bool QUAD>
int potential_contact_host(ptrdiff_t ne, const int *s0, const int *s1, const int *s2, const int *s3, ptrdiff_t nv,
                           const G *sx, const G *sy, const G *sz, T extrusion, ptrdiff_t *pc_ptr, int **out_idx) {
    if (!pc_ptr || !out_idx) return fail(SSDF_ERR_INVALID_ARGUMENT, "null pc_ptr or out_pc_idx");
    *out_idx = nullptr;
    if (ne < 0 || nv < 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "negative size");
    if (ne > 0 && (!s0 || !s1 || !s2 || (QUAD && !s3))) return fail(SSDF_ERR_INVALID_ARGUMENT, "null index array");
    if (nv > 0 && (!sx || !sy || !sz)) return fail(SSDF_ERR_INVALID_ARGUMENT, "null vertex coordinate array");
    const int nk = QUAD ? 4 : 3;
    const int *s[4] = {s0, s1, s2, s3};
    for (int k = 0; k < nk; k++)
        for (ptrdiff_t e = 0; e < ne; e++)
            if (s[k][e] < 0 || s[k][e] >= nv)
                return fail(SSDF_ERR_INVALID_ARGUMENT, "element " + std::to_string(e) + " has a vertex index outside [0, " +
                                                           std::to_string(nv) + ")");
    if (ne > kMaxTriangles) return fail(SSDF_ERR_NOT_SUPPORTED, "too many elements for one BVH");
    pc_ptr[0] = 0;
    if (ne == 0) {
        *out_idx = static_cast<int *>(malloc(sizeof(int)));
        return *out_idx ? SSDF_OK : fail(SSDF_ERR_OUT_OF_MEMORY, "host index array");
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(SSDF_ERR_CUDA, "no usable CUDA device");
    cudaStream_t stream = library_stream();
    if (!stream) return fail(SSDF_ERR_CUDA, "could not create the library stream");
    Buffers buf(stream);
    MeshHold mh;
    mh.stream = stream;
    PairArgs a{};
    a.ne = int(ne);
    a.nk = nk;
    void *d[4] = {nullptr, nullptr, nullptr, nullptr}, *vx, *vy, *vz;
    for (int k = 0; k < nk; k++) SSDF_CHECK(buf.upload(&d[k], s[k], sizeof(int) * size_t(ne)));
    SSDF_CHECK(buf.upload(&vx, sx, sizeof(G) * size_t(nv)));
    SSDF_CHECK(buf.upload(&vy, sy, sizeof(G) * size_t(nv)));
    SSDF_CHECK(buf.upload(&vz, sz, sizeof(G) * size_t(nv)));
    for (int k = 0; k < 4; k++) a.e[k] = static_cast<const int *>(d[k]);
    void *prims, *bx, *by, *bz, *t0, *t1;
    SSDF_CHECK(buf.alloc(&prims, sizeof(float4) * 3 * size_t(ne)));
    const unsigned blocks = unsigned((ne + 127) / 128);
    k_quad_records<<<unsigned((ne + 255) / 256), 256, 0, stream>>>(int(ne), a.e[0], a.e[1], a.e[2], QUAD ? a.e[3] : a.e[2],
                                                                  vx, vy, vz, sizeof(G) == 8, (float4 *)prims);
    SSDF_CUDA(cudaGetLastError());
    for (void **q : {&bx, &by, &bz}) SSDF_CHECK(buf.alloc(q, sizeof(float) * 2 * size_t(ne)));
    SSDF_CHECK(buf.alloc(&t0, sizeof(int) * size_t(ne)));
    SSDF_CHECK(buf.alloc(&t1, sizeof(int) * size_t(ne)));
    k_box_vertices<<<blocks, 128, 0, stream>>>(int(ne), nk, (const float4 *)prims, (float *)bx, (float *)by,
                                               (float *)bz, (int *)t0, (int *)t1);
    SSDF_CUDA(cudaGetLastError());
    ssdf_build_opts bo;
    bo.leaf_size = env_int("SSDF_B200_LEAF", 0), bo.keep_fp64 = 0, bo.normals = 0;
    bo.treelet_opt = call_treelet_rounds(ne);
    SSDF_CHECK(ssdf_mesh_create(&mh.mesh, ne, (const int *)t0, (const int *)t1, (const int *)t1, 2 * ne, bx, by, bz,
                                SSDF_F32, 1, &bo, stream));
    a.prims = (const float4 *)prims;
    a.nodes = mh.mesh->m.nodes32;
    a.boxes = mh.mesh->m.tris32;
    a.ext = float(extrusion);
    a.inner = float(T(0.1) * extrusion);
    void *cnt, *off, *tot;
    SSDF_CHECK(buf.alloc(&cnt, sizeof(int) * size_t(ne)));
    SSDF_CHECK(buf.alloc(&off, sizeof(int) * size_t(ne)));
    SSDF_CHECK(buf.alloc(&tot, sizeof(unsigned long long)));
    SSDF_CUDA(cudaMemsetAsync(tot, 0, sizeof(unsigned long long), stream));
    a.count = (int *)cnt;
    a.total = (unsigned long long *)tot;
    k_pairs<false><<<blocks, 128, 0, stream>>>(a);
    SSDF_CUDA(cudaGetLastError());
    unsigned long long total = 0;
    SSDF_CUDA(cudaMemcpyAsync(&total, tot, sizeof(total), cudaMemcpyDeviceToHost, stream));
    SSDF_CUDA(cudaStreamSynchronize(stream));
    if (total > 0x7fffffffull) return fail(SSDF_ERR_NOT_SUPPORTED, "more than 2^31 - 1 candidate pairs");
    SSDF_CHECK(exclusive_scan_i32((const int *)cnt, (int *)off, int(ne), stream));
    void *didx;
    SSDF_CHECK(buf.alloc(&didx, sizeof(int) * size_t(total)));
    a.offset = (const int *)off;
    a.idx = (int *)didx;
    k_pairs<true><<<blocks, 128, 0, stream>>>(a);
    SSDF_CUDA(cudaGetLastError());
    int *host = static_cast<int *>(malloc(sizeof(int) * size_t(total > 0 ? total : 1)));
    if (!host) return fail(SSDF_ERR_OUT_OF_MEMORY, "host index array");
    std::vector<int> hoff(size_t(ne) + 1);
    cudaError_t e = cudaMemcpyAsync(hoff.data(), off, sizeof(int) * size_t(ne), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && total > 0)
        e = cudaMemcpyAsync(host, didx, sizeof(int) * size_t(total), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        free(host);
        return cuda_fail(e, "contact pair download", __FILE__, __LINE__);
    }
    for (ptrdiff_t i = 1; i < ne; i++) pc_ptr[i] = hoff[size_t(i)];
    pc_ptr[ne] = ptrdiff_t(total);
    *out_idx = host;
    return SSDF_OK;
}
}  // namespace
}  // namespace ssdf_b200

using ssdf_b200::within_radius_host;

#define RADIUS_ARGS(G, T)                                                                                         \
    ptrdiff_t npoints, const G *x, const G *y, const G *z, ptrdiff_t nselements, const int *s0, const int *s1,    \
        const int *s2, ptrdiff_t nspoints, const G *sx, const G *sy, const G *sz, ptrdiff_t radius_stride,        \
        const T *radius_squared, int *outtri, T *out_sqr_dist
#define QUAD_ARGS(G, T)                                                                                           \
    ptrdiff_t npoints, const G *x, const G *y, const G *z, ptrdiff_t nselements, const int *s0, const int *s1,    \
        const int *s2, const int *s3, ptrdiff_t nspoints, const G *sx, const G *sy, const G *sz,                  \
        ptrdiff_t radius_stride, const T *radius_squared, int *outtri, T *out_sqr_dist

#define RADIUS_FUNCS(SUF, G, T)                                                                                   \
    int ssdf_b200_closest_within_radius_bvh_##SUF(RADIUS_ARGS(G, T), T *closest_x, T *closest_y, T *closest_z,    \
                                                  int skip_self) {                                                \
        return within_radius_host<G, T, false, false>(npoints, x, y, z, nselements, s0, s1, s2, nullptr, nspoints, \
                                                      sx, sy, sz, radius_stride, radius_squared, outtri,          \
                                                      out_sqr_dist, closest_x, closest_y, closest_z, skip_self);  \
    }                                                                                                             \
    int ssdf_b200_closest_within_radius_local_bvh_##SUF(RADIUS_ARGS(G, T), T *closest_s, T *closest_t,            \
                                                        int skip_self) {                                          \
        return within_radius_host<G, T, false, true>(npoints, x, y, z, nselements, s0, s1, s2, nullptr, nspoints,  \
                                                     sx, sy, sz, radius_stride, radius_squared, outtri,           \
                                                     out_sqr_dist, closest_s, closest_t, nullptr, skip_self);     \
    }                                                                                                             \
    int ssdf_b200_closest_within_radius_quads_bvh_##SUF(QUAD_ARGS(G, T), T *closest_x, T *closest_y,              \
                                                        T *closest_z, int skip_self) {                            \
        return within_radius_host<G, T, true, false>(npoints, x, y, z, nselements, s0, s1, s2, s3, nspoints, sx,   \
                                                     sy, sz, radius_stride, radius_squared, outtri, out_sqr_dist, \
                                                     closest_x, closest_y, closest_z, skip_self);                 \
    }                                                                                                             \
    int ssdf_b200_closest_within_radius_quads_local_bvh_##SUF(QUAD_ARGS(G, T), T *closest_s, T *closest_t,        \
                                                              int skip_self) {                                    \
        return within_radius_host<G, T, true, true>(npoints, x, y, z, nselements, s0, s1, s2, s3, nspoints, sx,    \
                                                    sy, sz, radius_stride, radius_squared, outtri, out_sqr_dist,  \
                                                    closest_s, closest_t, nullptr, skip_self);                    \
    }

extern "C" {
RADIUS_FUNCS(ff, float, float)
RADIUS_FUNCS(fd, float, double)
RADIUS_FUNCS(dd, double, double)
}

extern "C" {
int ssdf_b200_potential_contact_triangles_bvh_ff(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                                 ptrdiff_t nspoints, const float *sx, const float *sy, const float *sz,
                                                 float extrusion, ptrdiff_t *pc_ptr, int **out_pc_idx) {
    return ssdf_b200::potential_contact_host<float, float, false>(nselements, s0, s1, s2, nullptr, nspoints, sx, sy, sz,
                                                                   extrusion, pc_ptr, out_pc_idx);
}
int ssdf_b200_potential_contact_triangles_bvh_dd(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                                 ptrdiff_t nspoints, const double *sx, const double *sy,
                                                 const double *sz, double extrusion, ptrdiff_t *pc_ptr,
                                                 int **out_pc_idx) {
    return ssdf_b200::potential_contact_host<double, double, false>(nselements, s0, s1, s2, nullptr, nspoints, sx, sy,
                                                                     sz, extrusion, pc_ptr, out_pc_idx);
}
int ssdf_b200_potential_contact_quads_bvh_ff(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                             const int *s3, ptrdiff_t nspoints, const float *sx, const float *sy,
                                             const float *sz, float extrusion, ptrdiff_t *pc_ptr, int **out_pc_idx) {
    return ssdf_b200::potential_contact_host<float, float, true>(nselements, s0, s1, s2, s3, nspoints, sx, sy, sz,
                                                                  extrusion, pc_ptr, out_pc_idx);
}
int ssdf_b200_potential_contact_quads_bvh_dd(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                             const int *s3, ptrdiff_t nspoints, const double *sx, const double *sy,
                                             const double *sz, double extrusion, ptrdiff_t *pc_ptr,
                                             int **out_pc_idx) {
    return ssdf_b200::potential_contact_host<double, double, true>(nselements, s0, s1, s2, s3, nspoints, sx, sy, sz,
                                                                    extrusion, pc_ptr, out_pc_idx);
}
void ssdf_b200_free(void *p) { free(p); }
}
