// device_geom.cuh -- point/triangle/box geometry on the device.
//
// The whole library is compiled with -fmad=false, so the plain expressions below are evaluated
// with one rounding per operation in the written order: the "exact" routines are bitwise the
// reference's (ssdf builds as C++17 without FMA contraction). Where a fused multiply-add is
// wanted (the FP32 filter of the fix-up path) it is written as fmaf() explicitly.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ssdf_b200 {

// Squared point-triangle distance, Ericson's Voronoi-region walk (Real-Time Collision Detection,
// 5.1.5), term by term as serial/ssdf.hpp:49-121. Exact in T's arithmetic (IEEE division).
template <typename T>
__device__ __forceinline__ T tri_dist_sq_exact(const T px, const T py, const T pz, const T ax, const T ay,
                                               const T az, const T bx, const T by, const T bz, const T cx,
                                               const T cy, const T cz) {
    const T abx = bx - ax, aby = by - ay, abz = bz - az;
    const T acx = cx - ax, acy = cy - ay, acz = cz - az;
    const T apx = px - ax, apy = py - ay, apz = pz - az;
    const T d1 = abx * apx + aby * apy + abz * apz;
    const T d2 = acx * apx + acy * apy + acz * apz;
    if (d1 <= T(0) && d2 <= T(0)) return apx * apx + apy * apy + apz * apz;
    const T bpx = px - bx, bpy = py - by, bpz = pz - bz;
    const T d3 = abx * bpx + aby * bpy + abz * bpz;
    const T d4 = acx * bpx + acy * bpy + acz * bpz;
    if (d3 >= T(0) && d4 <= d3) return bpx * bpx + bpy * bpy + bpz * bpz;
    const T vc = d1 * d4 - d3 * d2;
    if (vc <= T(0) && d1 >= T(0) && d3 <= T(0)) {
        const T v = d1 / (d1 - d3);
        const T dx = px - (ax + v * abx), dy = py - (ay + v * aby), dz = pz - (az + v * abz);
        return dx * dx + dy * dy + dz * dz;
    }
    const T cpx = px - cx, cpy = py - cy, cpz = pz - cz;
    const T d5 = abx * cpx + aby * cpy + abz * cpz;
    const T d6 = acx * cpx + acy * cpy + acz * cpz;
    if (d6 >= T(0) && d5 <= d6) return cpx * cpx + cpy * cpy + cpz * cpz;
    const T vb = d5 * d2 - d1 * d6;
    if (vb <= T(0) && d2 >= T(0) && d6 <= T(0)) {
        const T w = d2 / (d2 - d6);
        const T dx = px - (ax + w * acx), dy = py - (ay + w * acy), dz = pz - (az + w * acz);
        return dx * dx + dy * dy + dz * dz;
    }
    const T va = d3 * d6 - d5 * d4;
    if (va <= T(0) && (d4 - d3) >= T(0) && (d5 - d6) >= T(0)) {
        const T w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        const T dx = px - (bx + w * (cx - bx)), dy = py - (by + w * (cy - by)), dz = pz - (bz + w * (cz - bz));
        return dx * dx + dy * dy + dz * dz;
    }
    const T denom = T(1) / (va + vb + vc);
    const T v = vb * denom;
    const T w = vc * denom;
    const T dx = px - (ax + abx * v + acx * w);
    const T dy = py - (ay + aby * v + acy * w);
    const T dz = pz - (az + abz * v + acz * w);
    return dx * dx + dy * dy + dz * dz;
}

// The closest point itself, same regions (serial/ssdf.hpp:143-239).
template <typename T>
__device__ __forceinline__ void tri_closest_point_exact(const T px, const T py, const T pz, const T ax, const T ay,
                                                        const T az, const T bx, const T by, const T bz, const T cx,
                                                        const T cy, const T cz, T &ox, T &oy, T &oz) {
    const T abx = bx - ax, aby = by - ay, abz = bz - az;
    const T acx = cx - ax, acy = cy - ay, acz = cz - az;
    const T apx = px - ax, apy = py - ay, apz = pz - az;
    const T d1 = abx * apx + aby * apy + abz * apz;
    const T d2 = acx * apx + acy * apy + acz * apz;
    if (d1 <= T(0) && d2 <= T(0)) {
        ox = ax, oy = ay, oz = az;
        return;
    }
    const T bpx = px - bx, bpy = py - by, bpz = pz - bz;
    const T d3 = abx * bpx + aby * bpy + abz * bpz;
    const T d4 = acx * bpx + acy * bpy + acz * bpz;
    if (d3 >= T(0) && d4 <= d3) {
        ox = bx, oy = by, oz = bz;
        return;
    }
    const T vc = d1 * d4 - d3 * d2;
    if (vc <= T(0) && d1 >= T(0) && d3 <= T(0)) {
        const T v = d1 / (d1 - d3);
        ox = ax + v * abx, oy = ay + v * aby, oz = az + v * abz;
        return;
    }
    const T cpx = px - cx, cpy = py - cy, cpz = pz - cz;
    const T d5 = abx * cpx + aby * cpy + abz * cpz;
    const T d6 = acx * cpx + acy * cpy + acz * cpz;
    if (d6 >= T(0) && d5 <= d6) {
        ox = cx, oy = cy, oz = cz;
        return;
    }
    const T vb = d5 * d2 - d1 * d6;
    if (vb <= T(0) && d2 >= T(0) && d6 <= T(0)) {
        const T w = d2 / (d2 - d6);
        ox = ax + w * acx, oy = ay + w * acy, oz = az + w * acz;
        return;
    }
    const T va = d3 * d6 - d5 * d4;
    if (va <= T(0) && (d4 - d3) >= T(0) && (d5 - d6) >= T(0)) {
        const T w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        const T bcx = cx - bx, bcy = cy - by, bcz = cz - bz;
        ox = bx + w * bcx, oy = by + w * bcy, oz = bz + w * bcz;
        return;
    }
    const T denom = T(1) / (va + vb + vc);
    const T v = vb * denom;
    const T w = vc * denom;
    ox = ax + abx * v + acx * w;
    oy = ay + aby * v + acy * w;
    oz = az + abz * v + acz * w;
}

// FP32 filter of the fix-up path: Ericson's regions (Real-Time Collision Detection, 5.1.5) over a
// precomputed record -- corner a, edges ab and ac, and the products ab.ab, ac.ac, ab.ac -- so that
// the dot products with b - p and c - p follow from those with a - p by one subtraction each, with
// fused multiply-adds and an approximate quotient on the edges. In the face region the key is the
// squared distance to the plane, (n.ap)^2 / n.n with n = ab x ac, rather than the distance to the
// point the barycentric solve gives: its rounding error does not grow with the square of the
// triangle's aspect ratio. The three corner regions are tested before the edges (A, B, C, then AB,
// AC, BC, then the face): most keys of a grid walk end at a corner (86 % of the tests on the
// torus-knot grid), and testing C before AB spares those lanes the edge product vc. Every branch
// whose sign tests hold in float is covered by the bound below, so the order leaves it unchanged.
// The error against the exact distance (input rounding, every fmaf, the
// quotient and reciprocal, the region decisions) is bounded by
//   u (8 R + 7.7 alpha L) + min(D, 2 D^2 / d),  D = 90 u alpha R,  u = 2^-24,
// R the largest distance from p to a corner, L the longest edge, alpha = L / (smallest altitude),
// d the distance; the fix-up window is sized per mesh to twice that (mesh_build.cu, filter_bound).
struct FiltRec {
    float ax, ay, az, abx, aby, abz, acx, acy, acz, abab, acac, abac;
    float pen;  // 0, or +inf for a proxy (a lower bound that may enter the window, never its centre)
};
__device__ __forceinline__ float tri_dist_sq_filter(const float px, const float py, const float pz, const FiltRec &r) {
    const float apx = px - r.ax, apy = py - r.ay, apz = pz - r.az;
    const float d1 = fmaf(r.abx, apx, fmaf(r.aby, apy, r.abz * apz));
    const float d2 = fmaf(r.acx, apx, fmaf(r.acy, apy, r.acz * apz));
    if (d1 <= 0.f && d2 <= 0.f) return fmaf(apx, apx, fmaf(apy, apy, apz * apz));
    const float d3 = d1 - r.abab, d4 = d2 - r.abac;  // ab.(p - b), ac.(p - b)
    if (d3 >= 0.f && d4 <= d3) {
        const float bx = apx - r.abx, by = apy - r.aby, bz = apz - r.abz;
        return fmaf(bx, bx, fmaf(by, by, bz * bz));
    }
    const float d5 = d1 - r.abac, d6 = d2 - r.acac;  // ab.(p - c), ac.(p - c)
    if (d6 >= 0.f && d5 <= d6) {
        const float cx = apx - r.acx, cy = apy - r.acy, cz = apz - r.acz;
        return fmaf(cx, cx, fmaf(cy, cy, cz * cz));
    }
    const float vc = fmaf(d1, d4, -d3 * d2);
    if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
        const float v = __fdividef(d1, d1 - d3);
        const float dx = fmaf(-v, r.abx, apx), dy = fmaf(-v, r.aby, apy), dz = fmaf(-v, r.abz, apz);
        return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    }
    const float vb = fmaf(d5, d2, -d1 * d6);
    if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
        const float w = __fdividef(d2, d2 - d6);
        const float dx = fmaf(-w, r.acx, apx), dy = fmaf(-w, r.acy, apy), dz = fmaf(-w, r.acz, apz);
        return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    }
    const float va = fmaf(d3, d6, -d5 * d4);
    if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
        const float w = __fdividef(d4 - d3, (d4 - d3) + (d5 - d6));
        // p - (b + w (c - b)) = (p - a) - ab - w (ac - ab)
        const float dx = fmaf(-w, r.acx - r.abx, apx - r.abx);
        const float dy = fmaf(-w, r.acy - r.aby, apy - r.aby);
        const float dz = fmaf(-w, r.acz - r.abz, apz - r.abz);
        return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    }
    // inside: the plane's distance, n = ab x ac
    const float nx = fmaf(r.aby, r.acz, -r.abz * r.acy);
    const float ny = fmaf(r.abz, r.acx, -r.abx * r.acz);
    const float nz = fmaf(r.abx, r.acy, -r.aby * r.acx);
    const float nq = fmaf(nx, apx, fmaf(ny, apy, nz * apz));
    const float nn = fmaf(nx, nx, fmaf(ny, ny, nz * nz));
    return nq * (nq * __frcp_rn(nn));  // this order keeps every intermediate finite for |coordinates| <= 2^28
}


// Point-box squared distance (serial/edf/edf.hpp:55-69 computes the same quantity); used only to
// prune, with a margin, so its rounding never decides a result.
template <typename T>
__device__ __forceinline__ T box_dist_sq(const T px, const T py, const T pz, const T lox, const T hix, const T loy,
                                         const T hiy, const T loz, const T hiz) {
    const T dx = fmax(fmax(lox - px, px - hix), T(0));
    const T dy = fmax(fmax(loy - py, py - hiy), T(0));
    const T dz = fmax(fmax(loz - pz, pz - hiz), T(0));
    return dx * dx + dy * dy + dz * dz;
}

// The same distance as p - clamp(p, lo, hi) per axis: bitwise the magnitude of max(lo - p, p - hi, 0)
// (and +inf for an inverted, empty box) in three instructions per axis instead of four.
__device__ __forceinline__ float box_dist_sq_fast(const float px, const float py, const float pz, const float lox,
                                                  const float hix, const float loy, const float hiy,
                                                  const float loz, const float hiz) {
    const float dx = px - fminf(fmaxf(px, lox), hix);
    const float dy = py - fminf(fmaxf(py, loy), hiy);
    const float dz = pz - fminf(fmaxf(pz, loz), hiz);
    return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
}

// Node-grid coordinate in G precision (serial/bvh/bvh.cpp:1665-1667, 1744): lo + i * h, one
// rounding per operation, widened to double.
template <typename G>
__device__ __forceinline__ double grid_coord(const G lo, const G h, const long long i) {
    return double(lo + G(i) * h);
}

}  // namespace ssdf_b200
