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

// FP32 filter of the fix-up path: the same regions with fused multiply-adds and an approximate
// reciprocal. Its error against the exact double value is covered by the fix-up window.
__device__ __forceinline__ float tri_dist_sq_fast(const float px, const float py, const float pz, const float ax,
                                                  const float ay, const float az, const float bx, const float by,
                                                  const float bz, const float cx, const float cy, const float cz) {
    const float abx = bx - ax, aby = by - ay, abz = bz - az;
    const float acx = cx - ax, acy = cy - ay, acz = cz - az;
    const float apx = px - ax, apy = py - ay, apz = pz - az;
    const float d1 = fmaf(abx, apx, fmaf(aby, apy, abz * apz));
    const float d2 = fmaf(acx, apx, fmaf(acy, apy, acz * apz));
    if (d1 <= 0.f && d2 <= 0.f) return fmaf(apx, apx, fmaf(apy, apy, apz * apz));
    const float bpx = px - bx, bpy = py - by, bpz = pz - bz;
    const float d3 = fmaf(abx, bpx, fmaf(aby, bpy, abz * bpz));
    const float d4 = fmaf(acx, bpx, fmaf(acy, bpy, acz * bpz));
    if (d3 >= 0.f && d4 <= d3) return fmaf(bpx, bpx, fmaf(bpy, bpy, bpz * bpz));
    const float vc = fmaf(d1, d4, -d3 * d2);
    if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
        const float v = __fdividef(d1, d1 - d3);
        const float dx = apx - v * abx, dy = apy - v * aby, dz = apz - v * abz;
        return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    }
    const float cpx = px - cx, cpy = py - cy, cpz = pz - cz;
    const float d5 = fmaf(abx, cpx, fmaf(aby, cpy, abz * cpz));
    const float d6 = fmaf(acx, cpx, fmaf(acy, cpy, acz * cpz));
    if (d6 >= 0.f && d5 <= d6) return fmaf(cpx, cpx, fmaf(cpy, cpy, cpz * cpz));
    const float vb = fmaf(d5, d2, -d1 * d6);
    if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
        const float w = __fdividef(d2, d2 - d6);
        const float dx = apx - w * acx, dy = apy - w * acy, dz = apz - w * acz;
        return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    }
    const float va = fmaf(d3, d6, -d5 * d4);
    if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
        const float w = __fdividef(d4 - d3, (d4 - d3) + (d5 - d6));
        const float dx = bpx - w * (cx - bx), dy = bpy - w * (cy - by), dz = bpz - w * (cz - bz);
        return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    }
    const float denom = __frcp_rn(va + vb + vc);
    const float v = vb * denom;
    const float w = vc * denom;
    const float dx = apx - fmaf(abx, v, acx * w);
    const float dy = apy - fmaf(aby, v, acy * w);
    const float dz = apz - fmaf(abz, v, acz * w);
    return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
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
