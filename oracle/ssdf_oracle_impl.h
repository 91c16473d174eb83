/*
 * ssdf_oracle_impl.h -- the per-precision body of the CPU oracle, included twice by
 * ssdf_oracle.c (REAL = double, SUF = _d; REAL = float, SUF = _f).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library, never part of it.
 *
 * Each routine restates one zulianp/ssdf routine with the same expression order and the
 * same branch tests. ssdf builds as C++17 without GNU extensions, so GCC compiles it with
 * -ffp-contract=off and (x86-64) SSE arithmetic: no fused multiply-add, no excess precision.
 * This file is compiled the same way, so its double results are bitwise ssdf's.
 */

#ifndef REAL
#error "define REAL and SUF before including ssdf_oracle_impl.h"
#endif

#define OR_CAT2(a, b) a##b
#define OR_CAT(a, b) OR_CAT2(a, b)
#define OR_NAME(n) OR_CAT(n, SUF)

/* Squared distance from p to triangle (a, b, c): Ericson's Voronoi-region walk
 * (Real-Time Collision Detection, 5.1.5). Follows serial/ssdf.hpp:49-121 term by term. */
REAL OR_NAME(oracle_point_triangle_dist_sq)(const REAL px, const REAL py, const REAL pz,
                                            const REAL ax, const REAL ay, const REAL az,
                                            const REAL bx, const REAL by, const REAL bz,
                                            const REAL cx, const REAL cy, const REAL cz) {
    const REAL abx = bx - ax, aby = by - ay, abz = bz - az;
    const REAL acx = cx - ax, acy = cy - ay, acz = cz - az;
    const REAL apx = px - ax, apy = py - ay, apz = pz - az;

    const REAL d1 = abx * apx + aby * apy + abz * apz;
    const REAL d2 = acx * apx + acy * apy + acz * apz;
    if (d1 <= (REAL)0 && d2 <= (REAL)0) return apx * apx + apy * apy + apz * apz;

    const REAL bpx = px - bx, bpy = py - by, bpz = pz - bz;
    const REAL d3 = abx * bpx + aby * bpy + abz * bpz;
    const REAL d4 = acx * bpx + acy * bpy + acz * bpz;
    if (d3 >= (REAL)0 && d4 <= d3) return bpx * bpx + bpy * bpy + bpz * bpz;

    const REAL vc = d1 * d4 - d3 * d2;
    if (vc <= (REAL)0 && d1 >= (REAL)0 && d3 <= (REAL)0) {
        const REAL v = d1 / (d1 - d3);
        const REAL qx = ax + v * abx, qy = ay + v * aby, qz = az + v * abz;
        const REAL dx = px - qx, dy = py - qy, dz = pz - qz;
        return dx * dx + dy * dy + dz * dz;
    }

    const REAL cpx = px - cx, cpy = py - cy, cpz = pz - cz;
    const REAL d5 = abx * cpx + aby * cpy + abz * cpz;
    const REAL d6 = acx * cpx + acy * cpy + acz * cpz;
    if (d6 >= (REAL)0 && d5 <= d6) return cpx * cpx + cpy * cpy + cpz * cpz;

    const REAL vb = d5 * d2 - d1 * d6;
    if (vb <= (REAL)0 && d2 >= (REAL)0 && d6 <= (REAL)0) {
        const REAL w = d2 / (d2 - d6);
        const REAL qx = ax + w * acx, qy = ay + w * acy, qz = az + w * acz;
        const REAL dx = px - qx, dy = py - qy, dz = pz - qz;
        return dx * dx + dy * dy + dz * dz;
    }

    const REAL va = d3 * d6 - d5 * d4;
    if (va <= (REAL)0 && (d4 - d3) >= (REAL)0 && (d5 - d6) >= (REAL)0) {
        const REAL w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        const REAL qx = bx + w * (cx - bx), qy = by + w * (cy - by), qz = bz + w * (cz - bz);
        const REAL dx = px - qx, dy = py - qy, dz = pz - qz;
        return dx * dx + dy * dy + dz * dz;
    }

    const REAL denom = (REAL)1 / (va + vb + vc);
    const REAL v = vb * denom;
    const REAL w = vc * denom;
    const REAL qx = ax + abx * v + acx * w;
    const REAL qy = ay + aby * v + acy * w;
    const REAL qz = az + abz * v + acz * w;
    const REAL dx = px - qx, dy = py - qy, dz = pz - qz;
    return dx * dx + dy * dy + dz * dz;
}

/* The closest point itself, same regions: serial/ssdf.hpp:143-239. */
void OR_NAME(oracle_point_triangle_closest_point)(const REAL px, const REAL py, const REAL pz,
                                                  const REAL ax, const REAL ay, const REAL az,
                                                  const REAL bx, const REAL by, const REAL bz,
                                                  const REAL cx, const REAL cy, const REAL cz,
                                                  REAL *outx, REAL *outy, REAL *outz) {
    const REAL abx = bx - ax, aby = by - ay, abz = bz - az;
    const REAL acx = cx - ax, acy = cy - ay, acz = cz - az;
    const REAL apx = px - ax, apy = py - ay, apz = pz - az;

    const REAL d1 = abx * apx + aby * apy + abz * apz;
    const REAL d2 = acx * apx + acy * apy + acz * apz;
    if (d1 <= (REAL)0 && d2 <= (REAL)0) {
        *outx = ax, *outy = ay, *outz = az;
        return;
    }

    const REAL bpx = px - bx, bpy = py - by, bpz = pz - bz;
    const REAL d3 = abx * bpx + aby * bpy + abz * bpz;
    const REAL d4 = acx * bpx + acy * bpy + acz * bpz;
    if (d3 >= (REAL)0 && d4 <= d3) {
        *outx = bx, *outy = by, *outz = bz;
        return;
    }

    const REAL vc = d1 * d4 - d3 * d2;
    if (vc <= (REAL)0 && d1 >= (REAL)0 && d3 <= (REAL)0) {
        const REAL v = d1 / (d1 - d3);
        *outx = ax + v * abx, *outy = ay + v * aby, *outz = az + v * abz;
        return;
    }

    const REAL cpx = px - cx, cpy = py - cy, cpz = pz - cz;
    const REAL d5 = abx * cpx + aby * cpy + abz * cpz;
    const REAL d6 = acx * cpx + acy * cpy + acz * cpz;
    if (d6 >= (REAL)0 && d5 <= d6) {
        *outx = cx, *outy = cy, *outz = cz;
        return;
    }

    const REAL vb = d5 * d2 - d1 * d6;
    if (vb <= (REAL)0 && d2 >= (REAL)0 && d6 <= (REAL)0) {
        const REAL w = d2 / (d2 - d6);
        *outx = ax + w * acx, *outy = ay + w * acy, *outz = az + w * acz;
        return;
    }

    const REAL va = d3 * d6 - d5 * d4;
    if (va <= (REAL)0 && (d4 - d3) >= (REAL)0 && (d5 - d6) >= (REAL)0) {
        const REAL w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        const REAL bcx = cx - bx, bcy = cy - by, bcz = cz - bz;
        *outx = bx + w * bcx, *outy = by + w * bcy, *outz = bz + w * bcz;
        return;
    }

    const REAL denom = (REAL)1 / (va + vb + vc);
    const REAL v = vb * denom;
    const REAL w = vc * denom;
    *outx = ax + abx * v + acx * w;
    *outy = ay + aby * v + acy * w;
    *outz = az + abz * v + acz * w;
}

/* Point-box squared distance: serial/edf/edf.hpp:55-69. */
REAL OR_NAME(oracle_point_aabb_distance_squared)(const REAL px, const REAL py, const REAL pz,
                                                 const REAL minx, const REAL maxx,
                                                 const REAL miny, const REAL maxy,
                                                 const REAL minz, const REAL maxz) {
    const REAL dx = (px < minx) ? (minx - px) : (px > maxx ? px - maxx : (REAL)0);
    const REAL dy = (py < miny) ? (miny - py) : (py > maxy ? py - maxy : (REAL)0);
    const REAL dz = (pz < minz) ? (minz - pz) : (pz > maxz ? pz - maxz : (REAL)0);
    return dx * dx + dy * dy + dz * dz;
}

/* Signed distance to a box, negative inside: serial/edf/edf.hpp:193-221. */
REAL OR_NAME(oracle_point_aabb_signed_distance)(const REAL px, const REAL py, const REAL pz,
                                                const REAL minx, const REAL maxx,
                                                const REAL miny, const REAL maxy,
                                                const REAL minz, const REAL maxz) {
    const REAL hx = (maxx - minx) * (REAL)0.5;
    const REAL hy = (maxy - miny) * (REAL)0.5;
    const REAL hz = (maxz - minz) * (REAL)0.5;
    const REAL cx = (maxx + minx) * (REAL)0.5;
    const REAL cy = (maxy + miny) * (REAL)0.5;
    const REAL cz = (maxz + minz) * (REAL)0.5;
    const REAL qx = OR_ABS(px - cx) - hx;
    const REAL qy = OR_ABS(py - cy) - hy;
    const REAL qz = OR_ABS(pz - cz) - hz;
    const REAL ox = qx > (REAL)0 ? qx : (REAL)0;
    const REAL oy = qy > (REAL)0 ? qy : (REAL)0;
    const REAL oz = qz > (REAL)0 ? qz : (REAL)0;
    const REAL outside = OR_SQRT(ox * ox + oy * oy + oz * oz);
    /* std::max(qx, std::max(qy, qz)) then std::min<T>(0, .) */
    const REAL myz = (qy < qz) ? qz : qy;
    const REAL mxyz = (qx < myz) ? myz : qx;
    const REAL inside = (mxyz < (REAL)0) ? mxyz : (REAL)0;
    return outside + inside;
}

/* Bounding box of n >= 1 points as six extremes (xmin, xmax, ymin, ymax, zmin, zmax): the scalar
 * reduction of serial/edf/edf.hpp:500-539 with std::min(m, v) = (v < m ? v : m), seeded with the
 * first point. */
void OR_NAME(oracle_compute_aabb)(const ptrdiff_t n, const REAL *x, const REAL *y, const REAL *z, REAL *box6) {
    REAL b[6] = {x[0], x[0], y[0], y[0], z[0], z[0]};
    for (ptrdiff_t i = 0; i < n; i++) {
        b[0] = x[i] < b[0] ? x[i] : b[0];
        b[1] = b[1] < x[i] ? x[i] : b[1];
        b[2] = y[i] < b[2] ? y[i] : b[2];
        b[3] = b[3] < y[i] ? y[i] : b[3];
        b[4] = z[i] < b[4] ? z[i] : b[4];
        b[5] = b[5] < z[i] ? z[i] : b[5];
    }
    for (int k = 0; k < 6; k++) box6[k] = b[k];
}

/* out[i] = signed distance of point i to box6 (minx, maxx, miny, maxy, minz, maxz):
 * serial/edf/edf.hpp:541-557. */
void OR_NAME(oracle_all_points_aabb_signed_distance)(const ptrdiff_t n, const REAL *x, const REAL *y,
                                                     const REAL *z, const REAL *box6, REAL *out) {
    for (ptrdiff_t i = 0; i < n; i++)
        out[i] = OR_NAME(oracle_point_aabb_signed_distance)(x[i], y[i], z[i], box6[0], box6[1], box6[2], box6[3],
                                                            box6[4], box6[5]);
}

/*
 * Unsigned distance with the in/out `out` of ssdf::edf / edf_celllist
 * (serial/ssdf.hpp:447-619, 642-963): on entry out[p] is the current best distance, on exit
 * out[p] = sqrt(min(out[p]*out[p], min_t d2(p, t))). Both reference routines prune only boxes
 * that cannot improve, so their value is this brute-force minimum; the oracle evaluates every
 * triangle. The closest-triangle index is this build's addition (serial/bvh/bvh.cpp:125-197
 * is the pattern): the lowest index among triangles whose d2 equals the minimum, written to
 * outtri[p] only when some triangle improves on the incoming value (strictly), as
 * closest_point_bvh does. outtri may be NULL. An empty mesh leaves out untouched
 * (serial/ssdf.hpp:462).
 */
int OR_NAME(oracle_edf)(const ptrdiff_t npoints, const REAL *x, const REAL *y, const REAL *z,
                        const ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                        const ptrdiff_t nspoints, const REAL *sx, const REAL *sy, const REAL *sz,
                        REAL *out, int *outtri) {
    if (nselements == 0 || nspoints == 0) return 0;
#pragma omp parallel for schedule(dynamic, 64)
    for (ptrdiff_t p = 0; p < npoints; p++) {
        const REAL px = x[p], py = y[p], pz = z[p];
        REAL best = out[p] * out[p];
        int bt = -1;
        for (ptrdiff_t t = 0; t < nselements; t++) {
            const int i0 = s0[t], i1 = s1[t], i2 = s2[t];
            const REAL d2 = OR_NAME(oracle_point_triangle_dist_sq)(px, py, pz, sx[i0], sy[i0], sz[i0],
                                                                 sx[i1], sy[i1], sz[i1], sx[i2], sy[i2], sz[i2]);
            if (d2 < best) {
                best = d2;
                bt = (int)t;
            }
        }
        out[p] = OR_SQRT(best);
        if (outtri && bt >= 0) outtri[p] = bt;
    }
    return 0;
}

/*
 * Node-grid coordinates in the reference's G precision (serial/bvh/bvh.cpp:1665-1667, 1744):
 * h = (max - min) / (n - 1) (0 when n == 1), q = min + i * h evaluated in REAL, then widened to
 * double; point index i + j * nx + k * nx * ny (x fastest).
 */
void OR_NAME(oracle_grid_points)(const ptrdiff_t nx, const ptrdiff_t ny, const ptrdiff_t nz,
                                 const REAL xmin, const REAL ymin, const REAL zmin,
                                 const REAL xmax, const REAL ymax, const REAL zmax,
                                 double *qx, double *qy, double *qz) {
    const REAL hx = (nx > 1) ? (xmax - xmin) / (REAL)(nx - 1) : (REAL)0;
    const REAL hy = (ny > 1) ? (ymax - ymin) / (REAL)(ny - 1) : (REAL)0;
    const REAL hz = (nz > 1) ? (zmax - zmin) / (REAL)(nz - 1) : (REAL)0;
    for (ptrdiff_t k = 0; k < nz; k++)
        for (ptrdiff_t j = 0; j < ny; j++)
            for (ptrdiff_t i = 0; i < nx; i++) {
                const ptrdiff_t id = i + j * nx + k * nx * ny;
                qx[id] = (double)(xmin + (REAL)i * hx);
                qy[id] = (double)(ymin + (REAL)j * hy);
                qz[id] = (double)(zmin + (REAL)k * hz);
            }
}

#undef OR_NAME
#undef OR_CAT
#undef OR_CAT2
