/*
 * ssdf_oracle_contact_prim.h -- point-segment, point-triangle (barycentric) and point-quad
 * closest points in REAL; included by ssdf_oracle_contact.c once per REAL. Every expression is
 * evaluated in the order written, one rounding per operation, as the reference's C++ templates
 * are (C++17, no FMA contraction).
 */

#define OC_CAT2(a, b) a##b
#define OC_CAT(a, b) OC_CAT2(a, b)
#define OC_NAME(n) OC_CAT(n, SUF)

/* Squared distance from q to segment ab and the clamped parameter u of the closest point
 * a + u (b - a): serial/edf/edf.hpp:222-249. A zero-length segment gives u = 0. The clamp is
 * std::clamp's (a NaN parameter stays NaN). */
static REAL OC_NAME(oc_segment)(const REAL qx, const REAL qy, const REAL qz, const REAL ax, const REAL ay,
                                const REAL az, const REAL bx, const REAL by, const REAL bz, REAL *u_out) {
    const REAL ex = bx - ax, ey = by - ay, ez = bz - az;
    const REAL fx = qx - ax, fy = qy - ay, fz = qz - az;
    const REAL len2 = ex * ex + ey * ey + ez * ez;
    REAL u = (REAL)0;
    if (len2 > (REAL)0) {
        const REAL r = (fx * ex + fy * ey + fz * ez) / len2;
        u = r < (REAL)0 ? (REAL)0 : ((REAL)1 < r ? (REAL)1 : r);
    }
    const REAL px = ax + u * ex, py = ay + u * ey, pz = az + u * ez;
    const REAL dx = qx - px, dy = qy - py, dz = qz - pz;
    *u_out = u;
    return dx * dx + dy * dy + dz * dz;
}

/* Squared distance from q to triangle abc and the barycentric weights (wa, wb, wc) of the
 * closest point: serial/edf/edf.hpp:251-386. A triangle whose squared normal is at most
 * 64 eps (longest squared edge)^2 is treated as its three edges, ab then bc then ca, the first
 * strictly smaller distance winning; otherwise Ericson's Voronoi regions (vertex a, vertex b,
 * edge ab, vertex c, edge ac, edge bc, face). */
REAL OC_NAME(oracle_point_triangle_barycentric)(const REAL qx, const REAL qy, const REAL qz, const REAL ax,
                                                const REAL ay, const REAL az, const REAL bx, const REAL by,
                                                const REAL bz, const REAL cx, const REAL cy, const REAL cz,
                                                REAL *wa, REAL *wb, REAL *wc) {
    const REAL abx = bx - ax, aby = by - ay, abz = bz - az;
    const REAL acx = cx - ax, acy = cy - ay, acz = cz - az;
    const REAL bcx = cx - bx, bcy = cy - by, bcz = cz - bz;
    const REAL lab = abx * abx + aby * aby + abz * abz;
    const REAL lac = acx * acx + acy * acy + acz * acz;
    const REAL lbc = bcx * bcx + bcy * bcy + bcz * bcz;
    const REAL nx = aby * acz - abz * acy;
    const REAL ny = abz * acx - abx * acz;
    const REAL nz = abx * acy - aby * acx;
    const REAL inner = lac < lbc ? lbc : lac; /* std::max(ac2, bc2) */
    const REAL lmax = lab < inner ? inner : lab;
    const REAL n2 = nx * nx + ny * ny + nz * nz;

    if (lmax <= (REAL)0 || n2 <= OR_EPS * (REAL)64 * lmax * lmax) {
        REAL u;
        REAL best = OC_NAME(oc_segment)(qx, qy, qz, ax, ay, az, bx, by, bz, &u);
        *wa = (REAL)1 - u, *wb = u, *wc = (REAL)0;
        REAL d = OC_NAME(oc_segment)(qx, qy, qz, bx, by, bz, cx, cy, cz, &u);
        if (d < best) best = d, *wa = (REAL)0, *wb = (REAL)1 - u, *wc = u;
        d = OC_NAME(oc_segment)(qx, qy, qz, cx, cy, cz, ax, ay, az, &u);
        if (d < best) best = d, *wa = u, *wb = (REAL)0, *wc = (REAL)1 - u;
        return best;
    }

    const REAL aqx = qx - ax, aqy = qy - ay, aqz = qz - az;
    const REAL d1 = abx * aqx + aby * aqy + abz * aqz;
    const REAL d2 = acx * aqx + acy * aqy + acz * aqz;
    if (d1 <= (REAL)0 && d2 <= (REAL)0) {
        *wa = (REAL)1, *wb = (REAL)0, *wc = (REAL)0;
        return aqx * aqx + aqy * aqy + aqz * aqz;
    }

    const REAL bqx = qx - bx, bqy = qy - by, bqz = qz - bz;
    const REAL d3 = abx * bqx + aby * bqy + abz * bqz;
    const REAL d4 = acx * bqx + acy * bqy + acz * bqz;
    if (d3 >= (REAL)0 && d4 <= d3) {
        *wa = (REAL)0, *wb = (REAL)1, *wc = (REAL)0;
        return bqx * bqx + bqy * bqy + bqz * bqz;
    }

    const REAL vc = d1 * d4 - d3 * d2;
    if (vc <= (REAL)0 && d1 >= (REAL)0 && d3 <= (REAL)0) {
        const REAL v = d1 / (d1 - d3);
        const REAL dx = qx - (ax + v * abx), dy = qy - (ay + v * aby), dz = qz - (az + v * abz);
        *wa = (REAL)1 - v, *wb = v, *wc = (REAL)0;
        return dx * dx + dy * dy + dz * dz;
    }

    const REAL cqx = qx - cx, cqy = qy - cy, cqz = qz - cz;
    const REAL d5 = abx * cqx + aby * cqy + abz * cqz;
    const REAL d6 = acx * cqx + acy * cqy + acz * cqz;
    if (d6 >= (REAL)0 && d5 <= d6) {
        *wa = (REAL)0, *wb = (REAL)0, *wc = (REAL)1;
        return cqx * cqx + cqy * cqy + cqz * cqz;
    }

    const REAL vb = d5 * d2 - d1 * d6;
    if (vb <= (REAL)0 && d2 >= (REAL)0 && d6 <= (REAL)0) {
        const REAL w = d2 / (d2 - d6);
        const REAL dx = qx - (ax + w * acx), dy = qy - (ay + w * acy), dz = qz - (az + w * acz);
        *wa = (REAL)1 - w, *wb = (REAL)0, *wc = w;
        return dx * dx + dy * dy + dz * dz;
    }

    const REAL va = d3 * d6 - d5 * d4;
    if (va <= (REAL)0 && (d4 - d3) >= (REAL)0 && (d5 - d6) >= (REAL)0) {
        const REAL w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        const REAL dx = qx - (bx + w * bcx), dy = qy - (by + w * bcy), dz = qz - (bz + w * bcz);
        *wa = (REAL)0, *wb = (REAL)1 - w, *wc = w;
        return dx * dx + dy * dy + dz * dz;
    }

    const REAL inv = (REAL)1 / (va + vb + vc);
    const REAL v = vb * inv;
    const REAL w = vc * inv;
    const REAL dx = qx - (ax + abx * v + acx * w);
    const REAL dy = qy - (ay + aby * v + acy * w);
    const REAL dz = qz - (az + abz * v + acz * w);
    *wa = (REAL)1 - v - w, *wb = v, *wc = w;
    return dx * dx + dy * dy + dz * dz;
}

/* Bilinear parameters (s, t) in [0, 1]^2 of the point of quad v0 v1 v2 v3 closest to p:
 * serial/edf/edf.hpp:388-489. The quad is split along the diagonal 0-2 when it is convex in
 * the projection that drops the dominant axis of its Newell normal (or, when that projected
 * area is within 64 eps of zero, when 0-2 is the shorter diagonal), else along 1-3; each half
 * is solved with the triangle routine above and the strictly closer half wins, its weights
 * mapped to (s, t) and clamped. */
void OC_NAME(oracle_point_to_quad_closest_point)(const REAL px, const REAL py, const REAL pz, const REAL x0,
                                                 const REAL y0, const REAL z0, const REAL x1, const REAL y1,
                                                 const REAL z1, const REAL x2, const REAL y2, const REAL z2,
                                                 const REAL x3, const REAL y3, const REAL z3, REAL *s, REAL *t) {
    /* Newell normal, four edge terms each */
    const REAL gx = (y0 - y1) * (z0 + z1) + (y1 - y2) * (z1 + z2) + (y2 - y3) * (z2 + z3) + (y3 - y0) * (z3 + z0);
    const REAL gy = (z0 - z1) * (x0 + x1) + (z1 - z2) * (x1 + x2) + (z2 - z3) * (x2 + x3) + (z3 - z0) * (x3 + x0);
    const REAL gz = (x0 - x1) * (y0 + y1) + (x1 - x2) * (y1 + y2) + (x2 - x3) * (y2 + y3) + (x3 - x0) * (y3 + y0);
    const REAL ax_ = OR_ABS(gx), ay_ = OR_ABS(gy), az_ = OR_ABS(gz);
    REAL u[4], v[4];
    if (ax_ >= ay_ && ax_ >= az_) {
        u[0] = y0, v[0] = z0, u[1] = y1, v[1] = z1, u[2] = y2, v[2] = z2, u[3] = y3, v[3] = z3;
    } else if (ay_ >= az_) {
        u[0] = x0, v[0] = z0, u[1] = x1, v[1] = z1, u[2] = x2, v[2] = z2, u[3] = x3, v[3] = z3;
    } else {
        u[0] = x0, v[0] = y0, u[1] = x1, v[1] = y1, u[2] = x2, v[2] = y2, u[3] = x3, v[3] = y3;
    }
    /* twice the signed projected area (shoelace, term by term) and the turns at corners 1 and 3 */
    const REAL area2 = u[0] * v[1] - v[0] * u[1] + u[1] * v[2] - v[1] * u[2] + u[2] * v[3] - v[2] * u[3] +
                       u[3] * v[0] - v[3] * u[0];
    const REAL turn1 = (u[1] - u[0]) * (v[2] - v[0]) - (v[1] - v[0]) * (u[2] - u[0]);
    const REAL turn3 = (u[3] - u[2]) * (v[0] - v[2]) - (v[3] - v[2]) * (u[0] - u[2]);

    int split02 = 1;
    if (OR_ABS(area2) > OR_EPS * (REAL)64) {
        const REAL sgn = area2 > (REAL)0 ? (REAL)1 : (REAL)-1;
        split02 = !(turn1 * sgn < (REAL)0 || turn3 * sgn < (REAL)0);
    } else {
        const REAL ex = x2 - x0, ey = y2 - y0, ez = z2 - z0;
        const REAL fx = x3 - x1, fy = y3 - y1, fz = z3 - z1;
        split02 = (ex * ex + ey * ey + ez * ez) <= (fx * fx + fy * fy + fz * fz);
    }

    REAL wa, wb, wc, s0, t0, s1, t1, d0, d1;
    if (split02) {
        d0 = OC_NAME(oracle_point_triangle_barycentric)(px, py, pz, x0, y0, z0, x1, y1, z1, x2, y2, z2, &wa, &wb,
                                                       &wc);
        s0 = wb + wc, t0 = wc;
        d1 = OC_NAME(oracle_point_triangle_barycentric)(px, py, pz, x0, y0, z0, x2, y2, z2, x3, y3, z3, &wa, &wb,
                                                       &wc);
        s1 = wb, t1 = wb + wc;
    } else {
        d0 = OC_NAME(oracle_point_triangle_barycentric)(px, py, pz, x0, y0, z0, x1, y1, z1, x3, y3, z3, &wa, &wb,
                                                       &wc);
        s0 = wb, t0 = wc;
        d1 = OC_NAME(oracle_point_triangle_barycentric)(px, py, pz, x1, y1, z1, x2, y2, z2, x3, y3, z3, &wa, &wb,
                                                       &wc);
        s1 = wa + wb, t1 = wb + wc;
    }
    if (d1 < d0) s0 = s1, t0 = t1;
    *s = s0 < (REAL)0 ? (REAL)0 : ((REAL)1 < s0 ? (REAL)1 : s0);
    *t = t0 < (REAL)0 ? (REAL)0 : ((REAL)1 < t0 ? (REAL)1 : t0);
}

/* Local coordinates (s, t) of p in triangle abc, p = a + s (b - a) + t (c - a) solved by the
 * normal equations: serial/bvh/bvh.cpp:60-83. */
void OC_NAME(oracle_triangle_local_st)(const REAL px, const REAL py, const REAL pz, const REAL ax, const REAL ay,
                                       const REAL az, const REAL bx, const REAL by, const REAL bz, const REAL cx,
                                       const REAL cy, const REAL cz, REAL *s, REAL *t) {
    const REAL ex = bx - ax, ey = by - ay, ez = bz - az;
    const REAL fx = cx - ax, fy = cy - ay, fz = cz - az;
    const REAL gx = px - ax, gy = py - ay, gz = pz - az;
    const REAL ee = ex * ex + ey * ey + ez * ez;
    const REAL ef = ex * fx + ey * fy + ez * fz;
    const REAL ff = fx * fx + fy * fy + fz * fz;
    const REAL ge = gx * ex + gy * ey + gz * ez;
    const REAL gf = gx * fx + gy * fy + gz * fz;
    const REAL inv = (REAL)1 / (ee * ff - ef * ef);
    *s = (ff * ge - ef * gf) * inv;
    *t = (ee * gf - ef * ge) * inv;
}

#undef OC_CAT2
#undef OC_CAT
#undef OC_NAME
