/*
 * Test support (not part of the library): checks the FP32 filter of the fix-up path against the error
 * bound its window is sized from. The filter (ssdf_b200/csrc/device_geom.cuh, tri_dist_sq_filter) is
 * restated here in C, in its region order (corners A, B, C, then the edges, then the face), with
 * fmaf, an IEEE reciprocal for __frcp_rn and, for __fdividef, the exact
 * quotient rounded and then moved by -2, 0 and +2 ulp (its documented worst case), the largest error
 * of the three taken. The record is built as mesh_build.cu's filter_record builds a well-conditioned
 * triangle's (float corners, edges rounded once, products in double rounded once).
 *
 * For each case the error |sqrt(key) - dist| against the double distance of the record's triangle is
 * compared with the bound
 *     u (8 R + 7.7 alpha L) + min(D, 2 D^2 / d),   D = 90 u alpha R,   u = 2^-24,
 * R the largest distance from the point to a corner, L the longest edge, alpha = L / smallest altitude.
 * Prints the largest error / bound and the largest error / (u R) near the triangle (d <= L).
 *
 * Usage: filter_bound_check <cases> <seed>
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

typedef struct {
    float ax, ay, az, abx, aby, abz, acx, acy, acz, abab, acac, abac;
} Rec;

static int g_shift = 0; /* ulps added to each quotient */

static float quot(float x, float y) {
    float q = (float)((double)x / (double)y);
    for (int k = 0; k < abs(g_shift); k++) q = nextafterf(q, g_shift > 0 ? INFINITY : -INFINITY);
    return q;
}

static float filter(float px, float py, float pz, const Rec *r) {
    const float apx = px - r->ax, apy = py - r->ay, apz = pz - r->az;
    const float d1 = fmaf(r->abx, apx, fmaf(r->aby, apy, r->abz * apz));
    const float d2 = fmaf(r->acx, apx, fmaf(r->acy, apy, r->acz * apz));
    if (d1 <= 0.f && d2 <= 0.f) return fmaf(apx, apx, fmaf(apy, apy, apz * apz));
    const float d3 = d1 - r->abab, d4 = d2 - r->abac;
    if (d3 >= 0.f && d4 <= d3) {
        const float bx = apx - r->abx, by = apy - r->aby, bz = apz - r->abz;
        return fmaf(bx, bx, fmaf(by, by, bz * bz));
    }
    const float d5 = d1 - r->abac, d6 = d2 - r->acac;
    if (d6 >= 0.f && d5 <= d6) {
        const float cx = apx - r->acx, cy = apy - r->acy, cz = apz - r->acz;
        return fmaf(cx, cx, fmaf(cy, cy, cz * cz));
    }
    const float vc = fmaf(d1, d4, -d3 * d2);
    if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
        const float v = quot(d1, d1 - d3);
        const float dx = fmaf(-v, r->abx, apx), dy = fmaf(-v, r->aby, apy), dz = fmaf(-v, r->abz, apz);
        return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    }
    const float vb = fmaf(d5, d2, -d1 * d6);
    if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
        const float w = quot(d2, d2 - d6);
        const float dx = fmaf(-w, r->acx, apx), dy = fmaf(-w, r->acy, apy), dz = fmaf(-w, r->acz, apz);
        return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    }
    const float va = fmaf(d3, d6, -d5 * d4);
    if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
        const float w = quot(d4 - d3, (d4 - d3) + (d5 - d6));
        const float dx = fmaf(-w, r->acx - r->abx, apx - r->abx);
        const float dy = fmaf(-w, r->acy - r->aby, apy - r->aby);
        const float dz = fmaf(-w, r->acz - r->abz, apz - r->abz);
        return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    }
    const float nx = fmaf(r->aby, r->acz, -r->abz * r->acy);
    const float ny = fmaf(r->abz, r->acx, -r->abx * r->acz);
    const float nz = fmaf(r->abx, r->acy, -r->aby * r->acx);
    const float nq = fmaf(nx, apx, fmaf(ny, apy, nz * apz));
    const float nn = fmaf(nx, nx, fmaf(ny, ny, nz * nz));
    return nq * (nq * (1.0f / nn));
}

/* Closest-point distance in double, by projecting on the plane and clamping to edges and corners. */
static double seg_dist2(const double p[3], const double a[3], const double b[3]) {
    double ab[3], ap[3], t = 0, l = 0, d2 = 0;
    for (int k = 0; k < 3; k++) ab[k] = b[k] - a[k], ap[k] = p[k] - a[k], t += ab[k] * ap[k], l += ab[k] * ab[k];
    t = l > 0 ? fmin(fmax(t / l, 0.0), 1.0) : 0.0;
    for (int k = 0; k < 3; k++) {
        const double e = ap[k] - t * ab[k];
        d2 += e * e;
    }
    return d2;
}

static double tri_dist(const double p[3], const double a[3], const double b[3], const double c[3]) {
    double e1[3], e2[3], n[3], ap[3];
    for (int k = 0; k < 3; k++) e1[k] = b[k] - a[k], e2[k] = c[k] - a[k], ap[k] = p[k] - a[k];
    n[0] = e1[1] * e2[2] - e1[2] * e2[1], n[1] = e1[2] * e2[0] - e1[0] * e2[2], n[2] = e1[0] * e2[1] - e1[1] * e2[0];
    const double nn = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
    const double s11 = e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2], s22 = e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2];
    const double s12 = e1[0] * e2[0] + e1[1] * e2[1] + e1[2] * e2[2];
    const double r1 = e1[0] * ap[0] + e1[1] * ap[1] + e1[2] * ap[2], r2 = e2[0] * ap[0] + e2[1] * ap[1] + e2[2] * ap[2];
    const double det = s11 * s22 - s12 * s12;
    if (det > 0) {
        const double v = (s22 * r1 - s12 * r2) / det, w = (s11 * r2 - s12 * r1) / det;
        if (v >= 0 && w >= 0 && v + w <= 1) {
            const double h = (n[0] * ap[0] + n[1] * ap[1] + n[2] * ap[2]);
            return fabs(h) / sqrt(nn);
        }
    }
    double d2 = seg_dist2(p, a, b);
    d2 = fmin(d2, seg_dist2(p, a, c));
    d2 = fmin(d2, seg_dist2(p, b, c));
    return sqrt(d2);
}

static uint64_t g_rng;
static double urand(void) {
    g_rng ^= g_rng << 13;
    g_rng ^= g_rng >> 7;
    g_rng ^= g_rng << 17;
    return (double)(g_rng >> 11) * (1.0 / 9007199254740992.0);
}
static double nrand(void) { return sqrt(-2.0 * log(urand() + 1e-300)) * cos(6.283185307179586 * urand()); }

int main(int argc, char **argv) {
    const long cases = argc > 1 ? atol(argv[1]) : 200000;
    g_rng = 0x9E3779B97F4A7C15ull ^ (uint64_t)(argc > 2 ? atol(argv[2]) : 1);
    const double u = ldexp(1.0, -24);
    double worst = 0, worst_near = 0;
    long used = 0;
    for (long it = 0; it < cases; it++) {
        /* a triangle of size `scale` at an offset up to 1e7, altitude 1/8 .. 1 of its base */
        const double off = urand() < 0.5 ? 0.0 : pow(10.0, urand() * 8 - 1);
        const double scale = pow(10.0, urand() * 6 - 3);
        const double o[3] = {off + nrand() * scale, 0.3 * off + nrand() * scale, -0.7 * off + nrand() * scale};
        double e1[3] = {nrand(), nrand(), nrand()}, t[3] = {nrand(), nrand(), nrand()}, e2[3];
        const double l1 = sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
        for (int k = 0; k < 3; k++) e1[k] *= scale / l1;
        const double te = (t[0] * e1[0] + t[1] * e1[1] + t[2] * e1[2]) / (scale * scale);
        for (int k = 0; k < 3; k++) t[k] -= te * e1[k];
        const double lt = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
        const double height = scale * (0.125 + 0.875 * urand()), along = 1.4 * urand() - 0.2;
        for (int k = 0; k < 3; k++) e2[k] = along * e1[k] + height * t[k] / lt;
        float f[3][3];
        for (int k = 0; k < 3; k++) f[0][k] = (float)o[k], f[1][k] = (float)(o[k] + e1[k]), f[2][k] = (float)(o[k] + e2[k]);
        double eb[3], ec[3];
        for (int k = 0; k < 3; k++) eb[k] = (double)f[1][k] - f[0][k], ec[k] = (double)f[2][k] - f[0][k];
        Rec r = {f[0][0], f[0][1], f[0][2], (float)eb[0], (float)eb[1], (float)eb[2], (float)ec[0], (float)ec[1],
                 (float)ec[2], (float)(eb[0] * eb[0] + eb[1] * eb[1] + eb[2] * eb[2]),
                 (float)(ec[0] * ec[0] + ec[1] * ec[1] + ec[2] * ec[2]), (float)(eb[0] * ec[0] + eb[1] * ec[1] + eb[2] * ec[2])};
        /* the record's triangle, exactly (float values in double) */
        const double A[3] = {r.ax, r.ay, r.az};
        const double B[3] = {A[0] + (double)r.abx, A[1] + (double)r.aby, A[2] + (double)r.abz};
        const double C[3] = {A[0] + (double)r.acx, A[1] + (double)r.acy, A[2] + (double)r.acz};
        double E1[3], E2[3], E3[3], n[3];
        for (int k = 0; k < 3; k++) E1[k] = B[k] - A[k], E2[k] = C[k] - A[k], E3[k] = C[k] - B[k];
        n[0] = E1[1] * E2[2] - E1[2] * E2[1], n[1] = E1[2] * E2[0] - E1[0] * E2[2], n[2] = E1[0] * E2[1] - E1[1] * E2[0];
        const double area2 = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        const double L2 = fmax(fmax(E1[0] * E1[0] + E1[1] * E1[1] + E1[2] * E1[2], E2[0] * E2[0] + E2[1] * E2[1] + E2[2] * E2[2]),
                               E3[0] * E3[0] + E3[1] * E3[1] + E3[2] * E3[2]);
        /* records rounding made degenerate or ill-conditioned are not filtered (proxies, or FP64) */
        if (!(area2 > 0) || !(64.0 * area2 * area2 >= L2 * L2)) continue;
        const double L = sqrt(L2), alpha = L2 / area2;
        /* a point near the face, an edge, a corner, or anywhere, off the plane by 0 .. 1e3 scale */
        double bv, bw;
        const int kind = (int)(urand() * 4);
        if (kind == 0) bv = urand(), bw = urand() * (1 - bv);
        else if (kind == 1) bv = urand(), bw = 1 - bv + (urand() - 0.5) * 1e-3;
        else if (kind == 2) bv = (urand() - 0.5) * 1e-3, bw = (urand() - 0.5) * 1e-3;
        else bv = 3 * urand() - 1, bw = 3 * urand() - 1;
        const double normal = urand() < 0.5 ? 0.0 : pow(10.0, urand() * 9 - 6) * scale * (urand() < 0.5 ? 1 : -1);
        const double jitter = urand() < 0.5 ? 0.0 : pow(10.0, urand() * 9 - 6) * scale;
        float P[3];
        for (int k = 0; k < 3; k++)
            P[k] = (float)(A[k] + bv * E1[k] + bw * E2[k] + normal * n[k] / area2 + jitter * nrand());
        const double p[3] = {P[0], P[1], P[2]};
        const double dist = tri_dist(p, A, B, C);
        double R = 0;
        for (int c = 0; c < 3; c++) {
            const double *V = c == 0 ? A : (c == 1 ? B : C);
            R = fmax(R, sqrt((p[0] - V[0]) * (p[0] - V[0]) + (p[1] - V[1]) * (p[1] - V[1]) + (p[2] - V[2]) * (p[2] - V[2])));
        }
        double err = 0;
        for (g_shift = -2; g_shift <= 2; g_shift += 2) {
            const float key = filter(P[0], P[1], P[2], &r);
            const double e = fabs(sqrt((double)key) - dist);
            err = e == e ? fmax(err, e) : INFINITY;
        }
        const double D = 90.0 * u * alpha * R;
        const double bound = u * (8.0 * R + 7.7 * alpha * L) + fmin(D, dist > 0 ? 2.0 * D * D / dist : D);
        worst = fmax(worst, err / bound);
        if (dist <= L) worst_near = fmax(worst_near, err / (u * R));
        used++;
    }
    printf("cases %ld worst_error_over_bound %.6f worst_near_error_over_uR %.4f\n", used, worst, worst_near);
    return 0;
}
