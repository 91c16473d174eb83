/*
 * ssdf_oracle_contact_query.h -- the brute-force closest-primitive-within-a-radius query for
 * coordinates GREAL and outputs TREAL; included by ssdf_oracle_contact.c once per (G, T).
 *
 * oracle_within_radius<SUF2>(..., s3, ..., local, ...) covers the four reference functions:
 *   s3 == NULL, local == 0: closest_within_radius_bvh        (serial/bvh/bvh.cpp:479-576)
 *   s3 == NULL, local != 0: closest_within_radius_local_bvh  (serial/bvh/bvh.cpp:367-477)
 *   s3 != NULL, local == 0: closest_within_radius_quads_bvh  (serial/bvh/bvh.cpp:578-706)
 *   s3 != NULL, local != 0: closest_within_radius_quads_local_bvh (serial/bvh/bvh.cpp:708-832)
 * Per point: the running squared distance starts at (float) radius_squared[pid * stride] and the
 * primitive -1; each primitive (skipped when skip_self and the point's index is one of its
 * corners) gives a float squared distance d2 that is kept when it is finite, at most the running
 * value, and (the tie rule of this build) not equal to a value already kept from a lower index.
 * Outputs: outtri = the primitive or -1; outd = the running value as TREAL; then either the float
 * closest point as TREAL (o0, o1, o2; zeros when none) or the local (s, t) (o0, o1; zeros when
 * none): for quads the bilinear parameters, for triangles triangle_local_coordinates_st in TREAL on
 * the float closest point and the corners converted to TREAL.
 */

#define OQ_CAT2(a, b) a##b
#define OQ_CAT(a, b) OQ_CAT2(a, b)
#define OQ_NAME(n) OQ_CAT(n, SUF2)

int OQ_NAME(oracle_within_radius)(const ptrdiff_t npoints, const GREAL *x, const GREAL *y, const GREAL *z,
                                  const ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                  const int *s3, const GREAL *sx, const GREAL *sy, const GREAL *sz,
                                  const ptrdiff_t stride, const TREAL *radius_squared, const int skip_self,
                                  const int local, int *outtri, TREAL *outd, TREAL *o0, TREAL *o1, TREAL *o2) {
#pragma omp parallel for schedule(dynamic, 64)
    for (ptrdiff_t pid = 0; pid < npoints; pid++) {
        const float qx = (float)x[pid], qy = (float)y[pid], qz = (float)z[pid];
        float best = (float)radius_squared[pid * stride];
        int bt = -1;
        float bx = 0.f, by = 0.f, bz = 0.f, bs = 0.f, bt_ = 0.f;
        for (ptrdiff_t e = 0; e < nselements; e++) {
            const int i0 = s0[e], i1 = s1[e], i2 = s2[e], i3 = s3 ? s3[e] : i2;
            if (skip_self && (pid == i0 || pid == i1 || pid == i2 || (s3 && pid == i3))) continue;
            float d2, cx, cy, cz, ps = 0.f, pt = 0.f;
            if (!s3) {
                oracle_point_triangle_closest_point_f(qx, qy, qz, (float)sx[i0], (float)sy[i0], (float)sz[i0],
                                                      (float)sx[i1], (float)sy[i1], (float)sz[i1], (float)sx[i2],
                                                      (float)sy[i2], (float)sz[i2], &cx, &cy, &cz);
            } else {
                const float ax = (float)sx[i0], ay = (float)sy[i0], az = (float)sz[i0];
                const float bx_ = (float)sx[i1], by_ = (float)sy[i1], bz_ = (float)sz[i1];
                const float cx_ = (float)sx[i2], cy_ = (float)sy[i2], cz_ = (float)sz[i2];
                const float dx_ = (float)sx[i3], dy_ = (float)sy[i3], dz_ = (float)sz[i3];
                oracle_point_to_quad_closest_point_f(qx, qy, qz, ax, ay, az, bx_, by_, bz_, cx_, cy_, cz_, dx_, dy_,
                                                     dz_, &ps, &pt);
                const float ms = 1.0f - ps, mt = 1.0f - pt;
                const float w0 = ms * mt, w1 = ps * mt, w2 = ps * pt, w3 = ms * pt;
                cx = ax * w0 + bx_ * w1 + cx_ * w2 + dx_ * w3;
                cy = ay * w0 + by_ * w1 + cy_ * w2 + dy_ * w3;
                cz = az * w0 + bz_ * w1 + cz_ * w2 + dz_ * w3;
            }
            const float dx = qx - cx, dy = qy - cy, dz = qz - cz;
            d2 = dx * dx + dy * dy + dz * dz;
            if (d2 == INFINITY) continue;
            if (d2 < best || (d2 == best && bt < 0)) {
                best = d2, bt = (int)e;
                bx = cx, by = cy, bz = cz, bs = ps, bt_ = pt;
            }
        }
        outtri[pid] = bt;
        outd[pid] = (TREAL)best;
        if (!local) {
            o0[pid] = (TREAL)bx, o1[pid] = (TREAL)by, o2[pid] = (TREAL)bz;
        } else if (s3) {
            o0[pid] = (TREAL)bs, o1[pid] = (TREAL)bt_;
        } else if (bt >= 0) {
            const int i0 = s0[bt], i1 = s1[bt], i2 = s2[bt];
            TREAL s, t;
            OQ_LOCAL_ST((TREAL)bx, (TREAL)by, (TREAL)bz, (TREAL)sx[i0], (TREAL)sy[i0], (TREAL)sz[i0], (TREAL)sx[i1],
                (TREAL)sy[i1], (TREAL)sz[i1], (TREAL)sx[i2], (TREAL)sy[i2], (TREAL)sz[i2], &s, &t);
            o0[pid] = s, o1[pid] = t;
        } else {
            o0[pid] = (TREAL)0, o1[pid] = (TREAL)0;
        }
    }
    return 0;
}

#undef OQ_CAT2
#undef OQ_CAT
#undef OQ_NAME
