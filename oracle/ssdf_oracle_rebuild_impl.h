/*
 * ssdf_oracle_rebuild_impl.h -- the per-precision body of the level-set oracle, included twice by
 * ssdf_oracle_rebuild.c (REAL = double, SUF = _d; REAL = float, SUF = _f).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library's sdf_rebuild path, never part of it.
 *
 * Restates serial/bvh/sdf_rebuild.cpp (G = T = REAL): marching tetrahedra in the reference's cell,
 * tetrahedron and triangle order (cells x fastest, then y, then z), the cubic refinement, and the
 * banded rebuild. The rebuild's distance follows the CUDA library's definition: the exact double
 * distance from the sample o + i h (evaluated in double) to the triangles, by brute force with the
 * reference's double point-triangle expression, bounded by the band; the reference itself searches
 * with cuBQL in float from the float-rounded sample, which cannot be built here.
 */

#ifndef REAL
#error "define REAL and SUF before including ssdf_oracle_rebuild_impl.h"
#endif

#define RB_CAT2(a, b) a##b
#define RB_CAT(a, b) RB_CAT2(a, b)
#define RB_NAME(n) RB_CAT(n, SUF)

/* Triangles of {f = level} (sdf_rebuild.cpp:190-250); x, y, z may be NULL (count only). */
ptrdiff_t RB_NAME(oracle_level_set_triangles)(const ptrdiff_t n[3], const REAL o[3], const REAL h[3], const REAL *f,
                                              const REAL level, REAL *x, REAL *y, REAL *z) {
    if (n[0] < 2 || n[1] < 2 || n[2] < 2) return 0;
    const ptrdiff_t sy = n[0], sz = n[0] * n[1];
    ptrdiff_t count = 0;
    for (ptrdiff_t k = 0; k + 1 < n[2]; k++)
        for (ptrdiff_t j = 0; j + 1 < n[1]; j++)
            for (ptrdiff_t i = 0; i + 1 < n[0]; i++) {
                ptrdiff_t g[8];
                double v[8], p[8][3];
                int above = 0;
                for (int c = 0; c < 8; c++) {
                    const ptrdiff_t idx[3] = {i + (c & 1), j + ((c >> 1) & 1), k + ((c >> 2) & 1)};
                    g[c] = idx[0] + idx[1] * sy + idx[2] * sz;
                    v[c] = (double)f[g[c]] - (double)level;
                    above += v[c] > 0;
                    for (int d = 0; d < 3; d++) p[c][d] = (double)o[d] + (double)idx[d] * (double)h[d];
                }
                if (above == 0 || above == 8) continue;
                for (int t = 0; t < 6; t++) {
                    double tri[2][3][3];
                    const int m = oracle_tet_triangles(g, v, p, kOracleTets[t], tri);
                    for (int s = 0; s < m; s++) {
                        int degenerate = 0;
                        for (int a = 0; a < 3; a++) {
                            const int b = (a + 1) % 3;
                            degenerate |= (REAL)tri[s][a][0] == (REAL)tri[s][b][0] &&
                                          (REAL)tri[s][a][1] == (REAL)tri[s][b][1] &&
                                          (REAL)tri[s][a][2] == (REAL)tri[s][b][2];
                        }
                        if (degenerate) continue;
                        if (x)
                            for (int a = 0; a < 3; a++) {
                                x[3 * count + a] = (REAL)tri[s][a][0];
                                y[3 * count + a] = (REAL)tri[s][a][1];
                                z[3 * count + a] = (REAL)tri[s][a][2];
                            }
                        count++;
                    }
                }
            }
    return count;
}

/* The cubic refinement (sdf_rebuild.cpp:132-188): weights in double, each pass along one axis. */
void RB_NAME(oracle_refine_field)(const ptrdiff_t n[3], const REAL *f, const ptrdiff_t factor, REAL *fine) {
    ptrdiff_t rn[3];
    for (int d = 0; d < 3; d++) rn[d] = (n[d] - 1) * factor + 1;
    const ptrdiff_t fx = rn[0], fxy = rn[0] * rn[1];
    for (ptrdiff_t k = 0; k < n[2]; k++)
        for (ptrdiff_t j = 0; j < n[1]; j++)
            for (ptrdiff_t i = 0; i < n[0]; i++)
                fine[i * factor + fx * (j * factor) + fxy * (k * factor)] = f[i + n[0] * (j + n[1] * k)];
    if (factor == 1) return;
    double *w = (double *)malloc(sizeof(double) * 4 * (size_t)factor);
    for (ptrdiff_t m = 0; m < factor; m++) {
        const double t = (double)m / (double)factor;
        w[4 * m + 0] = -t * (t - 1) * (t - 2) / 6;
        w[4 * m + 1] = (t + 1) * (t - 1) * (t - 2) / 2;
        w[4 * m + 2] = -(t + 1) * t * (t - 2) / 2;
        w[4 * m + 3] = (t + 1) * t * (t - 1) / 6;
    }
    for (int axis = 0; axis < 3; axis++) {
        const ptrdiff_t stride = axis == 0 ? 1 : (axis == 1 ? fx : fxy), na = n[axis];
        const int a1 = (axis + 1) % 3, a2 = (axis + 2) % 3;
        const ptrdiff_t s1 = a1 == 0 ? 1 : (a1 == 1 ? fx : fxy), s2 = a2 == 0 ? 1 : (a2 == 1 ? fx : fxy);
        const ptrdiff_t c1 = a1 < axis ? 1 : factor, c2 = a2 < axis ? 1 : factor;
        const ptrdiff_t n1 = a1 < axis ? rn[a1] : n[a1], n2 = a2 < axis ? rn[a2] : n[a2];
        for (ptrdiff_t q2 = 0; q2 < n2; q2++)
            for (ptrdiff_t q1 = 0; q1 < n1; q1++) {
                REAL *line = fine + q1 * c1 * s1 + q2 * c2 * s2;
                for (ptrdiff_t c = 0; c + 1 < na; c++) {
                    const REAL v0 = line[(c > 0 ? c - 1 : 0) * factor * stride], v1 = line[c * factor * stride];
                    const REAL v2 = line[(c + 1) * factor * stride];
                    const REAL v3 = line[(c + 2 < na - 1 ? c + 2 : na - 1) * factor * stride];
                    for (ptrdiff_t m = 1; m < factor; m++) {
                        const double *wm = w + 4 * m;
                        line[(c * factor + m) * stride] = (REAL)(wm[0] * v0 + wm[1] * v1 + wm[2] * v2 + wm[3] * v3);
                    }
                }
            }
    }
    free(w);
}

/* The banded rebuild on every stride-th sample (sdf_rebuild.cpp:252-299), distances as above. */
void RB_NAME(oracle_rebuild_sdf)(const ptrdiff_t n[3], const REAL o[3], const REAL h[3], const REAL *f,
                                 const REAL level, const REAL band, const ptrdiff_t stride, REAL *out) {
    const ptrdiff_t nt = RB_NAME(oracle_level_set_triangles)(n, o, h, f, level, NULL, NULL, NULL);
    REAL *sx = NULL, *sy = NULL, *sz = NULL;
    if (nt > 0) {
        sx = (REAL *)malloc(sizeof(REAL) * 3 * (size_t)nt);
        sy = (REAL *)malloc(sizeof(REAL) * 3 * (size_t)nt);
        sz = (REAL *)malloc(sizeof(REAL) * 3 * (size_t)nt);
        RB_NAME(oracle_level_set_triangles)(n, o, h, f, level, sx, sy, sz);
    }
    ptrdiff_t on[3];
    REAL oh[3];
    for (int d = 0; d < 3; d++) {
        on[d] = (n[d] - 1) / stride + 1;
        oh[d] = h[d] * (REAL)stride;
    }
    const ptrdiff_t total = on[0] * on[1] * on[2];
#pragma omp parallel for schedule(dynamic, 16)
    for (ptrdiff_t q = 0; q < total; q++) {
        const ptrdiff_t i = q % on[0], j = (q / on[0]) % on[1], k = q / (on[0] * on[1]);
        const REAL v = f[stride * (i + j * n[0] + k * n[0] * n[1])] - level;
        REAL d = band;
        if (nt > 0 && (v < 0 ? -v : v) < band) {
            const double px = (double)o[0] + (double)i * (double)oh[0];
            const double py = (double)o[1] + (double)j * (double)oh[1];
            const double pz = (double)o[2] + (double)k * (double)oh[2];
            double best = (double)band * (double)band;
            for (ptrdiff_t t = 0; t < nt; t++) {
                const double d2 = oracle_point_triangle_dist_sq_d(
                    px, py, pz, (double)sx[3 * t], (double)sy[3 * t], (double)sz[3 * t], (double)sx[3 * t + 1],
                    (double)sy[3 * t + 1], (double)sz[3 * t + 1], (double)sx[3 * t + 2], (double)sy[3 * t + 2],
                    (double)sz[3 * t + 2]);
                if (d2 < best) best = d2;
            }
            d = (REAL)sqrt(best);
        }
        out[q] = v > 0 ? d : (v < 0 ? -d : (REAL)0);
    }
    free(sx);
    free(sy);
    free(sz);
}

#undef RB_NAME
#undef RB_CAT
#undef RB_CAT2
