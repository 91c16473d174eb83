// gen_golden.cpp -- writes tests/golden/reference_tests.json: the inputs of zulianp/ssdf's own
// CPU tests for the distance path, regenerated exactly as those tests do, with the reference's
// outputs on them. Built and run by tests/golden/make_golden.py against the reference sources
// (it includes serial/ssdf.hpp from there); the JSON it writes is committed.
//
//   ssdf_test            tests/ssdf_test.cpp:12-61   one triangle, five points, edf_select<float>
//   ssdf_brute_force     tests/ssdf_brute_force_test.cpp:11-97   mt19937(1), U(-1,1), 50 triangles,
//                        20 points, edf<double> and edf_select<double> (= edf_celllist without cuBQL)
//   point_aabb           tests/point_aabb_distance_test.cpp:24-35   seven points, unit box
//   box_sdf              tests/signed_distance_box_test.cpp:23-38   eleven points
//   quad_closest         tests/point_quad_closest_point_test.cpp:8-160   segment, triangle and five
//                        quads (basic, warped, concave, concave notch, degenerate), double
//
// Doubles are printed with 17 significant digits and floats with 9, which round-trip exactly.
#include <cmath>
#include <cstdio>
#include <limits>
#include <random>
#include <vector>

#include "ssdf.hpp"

static void put_d(FILE *f, const char *name, const std::vector<double> &v, bool last = false) {
    std::fprintf(f, "    \"%s\": [", name);
    for (size_t i = 0; i < v.size(); i++) std::fprintf(f, "%s%.17g", i ? ", " : "", v[i]);
    std::fprintf(f, "]%s\n", last ? "" : ",");
}
static void put_f(FILE *f, const char *name, const std::vector<float> &v, bool last = false) {
    std::fprintf(f, "    \"%s\": [", name);
    for (size_t i = 0; i < v.size(); i++) std::fprintf(f, "%s%.9g", i ? ", " : "", (double)v[i]);
    std::fprintf(f, "]%s\n", last ? "" : ",");
}
static void put_i(FILE *f, const char *name, const std::vector<int> &v, bool last = false) {
    std::fprintf(f, "    \"%s\": [", name);
    for (size_t i = 0; i < v.size(); i++) std::fprintf(f, "%s%d", i ? ", " : "", v[i]);
    std::fprintf(f, "]%s\n", last ? "" : ",");
}

int main(int argc, char **argv) {
    FILE *f = argc > 1 ? std::fopen(argv[1], "w") : stdout;
    if (!f) return 1;
    std::fprintf(f, "{\n");

    {  // tests/ssdf_test.cpp
        std::vector<float> sx = {0.0f, 1.0f, 0.5f}, sy = {0.0f, 0.0f, 1.0f}, sz = {0.0f, 0.0f, 0.0f};
        std::vector<int> s0 = {0}, s1 = {1}, s2 = {2};
        std::vector<float> x = {0.5f, 0.0f, 1.0f, 0.5f, 0.25f}, y = {0.5f, 0.0f, 0.0f, 0.5f, 0.25f},
                           z = {0.0f, 0.0f, 0.0f, 1.0f, 0.0f};
        std::vector<float> out(5, 1111111.0f), brute(5);
        ssdf::edf_select<float, float, int>(5, x.data(), y.data(), z.data(), 1, s0.data(), s1.data(), s2.data(), 3,
                                            sx.data(), sy.data(), sz.data(), out.data());
        for (int p = 0; p < 5; p++)
            brute[p] = std::sqrt(ssdf::point_triangle_dist_sq(x[p], y[p], z[p], sx[0], sy[0], sz[0], sx[1], sy[1],
                                                              sz[1], sx[2], sy[2], sz[2]));
        std::fprintf(f, "  \"ssdf_test\": {\n");
        put_f(f, "sx", sx), put_f(f, "sy", sy), put_f(f, "sz", sz);
        put_i(f, "s0", s0), put_i(f, "s1", s1), put_i(f, "s2", s2);
        put_f(f, "x", x), put_f(f, "y", y), put_f(f, "z", z);
        std::fprintf(f, "    \"out_init\": 1111111.0,\n    \"tolerance\": 1e-5,\n");
        put_f(f, "edf_select", out);
        put_f(f, "brute", brute, true);
        std::fprintf(f, "  },\n");
    }

    {  // tests/ssdf_brute_force_test.cpp
        std::mt19937 rng(1);
        std::uniform_real_distribution<double> dist(-1.0, 1.0);
        const int ntri = 50, npt = 20;
        std::vector<double> sx(ntri * 3), sy(ntri * 3), sz(ntri * 3);
        for (int i = 0; i < ntri * 3; ++i) {
            sx[i] = dist(rng);
            sy[i] = dist(rng);
            sz[i] = dist(rng);
        }
        std::vector<int> s0(ntri), s1(ntri), s2(ntri);
        for (int t = 0; t < ntri; ++t) s0[t] = 3 * t, s1[t] = 3 * t + 1, s2[t] = 3 * t + 2;
        std::vector<double> x(npt), y(npt), z(npt);
        for (int i = 0; i < npt; ++i) {
            x[i] = dist(rng);
            y[i] = dist(rng);
            z[i] = dist(rng);
        }
        std::vector<double> out_edf(npt, 1e9), out_select(npt, 1e9), brute(npt);
        ssdf::edf<double, double, int>(npt, x.data(), y.data(), z.data(), ntri, s0.data(), s1.data(), s2.data(),
                                       ntri * 3, sx.data(), sy.data(), sz.data(), out_edf.data());
        ssdf::edf_select<double, double, int>(npt, x.data(), y.data(), z.data(), ntri, s0.data(), s1.data(),
                                              s2.data(), ntri * 3, sx.data(), sy.data(), sz.data(), out_select.data());
        for (int p = 0; p < npt; p++) {
            double best = std::numeric_limits<double>::max();
            for (int t = 0; t < ntri; ++t) {
                const int i0 = s0[t], i1 = s1[t], i2 = s2[t];
                best = std::min(best, ssdf::point_triangle_dist_sq(x[p], y[p], z[p], sx[i0], sy[i0], sz[i0], sx[i1],
                                                                   sy[i1], sz[i1], sx[i2], sy[i2], sz[i2]));
            }
            brute[p] = std::sqrt(best);
        }
        std::fprintf(f, "  \"ssdf_brute_force\": {\n");
        put_d(f, "sx", sx), put_d(f, "sy", sy), put_d(f, "sz", sz);
        put_i(f, "s0", s0), put_i(f, "s1", s1), put_i(f, "s2", s2);
        put_d(f, "x", x), put_d(f, "y", y), put_d(f, "z", z);
        std::fprintf(f, "    \"out_init\": 1e9,\n    \"tolerance\": 1e-7,\n");
        put_d(f, "edf", out_edf);
        put_d(f, "edf_select", out_select);
        put_d(f, "brute", brute, true);
        std::fprintf(f, "  },\n");
    }

    {  // tests/point_aabb_distance_test.cpp: unit box, (point, expected squared distance)
        const double c[7][4] = {{0.5, 0.5, 0.5, 0.0},   {0.0, 0.0, 0.0, 0.0},    {1.0, 0.2, 0.8, 0.0},
                                {-1.0, 0.5, 0.5, 1.0},  {0.5, 2.0, 0.5, 1.0},    {0.5, 0.5, -0.25, 0.0625},
                                {-1.0, -2.0, 3.0, 9.0}};
        std::vector<double> px, py, pz, expected, got;
        for (auto &r : c) {
            px.push_back(r[0]), py.push_back(r[1]), pz.push_back(r[2]), expected.push_back(r[3]);
            got.push_back(ssdf::point_aabb_distance_squared(r[0], r[1], r[2], 0.0, 1.0, 0.0, 1.0, 0.0, 1.0));
        }
        std::fprintf(f, "  \"point_aabb\": {\n    \"box\": [0.0, 1.0, 0.0, 1.0, 0.0, 1.0],\n");
        std::fprintf(f, "    \"tolerance\": 1e-12,\n");
        put_d(f, "x", px), put_d(f, "y", py), put_d(f, "z", pz);
        put_d(f, "expected", expected);
        put_d(f, "reference", got, true);
        std::fprintf(f, "  },\n");
    }

    {  // tests/signed_distance_box_test.cpp: box [-1,1]x[-2,2]x[0.5,1.5]
        const double c[11][4] = {{0.0, 0.0, 1.0, -0.5}, {0.0, 0.0, 1.4, -0.1}, {0.9, 0.0, 1.0, -0.1},
                                 {-0.8, 1.9, 1.0, -0.1}, {1.0, 0.0, 1.0, 0.0}, {0.0, -2.0, 1.0, 0.0},
                                 {0.0, 0.0, 1.5, 0.0},  {2.0, 0.0, 1.0, 1.0}, {0.0, -3.0, 1.0, 1.0},
                                 {0.0, 0.0, 3.0, 1.5},  {3.0, 4.0, -1.0, std::sqrt(2.0 * 2.0 + 2.0 * 2.0 + 1.5 * 1.5)}};
        std::vector<double> px, py, pz, expected, got;
        for (auto &r : c) {
            px.push_back(r[0]), py.push_back(r[1]), pz.push_back(r[2]), expected.push_back(r[3]);
            got.push_back(ssdf::point_aabb_signed_distance(r[0], r[1], r[2], -1.0, 1.0, -2.0, 2.0, 0.5, 1.5));
        }
        std::fprintf(f, "  \"box_sdf\": {\n    \"box\": [-1.0, 1.0, -2.0, 2.0, 0.5, 1.5],\n");
        std::fprintf(f, "    \"tolerance\": 1e-12,\n");
        put_d(f, "x", px), put_d(f, "y", py), put_d(f, "z", pz);
        put_d(f, "expected", expected);
        put_d(f, "reference", got, true);
        std::fprintf(f, "  },\n");
    }

    {  // tests/point_quad_closest_point_test.cpp: rows (point, 4 corners, expected s, t)
        const double c[5][17] = {
            {0.25, 0.75, 1, 0, 0, 0, 1, 0, 0, 1, 1, 0, 0, 1, 0, 0.25, 0.75},
            {0.7, 0.2, 0.225, 0, 0, 0, 1, 0, 0.25, 1, 1, 0.5, 0, 1, -0.25, 0.7, 0.2},
            {0.3, 1.0, 0, 0, 0, 0, 2, 0, 0, 0.75, 0.5, 0, 0, 2, 0, 0.4, 0.8},
            {11.0 / 12.0, 5.0 / 6.0, 0, 0, 0, 0, 2, 0, 0, 0.75, 0.5, 0, 0, 2, 0, 13.0 / 15.0, 1},
            {1.5, 1, 0, 0, 0, 0, 1, 0, 0, 2, 0, 0, 3, 0, 0, 1, 0.5}};
        std::vector<double> rows, expected, got;
        for (auto &r : c) {
            double s = -1, t = -1;
            ssdf::point_to_quad_closest_point<double>(r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7], r[8], r[9], r[10],
                                                      r[11], r[12], r[13], r[14], &s, &t);
            for (int k = 0; k < 15; k++) rows.push_back(r[k]);
            expected.push_back(r[15]), expected.push_back(r[16]);
            got.push_back(s), got.push_back(t);
        }
        double u = -1, wa = -1, wb = -1, wc = -1;
        const double dseg = ssdf::point_segment_parameter(0.25, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, &u);
        const double dtri = ssdf::point_triangle_barycentric(0.25, 0.25, 1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0,
                                                             0.0, &wa, &wb, &wc);
        std::fprintf(f, "  \"quad_closest\": {\n    \"tolerance\": 1e-12,\n");
        std::fprintf(f, "    \"names\": [\"basic\", \"warped\", \"concave\", \"concave notch\", \"degenerate\"],\n");
        put_d(f, "rows", rows);
        put_d(f, "expected", expected);
        put_d(f, "reference", got);
        put_d(f, "triangle", {0.25, 0.25, 1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0, 0.0});
        put_d(f, "triangle_expected", {1.0, 0.5, 0.25, 0.25});
        put_d(f, "triangle_reference", {dtri, wa, wb, wc});
        put_d(f, "segment_reference", {dseg, u}, true);
        std::fprintf(f, "  }\n");
    }

    std::fprintf(f, "}\n");
    if (f != stdout) std::fclose(f);
    return 0;
}
