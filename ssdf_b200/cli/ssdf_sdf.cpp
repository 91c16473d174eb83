// ssdf_sdf -- command-line distance field over raw files, the B200 counterpart of ssdf's
// drivers/sdf.exe.cpp: same arguments, file layout and environment switches, so a pipeline that
// calls that driver can call this binary instead.
//
//   ssdf_sdf <surface_folder> [surface_folder ...] <points_folder> <output_file>
//
// Each surface folder holds x.float32, y.float32, z.float32 (vertex coordinates) and i0.int32,
// i1.int32, i2.int32 (0-based triangle corners); the points folder x/y/z.float32; the output is
// float32[npoints], the unsigned distance to the union of the surfaces (drivers/sdf.exe.cpp:128-155).
// Environment (drivers/sdf.exe.cpp:286-334, 385-387):
//   SSDF_INPUT_SDF=<file>         start from these float32 distances instead of FLT_MAX;
//   SSDF_INIT_WITH_VOLUME_BOX=1   start from |signed distance| to the points' own bounding box;
//   SSDF_DOUBLE_PRECISION=1       compute in double (FP32 traversal with the FP64 fix-up), round
//                                 the result to float at the end;
//   SSDF_USE_BVH=0 (and SSDF_USE_CELL_LIST / SSDF_CELL_VALIDATE) select ssdf's edf_select dispatch
//                                 through the drop-in ssdf_edf_f / ssdf_edf_d instead.
// Unlike the reference driver, the points and the running distances stay on the device across the
// surfaces: one upload, then per surface a BVH build and an in/out query, one download at the end.
#include <cuda_runtime.h>

#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "ssdf_b200.h"

namespace {

int usage(const char *prog) {
    fprintf(stderr,
            "Usage: %s <surf_folder1> [surf_folder2] ... <points_folder> <output_file>\n\n"
            "Surface folder(s): x.float32 y.float32 z.float32 (coordinates), i0.int32 i1.int32 i2.int32\n"
            "Points folder: x.float32 y.float32 z.float32\n"
            "Output: float32 distance[npoints]\n"
            "Environment: SSDF_INPUT_SDF, SSDF_INIT_WITH_VOLUME_BOX, SSDF_DOUBLE_PRECISION, SSDF_USE_BVH\n",
            prog);
    return 1;
}

std::string join(const char *folder, const char *name) {
    std::string p = folder;
    if (p.empty() || p.back() != '/') p += '/';
    return p + name;
}

// Element count of a raw file of `elem`-byte values, or -1 (missing, unreadable, ragged size).
long long raw_count(const std::string &path, size_t elem) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return -1;
    long long n = -1;
    if (fseek(f, 0, SEEK_END) == 0) {
        const long size = ftell(f);
        if (size >= 0 && size % long(elem) == 0) n = size / long(elem);
    }
    fclose(f);
    return n;
}

template <typename V>
bool read_raw(const std::string &path, std::vector<V> &v) {
    const long long n = raw_count(path, sizeof(V));
    if (n < 0) {
        fprintf(stderr, "Error: Cannot open or invalid file '%s'\n", path.c_str());
        return false;
    }
    v.resize(size_t(n));
    FILE *f = fopen(path.c_str(), "rb");
    const bool ok = f && fread(v.data(), sizeof(V), size_t(n), f) == size_t(n);
    if (f) fclose(f);
    if (!ok) fprintf(stderr, "Error: Failed to read file '%s'\n", path.c_str());
    return ok;
}

int env_flag(const char *name) {
    const char *v = getenv(name);
    return v ? atoi(v) : 0;
}

struct Surface {
    std::string folder;
    long long nv = 0, nt = 0;
};

bool check_surface(const char *folder, Surface *s) {
    const long long nx = raw_count(join(folder, "x.float32"), 4), ni = raw_count(join(folder, "i0.int32"), 4);
    if (nx < 0) {
        fprintf(stderr, "Error: Cannot open or invalid file '%s'\n", join(folder, "x.float32").c_str());
        return false;
    }
    if (raw_count(join(folder, "y.float32"), 4) != nx || raw_count(join(folder, "z.float32"), 4) != nx) {
        fprintf(stderr, "Error: Surface coordinate files have mismatched sizes in '%s'\n", folder);
        return false;
    }
    if (ni < 0) {
        fprintf(stderr, "Error: Cannot open or invalid file '%s'\n", join(folder, "i0.int32").c_str());
        return false;
    }
    if (raw_count(join(folder, "i1.int32"), 4) != ni || raw_count(join(folder, "i2.int32"), 4) != ni) {
        fprintf(stderr, "Error: Surface index files have mismatched sizes in '%s'\n", folder);
        return false;
    }
    s->folder = folder;
    s->nv = nx;
    s->nt = ni;
    return true;
}

#define CLI_CHECK(call)                                                                          \
    do {                                                                                         \
        const int st_ = (call);                                                                  \
        if (st_ != SSDF_OK) {                                                                    \
            fprintf(stderr, "Error: %s failed: %s (%s)\n", #call, ssdf_status_string(st_), ssdf_last_error()); \
            return 1;                                                                            \
        }                                                                                        \
    } while (0)
#define CLI_CUDA(call)                                                                           \
    do {                                                                                         \
        const cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                                 \
            fprintf(stderr, "Error: %s failed: %s\n", #call, cudaGetErrorString(e_));           \
            return 1;                                                                            \
        }                                                                                        \
    } while (0)

// Surface distances through ssdf's edf_select dispatch on host arrays (SSDF_USE_BVH=0).
int run_host(const std::vector<Surface> &surfs, const std::vector<float> (&p)[3], std::vector<float> &out,
             bool f64) {
    const ptrdiff_t n = ptrdiff_t(out.size());
    std::vector<double> pd[3], od;
    if (f64) {
        for (int a = 0; a < 3; a++) pd[a].assign(p[a].begin(), p[a].end());
        od.assign(out.begin(), out.end());
    }
    for (const Surface &s : surfs) {
        std::vector<float> v[3];
        std::vector<int> t[3];
        const char *vn[3] = {"x.float32", "y.float32", "z.float32"}, *tn[3] = {"i0.int32", "i1.int32", "i2.int32"};
        for (int a = 0; a < 3; a++)
            if (!read_raw(join(s.folder.c_str(), vn[a]), v[a]) || !read_raw(join(s.folder.c_str(), tn[a]), t[a])) return 1;
        if (f64) {
            std::vector<double> vd[3];
            for (int a = 0; a < 3; a++) vd[a].assign(v[a].begin(), v[a].end());
            CLI_CHECK(ssdf_edf_d(n, pd[0].data(), pd[1].data(), pd[2].data(), ptrdiff_t(s.nt), t[0].data(), t[1].data(),
                                 t[2].data(), ptrdiff_t(s.nv), vd[0].data(), vd[1].data(), vd[2].data(), od.data()));
        } else {
            CLI_CHECK(ssdf_edf_f(n, p[0].data(), p[1].data(), p[2].data(), ptrdiff_t(s.nt), t[0].data(), t[1].data(),
                                 t[2].data(), ptrdiff_t(s.nv), v[0].data(), v[1].data(), v[2].data(), out.data()));
        }
    }
    if (f64)
        for (ptrdiff_t i = 0; i < n; i++) out[size_t(i)] = float(od[size_t(i)]);
    return 0;
}

// The device-resident path: points and distances uploaded once, one BVH per surface.
int run_device(const std::vector<Surface> &surfs, const std::vector<float> (&p)[3], std::vector<float> &out,
               bool f64) {
    const size_t n = out.size();
    cudaStream_t stream;
    CLI_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    const size_t eb = f64 ? sizeof(double) : sizeof(float);
    void *dp[3] = {nullptr, nullptr, nullptr}, *dout = nullptr;
    for (int a = 0; a < 3; a++) CLI_CUDA(cudaMalloc(&dp[a], eb * (n ? n : 1)));
    CLI_CUDA(cudaMalloc(&dout, eb * (n ? n : 1)));
    if (f64) {
        std::vector<double> tmp(n);
        for (int a = 0; a < 3; a++) {
            for (size_t i = 0; i < n; i++) tmp[i] = double(p[a][i]);
            CLI_CUDA(cudaMemcpy(dp[a], tmp.data(), eb * n, cudaMemcpyHostToDevice));
        }
    } else {
        for (int a = 0; a < 3; a++) CLI_CUDA(cudaMemcpy(dp[a], p[a].data(), eb * n, cudaMemcpyHostToDevice));
    }
    const int ct = f64 ? SSDF_F64 : SSDF_F32;
    if (f64) {
        std::vector<double> tmp(out.begin(), out.end());
        CLI_CUDA(cudaMemcpy(dout, tmp.data(), eb * n, cudaMemcpyHostToDevice));
    } else {
        CLI_CUDA(cudaMemcpy(dout, out.data(), eb * n, cudaMemcpyHostToDevice));
    }
    ssdf_query_opts qo;
    memset(&qo, 0, sizeof(qo));
    qo.precision = f64 ? SSDF_PREC_F32_FIXUP : SSDF_PREC_F32;
    qo.output = SSDF_OUT_EDF;
    qo.coord_type = ct;
    qo.out_type = ct;
    ssdf_build_opts bo;
    bo.leaf_size = 0;
    bo.keep_fp64 = f64 ? 1 : 0;
    bo.normals = 0;
    bo.treelet_opt = 1;
    for (size_t k = 0; k < surfs.size(); k++) {
        const Surface &s = surfs[k];
        std::vector<float> v[3];
        std::vector<int> t[3];
        const char *vn[3] = {"x.float32", "y.float32", "z.float32"}, *tn[3] = {"i0.int32", "i1.int32", "i2.int32"};
        for (int a = 0; a < 3; a++)
            if (!read_raw(join(s.folder.c_str(), vn[a]), v[a]) || !read_raw(join(s.folder.c_str(), tn[a]), t[a])) return 1;
        printf("  Processing surface %zu/%zu: %s (%lld points, %lld elements)\n", k + 1, surfs.size(), s.folder.c_str(),
               s.nv, s.nt);
        if (s.nt == 0 || s.nv == 0 || n == 0) continue;  // an empty surface leaves the distances as they are
        const auto t0 = std::chrono::steady_clock::now();
        ssdf_mesh *m = nullptr;
        if (f64) {
            std::vector<double> vd[3];
            for (int a = 0; a < 3; a++) vd[a].assign(v[a].begin(), v[a].end());
            CLI_CHECK(ssdf_mesh_create(&m, ptrdiff_t(s.nt), t[0].data(), t[1].data(), t[2].data(), ptrdiff_t(s.nv),
                                       vd[0].data(), vd[1].data(), vd[2].data(), SSDF_F64, 0, &bo, stream));
        } else {
            CLI_CHECK(ssdf_mesh_create(&m, ptrdiff_t(s.nt), t[0].data(), t[1].data(), t[2].data(), ptrdiff_t(s.nv),
                                       v[0].data(), v[1].data(), v[2].data(), SSDF_F32, 0, &bo, stream));
        }
        const int st = ssdf_query_points(m, ptrdiff_t(n), dp[0], dp[1], dp[2], dout, nullptr, nullptr, nullptr, nullptr,
                                         &qo, stream);
        const cudaError_t e = cudaStreamSynchronize(stream);
        ssdf_mesh_destroy(m);
        CLI_CHECK(st);
        CLI_CUDA(e);
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        printf("Time taken: %f ms\n", ms);
    }
    if (f64) {
        std::vector<double> tmp(n);
        CLI_CUDA(cudaMemcpy(tmp.data(), dout, eb * n, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < n; i++) out[i] = float(tmp[i]);
    } else {
        CLI_CUDA(cudaMemcpy(out.data(), dout, eb * n, cudaMemcpyDeviceToHost));
    }
    for (void *d : dp) cudaFree(d);
    cudaFree(dout);
    cudaStreamDestroy(stream);
    return 0;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 4) return usage(argv[0]);
    const char *points_folder = argv[argc - 2], *output_file = argv[argc - 1];
    printf("Checking files and determining sizes...\n");
    std::vector<Surface> surfs;
    for (int i = 1; i < argc - 2; i++) {
        Surface s;
        if (!check_surface(argv[i], &s)) return 1;
        printf("  Surface %d (%s): %lld points, %lld elements\n", i, argv[i], s.nv, s.nt);
        surfs.push_back(s);
    }
    std::vector<float> p[3];
    const char *pn[3] = {"x.float32", "y.float32", "z.float32"};
    for (int a = 0; a < 3; a++)
        if (!read_raw(join(points_folder, pn[a]), p[a])) return 1;
    if (p[1].size() != p[0].size() || p[2].size() != p[0].size()) {
        fprintf(stderr, "Error: Point coordinate files have mismatched sizes\n");
        return 1;
    }
    const size_t n = p[0].size();
    printf("  Points: %zu points\n", n);
    std::vector<float> out(n, FLT_MAX);
    bool volume_box = false;
    if (const char *in = getenv("SSDF_INPUT_SDF")) {
        printf("Reading input SDF from '%s'...\n", in);
        std::vector<float> init;
        if (!read_raw(in, init)) return 1;
        if (init.size() != n) {
            fprintf(stderr, "Error: Input SDF file has %zu points, expected %zu\n", init.size(), n);
            return 1;
        }
        out = init;
    } else {
        volume_box = env_flag("SSDF_INIT_WITH_VOLUME_BOX") != 0;
    }
    const bool f64 = env_flag("SSDF_DOUBLE_PRECISION") == 1;
    const char *bvh = getenv("SSDF_USE_BVH");
    const bool use_bvh = !bvh || atoi(bvh) != 0;
    printf("Processing surfaces...\n");
    if (volume_box && n > 0) {
        // the points' own box, then |signed distance| to it, in float as the reference driver does
        // before any precision switch (drivers/sdf.exe.cpp:316-326)
        float b[6];
        if (ssdf_b200_compute_aabb_ff(ptrdiff_t(n), p[0].data(), p[1].data(), p[2].data(), &b[0], &b[1], &b[2], &b[3],
                                      &b[4], &b[5]) != SSDF_OK ||
            ssdf_b200_all_points_aabb_signed_distance_ff(ptrdiff_t(n), p[0].data(), p[1].data(), p[2].data(), b[0], b[1],
                                                         b[2], b[3], b[4], b[5], out.data()) != SSDF_OK) {
            fprintf(stderr, "Error: box initialisation failed: %s\n", ssdf_last_error());
            return 1;
        }
        for (float &v : out) v = std::fabs(v);
    }
    const int rc = use_bvh ? run_device(surfs, p, out, f64) : run_host(surfs, p, out, f64);
    if (rc != 0) return rc;
    printf("Writing output to '%s'...\n", output_file);
    FILE *f = fopen(output_file, "wb");
    if (!f) {
        fprintf(stderr, "Error: Cannot open output file '%s'\n", output_file);
        return 1;
    }
    const bool ok = fwrite(out.data(), sizeof(float), n, f) == n;
    fclose(f);
    if (!ok) {
        fprintf(stderr, "Error: Failed to write SDF results\n");
        return 1;
    }
    printf("Successfully computed SDF for %zu points across %zu surfaces, written to '%s'\n", n, surfs.size(),
           output_file);
    return 0;
}
