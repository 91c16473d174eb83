// autotune.cu -- picks the BVH leaf size, traversal mode and BVH arity for a mesh and a query grid.
//
// No reference counterpart. The candidates are leaf sizes {2, 4, 8} x {warp packets, thread per
// query} x {binary, 4-wide}. Each is timed (CUDA events, best of two after a warm-up) on a sample of
// the grid: the same box at a resolution scaled down to at most 2^21 nodes, so the distances -- and
// the traversal cost per query -- stay those of the full grid. The winner is cached per size class
// (log2 of the triangle count, log2 of the node count, arithmetic) in a small JSON file, one entry
// per line, which later calls (and the batch path) read instead of re-timing.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>

#include "internal.h"

using namespace ssdf_b200;

namespace {

std::mutex g_cache_mutex;

std::string size_class(ptrdiff_t nt, long long nq, int precision) {
    char buf[96];
    snprintf(buf, sizeof(buf), "prec%d_tri2^%d_nodes2^%d", precision, int(std::lround(std::log2(double(nt)))),
             int(std::lround(std::log2(double(nq)))));
    return buf;
}

// File format: {\n "key": [leaf, traversal, arity, ms],\n ... }
std::map<std::string, ssdf_tuning> read_cache(const char *path) {
    std::map<std::string, ssdf_tuning> m;
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
        const size_t q0 = line.find('"'), q1 = line.find('"', q0 + 1), b = line.find('[');
        if (q0 == std::string::npos || q1 == std::string::npos || b == std::string::npos) continue;
        ssdf_tuning t;
        if (sscanf(line.c_str() + b, "[%d, %d, %d, %lf]", &t.leaf_size, &t.traversal, &t.arity, &t.ms) == 4)
            m[line.substr(q0 + 1, q1 - q0 - 1)] = t;
    }
    return m;
}

int write_cache(const char *path, const std::map<std::string, ssdf_tuning> &m) {
    const std::string tmp = std::string(path) + ".tmp";
    FILE *f = fopen(tmp.c_str(), "w");
    if (!f) return fail(SSDF_ERR_INVALID_ARGUMENT, std::string("cannot write the tuning cache ") + path);
    fprintf(f, "{\n");
    size_t k = 0;
    for (const auto &kv : m) {
        fprintf(f, "  \"%s\": [%d, %d, %d, %.6f]%s\n", kv.first.c_str(), kv.second.leaf_size, kv.second.traversal,
                kv.second.arity, kv.second.ms, ++k < m.size() ? "," : "");
    }
    fprintf(f, "}\n");
    fclose(f);
    if (rename(tmp.c_str(), path) != 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "cannot replace the tuning cache");
    return SSDF_OK;
}

}  // namespace

extern "C" {

int ssdf_autotune_grid(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints,
                       const double *sx, const double *sy, const double *sz, ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz,
                       const double lo[3], const double hi[3], int precision, const char *cache_path,
                       ssdf_tuning *best) {
    if (!best || !lo || !hi || nx <= 0 || ny <= 0 || nz <= 0 || nselements <= 0)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "ssdf_autotune_grid: bad arguments");
    if (precision < SSDF_PREC_F32 || precision > SSDF_PREC_F32_FIXUP)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "ssdf_autotune_grid: bad precision");
    const long long nq = (long long)nx * ny * nz;
    const std::string key = size_class(nselements, nq, precision);
    if (cache_path) {
        std::lock_guard<std::mutex> lock(g_cache_mutex);
        auto m = read_cache(cache_path);
        auto it = m.find(key);
        if (it != m.end()) {
            *best = it->second;
            return SSDF_OK;
        }
    }
    // sample grid: same box, at most 2^21 nodes
    const double f = std::min(1.0, std::cbrt(double(1 << 21) / double(nq)));
    const long long sn[3] = {std::max(2ll, (long long)std::llround(nx * f)), std::max(2ll, (long long)std::llround(ny * f)),
                             std::max(2ll, (long long)std::llround(nz * f))};
    const long long ns = sn[0] * sn[1] * sn[2];
    cudaStream_t stream;
    SSDF_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    void *out = nullptr;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int st = SSDF_OK;
    if (cudaMalloc(&out, sizeof(double) * size_t(ns)) != cudaSuccess) st = fail(SSDF_ERR_OUT_OF_MEMORY, "autotune output");
    ssdf_tuning win;
    win.ms = 1e30;
    win.leaf_size = 4, win.traversal = 1, win.arity = 2;
    const int leaves[3] = {2, 4, 8};
    for (int li = 0; li < 3 && st == SSDF_OK; li++) {
        ssdf_build_opts bo;
        bo.leaf_size = leaves[li];
        bo.keep_fp64 = 1;
        bo.normals = 1;
        bo.treelet_opt = kResidentTreeletRounds;
        ssdf_mesh *m = nullptr;
        st = ssdf_mesh_create(&m, nselements, s0, s1, s2, nspoints, sx, sy, sz, SSDF_F64, 0, &bo, stream);
        if (st != SSDF_OK) break;
        ssdf_query_opts qo;
        memset(&qo, 0, sizeof(qo));
        qo.precision = precision;
        qo.output = precision == SSDF_PREC_F32 ? SSDF_OUT_SQEDF : SSDF_OUT_SDF;
        qo.coord_type = SSDF_F64;
        qo.out_type = SSDF_F64;
        for (int trav = 1; trav <= 2 && st == SSDF_OK; trav++) {
            for (int ar = 2; ar <= 4 && st == SSDF_OK; ar += 2) {
                QueryArgs a;
                st = fill_grid_args(m, sn[0], sn[1], sn[2], lo, hi, out, nullptr, &qo, &a);
                if (st != SSDF_OK) break;
                a.force_traversal = trav;
                a.force_arity = ar;
                float bestms = 1e30f;
                for (int rep = 0; rep < 3 && st == SSDF_OK; rep++) {
                    if (precision == SSDF_PREC_F32) cudaMemsetAsync(out, 0x7f, sizeof(double) * size_t(ns), stream);
                    cudaEventRecord(e0, stream);
                    st = launch_query(a, precision, stream);
                    cudaEventRecord(e1, stream);
                    if (cudaEventSynchronize(e1) != cudaSuccess) st = fail(SSDF_ERR_CUDA, "autotune timing");
                    float ms = 0.f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    if (rep > 0) bestms = std::min(bestms, ms);
                }
                if (st == SSDF_OK && bestms < win.ms) {
                    win.ms = bestms;
                    win.leaf_size = leaves[li];
                    win.traversal = trav;
                    win.arity = ar;
                }
            }
        }
        ssdf_mesh_destroy(m);
    }
    cudaFree(out);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(stream);
    if (st != SSDF_OK) return st;
    *best = win;
    if (cache_path) {
        std::lock_guard<std::mutex> lock(g_cache_mutex);
        auto m = read_cache(cache_path);
        m[key] = win;
        SSDF_CHECK(write_cache(cache_path, m));
    }
    return SSDF_OK;
}

}  // extern "C"
