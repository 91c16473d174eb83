// capi.cu -- the exported C ABI (include/ssdf_b200.h): drop-in entry points over host arrays,
// the device-resident mesh handle API, status codes and error messages.
//
// Host-array entry points follow the reference's contract (serial/ssdf.hpp:447-460,
// serial/bvh/bvh.hpp:19-227): blocking, caller owns every buffer, scratch freed before return,
// `out` in/out where the reference's is. They stage through device memory on a per-thread
// non-blocking stream. No entry point aborts: failures return a status and set a message.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "internal.h"

namespace ssdf_b200 {

int query_counts(int64_t *tri, int64_t *box, int64_t *fix, int64_t *fallback);

namespace {
thread_local std::string t_error;
thread_local cudaStream_t t_stream = nullptr;
thread_local int t_stream_device = -1;
}  // namespace

void set_error(const std::string &msg) { t_error = msg; }

int fail(int status, const std::string &msg) {
    t_error = msg;
    return status;
}

int cuda_fail(cudaError_t err, const char *what, const char *file, int line) {
    const char *base = strrchr(file, '/');
    t_error = std::string(what) + ": " + cudaGetErrorString(err) + " (" + (base ? base + 1 : file) + ":" +
              std::to_string(line) + ")";
    return err == cudaErrorMemoryAllocation ? SSDF_ERR_OUT_OF_MEMORY : SSDF_ERR_CUDA;
}

int env_int(const char *name, int dflt) {
    const char *v = getenv(name);
    return v ? atoi(v) : dflt;
}

const char *env_str(const char *name) { return getenv(name); }

// The library's scratch (overflow lists, staging buffers, mesh storage) comes from the device's
// default stream-ordered pool. With the pool's default release threshold of 0, memory freed back to it
// is returned to the device at every synchronisation, so the next query maps it again (134 MB of
// overflow list for a 256^3 grid), at a cost that varied from run to run by up to half the query.
// The library keeps freed memory in the pool instead (once per device); it stays reusable by any
// cudaMallocAsync of the process and is released by cudaMemPoolTrimTo or at exit.
void retain_pool_memory() {
    static std::mutex mu;
    static bool done[64] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = ~uint64_t(0);
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    done[dev] = true;
}

cudaStream_t library_stream() {
    retain_pool_memory();
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    if (!t_stream || t_stream_device != dev) {
        cudaStream_t s = nullptr;
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
        t_stream = s;
        t_stream_device = dev;
    }
    return t_stream;
}

namespace {

// Device buffer list freed (stream-ordered) when it goes out of scope.
struct Scratch {
    cudaStream_t stream;
    std::vector<void *> ptrs;
    explicit Scratch(cudaStream_t s) : stream(s) {}
    ~Scratch() {
        for (void *p : ptrs) cudaFreeAsync(p, stream);
        cudaStreamSynchronize(stream);
    }
    int alloc(void **p, size_t bytes) {
        cudaError_t e = cudaMallocAsync(p, bytes ? bytes : 16, stream);
        if (e != cudaSuccess) return fail(SSDF_ERR_OUT_OF_MEMORY, "device allocation of " + std::to_string(bytes) + " bytes");
        ptrs.push_back(*p);
        return SSDF_OK;
    }
    int upload(void **dst, const void *src, size_t bytes) {
        SSDF_CHECK(alloc(dst, bytes));
        SSDF_CUDA(cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, stream));
        return SSDF_OK;
    }
};

int ready_stream(cudaStream_t *s) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
        return fail(SSDF_ERR_CUDA, std::string("no usable CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "none"));
    *s = library_stream();
    if (!*s) return fail(SSDF_ERR_CUDA, "could not create the library stream");
    return SSDF_OK;
}

int check_mesh_host(ptrdiff_t nt, const int *s0, const int *s1, const int *s2, ptrdiff_t nv, const void *sx,
                    const void *sy, const void *sz) {
    if (nt < 0 || nv < 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "negative mesh size");
    if (nt > 0 && (!s0 || !s1 || !s2)) return fail(SSDF_ERR_INVALID_ARGUMENT, "null triangle index array");
    if (nv > 0 && (!sx || !sy || !sz)) return fail(SSDF_ERR_INVALID_ARGUMENT, "null vertex coordinate array");
    for (ptrdiff_t t = 0; t < nt; t++) {
        if (s0[t] < 0 || s0[t] >= nv || s1[t] < 0 || s1[t] >= nv || s2[t] < 0 || s2[t] >= nv)
            return fail(SSDF_ERR_INVALID_ARGUMENT,
                        "triangle " + std::to_string(t) + " has a vertex index outside [0, " + std::to_string(nv) + ")");
    }
    return SSDF_OK;
}

int precision_from_env(int dflt) {
    const char *v = env_str("SSDF_B200_PRECISION");
    if (!v) return dflt;
    if (!strcmp(v, "f64")) return SSDF_PREC_F64;
    if (!strcmp(v, "f32")) return SSDF_PREC_F32;
    if (!strcmp(v, "f32x") || !strcmp(v, "fixup")) return SSDF_PREC_F32_FIXUP;
    return dflt;
}

// SSDF_B200_TAU: a wider fix-up window than the mesh's own minimum (never a narrower one).
float tau_rel_from_env() {
    const char *v = env_str("SSDF_B200_TAU");
    const float t = v ? float(atof(v)) : 0.f;
    return t > 0.f ? t : 1.0f / 65536.0f;
}

ssdf_build_opts build_opts_for(int precision, int output, long long nqueries) {
    ssdf_build_opts o;
    o.leaf_size = env_int("SSDF_B200_LEAF", 0);
    o.keep_fp64 = (precision != SSDF_PREC_F32 || output == SSDF_OUT_SDF || output == SSDF_OUT_CLOSEST) ? 1 : 0;
    o.normals = output == SSDF_OUT_SDF ? 1 : 0;
    o.treelet_opt = call_treelet_rounds(nqueries);
    return o;
}

struct MeshGuard {
    ssdf_mesh *mesh = nullptr;
    ~MeshGuard() {
        if (mesh) ssdf_mesh_destroy(mesh);
    }
};

// The BVH entry points over host arrays: build, upload, query, download.
template <typename G, typename T>
int bvh_points_host(ptrdiff_t npoints, const G *x, const G *y, const G *z, ptrdiff_t nt, const int *s0, const int *s1,
                    const int *s2, ptrdiff_t nv, const G *sx, const G *sy, const G *sz, T *out, int *outtri, G *outx,
                    G *outy, G *outz, int output, int precision) {
    if (npoints < 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "negative npoints");
    SSDF_CHECK(check_mesh_host(nt, s0, s1, s2, nv, sx, sy, sz));
    if (nt == 0 || nv == 0 || npoints == 0) return SSDF_OK;
    if (!x || !y || !z || !out) return fail(SSDF_ERR_INVALID_ARGUMENT, "null point or output array");
    cudaStream_t stream;
    SSDF_CHECK(ready_stream(&stream));
    const int cf = sizeof(G) == 8 ? SSDF_F64 : SSDF_F32;
    MeshGuard mg;
    const ssdf_build_opts bo = build_opts_for(precision, output, npoints);
    SSDF_CHECK(ssdf_mesh_create(&mg.mesh, nt, s0, s1, s2, nv, sx, sy, sz, cf, 0, &bo, stream));
    Scratch sc(stream);
    void *dx, *dy, *dz, *dout, *dtri = nullptr, *dox = nullptr, *doy = nullptr, *doz = nullptr;
    const size_t gb = sizeof(G) * size_t(npoints), tb = sizeof(T) * size_t(npoints), ib = sizeof(int) * size_t(npoints);
    SSDF_CHECK(sc.upload(&dx, x, gb));
    SSDF_CHECK(sc.upload(&dy, y, gb));
    SSDF_CHECK(sc.upload(&dz, z, gb));
    if (output == SSDF_OUT_SDF) SSDF_CHECK(sc.alloc(&dout, tb));
    else SSDF_CHECK(sc.upload(&dout, out, tb));
    if (outtri) {
        if (output == SSDF_OUT_SDF) SSDF_CHECK(sc.alloc(&dtri, ib));
        else SSDF_CHECK(sc.upload(&dtri, outtri, ib));
    }
    if (output == SSDF_OUT_CLOSEST) {
        SSDF_CHECK(sc.upload(&dox, outx, gb));
        SSDF_CHECK(sc.upload(&doy, outy, gb));
        SSDF_CHECK(sc.upload(&doz, outz, gb));
    }
    ssdf_query_opts qo;
    memset(&qo, 0, sizeof(qo));
    qo.precision = precision;
    qo.output = output;
    qo.coord_type = cf;
    qo.out_type = sizeof(T) == 8 ? SSDF_F64 : SSDF_F32;
    SSDF_CHECK(ssdf_query_points(mg.mesh, npoints, dx, dy, dz, dout, (int *)dtri, dox, doy, doz, &qo, stream));
    SSDF_CUDA(cudaMemcpyAsync(out, dout, tb, cudaMemcpyDeviceToHost, stream));
    if (outtri) SSDF_CUDA(cudaMemcpyAsync(outtri, dtri, ib, cudaMemcpyDeviceToHost, stream));
    if (output == SSDF_OUT_CLOSEST) {
        SSDF_CUDA(cudaMemcpyAsync(outx, dox, gb, cudaMemcpyDeviceToHost, stream));
        SSDF_CUDA(cudaMemcpyAsync(outy, doy, gb, cudaMemcpyDeviceToHost, stream));
        SSDF_CUDA(cudaMemcpyAsync(outz, doz, gb, cudaMemcpyDeviceToHost, stream));
    }
    SSDF_CUDA(cudaStreamSynchronize(stream));
    return SSDF_OK;
}

template <typename G, typename T>
int bvh_grid_host(ptrdiff_t nt, const int *s0, const int *s1, const int *s2, ptrdiff_t nv, const G *sx, const G *sy,
                  const G *sz, ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz, G xmin, G ymin, G zmin, G xmax, G ymax,
                  G zmax, T *out, int *outtri, int output, int precision) {
    if (nx < 0 || ny < 0 || nz < 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "negative grid size");
    SSDF_CHECK(check_mesh_host(nt, s0, s1, s2, nv, sx, sy, sz));
    const long long n = (long long)nx * ny * nz;
    if (nt == 0 || nv == 0 || n == 0) return SSDF_OK;
    if (!out) return fail(SSDF_ERR_INVALID_ARGUMENT, "null output array");
    cudaStream_t stream;
    SSDF_CHECK(ready_stream(&stream));
    const int cf = sizeof(G) == 8 ? SSDF_F64 : SSDF_F32;
    MeshGuard mg;
    const ssdf_build_opts bo = build_opts_for(precision, output, n);
    SSDF_CHECK(ssdf_mesh_create(&mg.mesh, nt, s0, s1, s2, nv, sx, sy, sz, cf, 0, &bo, stream));
    Scratch sc(stream);
    void *dout, *dtri = nullptr;
    const size_t tb = sizeof(T) * size_t(n);
    if (output == SSDF_OUT_SDF) SSDF_CHECK(sc.alloc(&dout, tb));
    else SSDF_CHECK(sc.upload(&dout, out, tb));
    if (outtri) SSDF_CHECK(sc.alloc(&dtri, sizeof(int) * size_t(n)));
    ssdf_query_opts qo;
    memset(&qo, 0, sizeof(qo));
    qo.precision = precision;
    qo.output = output;
    qo.coord_type = cf;
    qo.out_type = sizeof(T) == 8 ? SSDF_F64 : SSDF_F32;
    const double lo[3] = {double(xmin), double(ymin), double(zmin)}, hi[3] = {double(xmax), double(ymax), double(zmax)};
    if (streamed_download_applies(n, out, outtri)) {
        // each slab chunk is copied out while the query goes on (pageable arrays through staging)
        QueryArgs a;
        SSDF_CHECK(fill_grid_args(mg.mesh, nx, ny, nz, lo, hi, dout, (int *)dtri, &qo, &a));
        return launch_query_streamed(a, qo.precision, out, outtri, stream);
    }
    SSDF_CHECK(ssdf_query_grid(mg.mesh, nx, ny, nz, lo, hi, dout, (int *)dtri, &qo, stream));
    SSDF_CUDA(cudaMemcpyAsync(out, dout, tb, cudaMemcpyDeviceToHost, stream));
    if (outtri) SSDF_CUDA(cudaMemcpyAsync(outtri, dtri, sizeof(int) * size_t(n), cudaMemcpyDeviceToHost, stream));
    SSDF_CUDA(cudaStreamSynchronize(stream));
    return SSDF_OK;
}

// edf / edf_celllist over host arrays (G == T).
template <typename T>
int dense_host(int celllist, ptrdiff_t npoints, const T *x, const T *y, const T *z, ptrdiff_t nt, const int *s0,
               const int *s1, const int *s2, ptrdiff_t nv, const T *sx, const T *sy, const T *sz, T *out,
               int *outtri) {
    if (npoints < 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "negative npoints");
    SSDF_CHECK(check_mesh_host(nt, s0, s1, s2, nv, sx, sy, sz));
    if (nt == 0 || nv == 0 || npoints == 0) return SSDF_OK;
    if (!x || !y || !z || !out) return fail(SSDF_ERR_INVALID_ARGUMENT, "null point or output array");
    cudaStream_t stream;
    SSDF_CHECK(ready_stream(&stream));
    Scratch sc(stream);
    void *dx, *dy, *dz, *dout, *ds0, *ds1, *ds2, *dsx, *dsy, *dsz, *dtri = nullptr;
    const size_t pb = sizeof(T) * size_t(npoints), vb = sizeof(T) * size_t(nv), ib = sizeof(int) * size_t(nt);
    SSDF_CHECK(sc.upload(&dx, x, pb));
    SSDF_CHECK(sc.upload(&dy, y, pb));
    SSDF_CHECK(sc.upload(&dz, z, pb));
    SSDF_CHECK(sc.upload(&dout, out, pb));
    SSDF_CHECK(sc.upload(&ds0, s0, ib));
    SSDF_CHECK(sc.upload(&ds1, s1, ib));
    SSDF_CHECK(sc.upload(&ds2, s2, ib));
    SSDF_CHECK(sc.upload(&dsx, sx, vb));
    SSDF_CHECK(sc.upload(&dsy, sy, vb));
    SSDF_CHECK(sc.upload(&dsz, sz, vb));
    if (outtri) SSDF_CHECK(sc.upload(&dtri, outtri, sizeof(int) * size_t(npoints)));
    const int f64 = sizeof(T) == 8;
    if (celllist)
        SSDF_CHECK(celllist_edf(f64, npoints, dx, dy, dz, nt, (int *)ds0, (int *)ds1, (int *)ds2, nv, dsx, dsy, dsz, dout,
                                (int *)dtri, stream));
    else
        SSDF_CHECK(brute_force_edf(f64, npoints, dx, dy, dz, nt, (int *)ds0, (int *)ds1, (int *)ds2, nv, dsx, dsy, dsz,
                                   dout, (int *)dtri, stream));
    SSDF_CUDA(cudaMemcpyAsync(out, dout, pb, cudaMemcpyDeviceToHost, stream));
    if (outtri) SSDF_CUDA(cudaMemcpyAsync(outtri, dtri, sizeof(int) * size_t(npoints), cudaMemcpyDeviceToHost, stream));
    SSDF_CUDA(cudaStreamSynchronize(stream));
    return SSDF_OK;
}

// ssdf::edf_select (serial/ssdf.hpp:965-1016), same environment variables; the BVH is this
// build's default, as it is the reference's in its cuBQL build.
template <typename T>
int edf_select_host(ptrdiff_t npoints, const T *x, const T *y, const T *z, ptrdiff_t nt, const int *s0, const int *s1,
                    const int *s2, ptrdiff_t nv, const T *sx, const T *sy, const T *sz, T *out) {
    if (env_int("SSDF_USE_BVH", 1)) {
        const int prec = precision_from_env(sizeof(T) == 8 ? SSDF_PREC_F32_FIXUP : SSDF_PREC_F32);
        return bvh_points_host<T, T>(npoints, x, y, z, nt, s0, s1, s2, nv, sx, sy, sz, out, nullptr, nullptr, nullptr,
                                     nullptr, SSDF_OUT_EDF, prec);
    }
    if (env_int("SSDF_CELL_VALIDATE", 0)) {
        if (npoints < 0 || (npoints > 0 && !out)) return fail(SSDF_ERR_INVALID_ARGUMENT, "null output array");
        std::vector<T> ref(out, out + npoints), test(out, out + npoints);
        SSDF_CHECK(dense_host<T>(0, npoints, x, y, z, nt, s0, s1, s2, nv, sx, sy, sz, ref.data(), nullptr));
        SSDF_CHECK(dense_host<T>(1, npoints, x, y, z, nt, s0, s1, s2, nv, sx, sy, sz, test.data(), nullptr));
        T max_diff = 0, diff_norm = 0;
        for (ptrdiff_t i = 0; i < npoints; ++i) {
            const T rel = std::abs(ref[i] - test[i]) / (std::abs(ref[i]) + T(1e-16));
            max_diff = std::max<T>(max_diff, rel);
            diff_norm += rel * rel;
        }
        if (max_diff > T(1e-5)) {
            fprintf(stderr, "EDF cell-list validation max rel diff: %g\n", double(max_diff));
            fprintf(stderr, "EDF cell-list validation rel diff norm: %g\n", double(std::sqrt(diff_norm)));
        }
        std::copy(test.begin(), test.end(), out);
        return SSDF_OK;
    }
    return dense_host<T>(env_int("SSDF_USE_CELL_LIST", 1) ? 1 : 0, npoints, x, y, z, nt, s0, s1, s2, nv, sx, sy, sz,
                         out, nullptr);
}

// ssdf::compute_aabb over host arrays (serial/edf/edf.hpp:500-539).
template <typename G, typename T>
int compute_aabb_host(ptrdiff_t n, const G *x, const G *y, const G *z, T *xmin, T *xmax, T *ymin, T *ymax, T *zmin,
                      T *zmax) {
    if (n <= 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "compute_aabb of no points");
    if (!x || !y || !z || !xmin || !xmax || !ymin || !ymax || !zmin || !zmax)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "compute_aabb: null pointer");
    cudaStream_t stream;
    SSDF_CHECK(ready_stream(&stream));
    T box[6];
    {
        Scratch sc(stream);
        void *dx, *dy, *dz, *db;
        SSDF_CHECK(sc.upload(&dx, x, sizeof(G) * size_t(n)));
        SSDF_CHECK(sc.upload(&dy, y, sizeof(G) * size_t(n)));
        SSDF_CHECK(sc.upload(&dz, z, sizeof(G) * size_t(n)));
        SSDF_CHECK(sc.alloc(&db, sizeof(box)));
        SSDF_CHECK((points_aabb_device<G, T>)(n, (const G *)dx, (const G *)dy, (const G *)dz, (T *)db, stream));
        SSDF_CUDA(cudaMemcpyAsync(box, db, sizeof(box), cudaMemcpyDeviceToHost, stream));
        SSDF_CUDA(cudaStreamSynchronize(stream));
    }
    *xmin = box[0], *xmax = box[1], *ymin = box[2], *ymax = box[3], *zmin = box[4], *zmax = box[5];
    return SSDF_OK;
}

// ssdf::all_points_aabb_signed_distance over host arrays (serial/edf/edf.hpp:541-557).
template <typename G, typename T>
int box_sdf_host(ptrdiff_t n, const G *x, const G *y, const G *z, T minx, T maxx, T miny, T maxy, T minz, T maxz,
                 T *out) {
    if (n < 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "negative point count");
    if (n == 0) return SSDF_OK;
    if (!x || !y || !z || !out) return fail(SSDF_ERR_INVALID_ARGUMENT, "all_points_aabb_signed_distance: null pointer");
    cudaStream_t stream;
    SSDF_CHECK(ready_stream(&stream));
    Scratch sc(stream);
    void *dx, *dy, *dz, *dout;
    SSDF_CHECK(sc.upload(&dx, x, sizeof(G) * size_t(n)));
    SSDF_CHECK(sc.upload(&dy, y, sizeof(G) * size_t(n)));
    SSDF_CHECK(sc.upload(&dz, z, sizeof(G) * size_t(n)));
    SSDF_CHECK(sc.alloc(&dout, sizeof(T) * size_t(n)));
    const T box[6] = {minx, maxx, miny, maxy, minz, maxz};
    SSDF_CHECK((points_box_sdf_device<G, T>)(n, (const G *)dx, (const G *)dy, (const G *)dz, box, 0, (T *)dout, stream));
    SSDF_CUDA(cudaMemcpyAsync(out, dout, sizeof(T) * size_t(n), cudaMemcpyDeviceToHost, stream));
    SSDF_CUDA(cudaStreamSynchronize(stream));
    return SSDF_OK;
}

}  // namespace
}  // namespace ssdf_b200

using namespace ssdf_b200;

extern "C" {

const char *ssdf_status_string(int status) {
    switch (status) {
        case SSDF_OK: return "SSDF_OK";
        case SSDF_ERR_INVALID_ARGUMENT: return "SSDF_ERR_INVALID_ARGUMENT";
        case SSDF_ERR_OUT_OF_MEMORY: return "SSDF_ERR_OUT_OF_MEMORY";
        case SSDF_ERR_CUDA: return "SSDF_ERR_CUDA";
        case SSDF_ERR_NOT_SUPPORTED: return "SSDF_ERR_NOT_SUPPORTED";
        case SSDF_ERR_INTERNAL: return "SSDF_ERR_INTERNAL";
        case SSDF_ERR_BUSY: return "SSDF_ERR_BUSY";
        default: return "SSDF_ERR_UNKNOWN";
    }
}

const char *ssdf_last_error(void) { return t_error.c_str(); }

const char *ssdf_b200_version(void) { return "ssdf_b200 0.1 (sm_100a)"; }

#define EDF_ARGS_NOOUT(G)                                                                                         \
    ptrdiff_t npoints, const G *x, const G *y, const G *z, ptrdiff_t nselements, const int *s0, const int *s1,      \
        const int *s2, ptrdiff_t nspoints, const G *sx, const G *sy, const G *sz
#define EDF_ARGS(G, T)                                                                                            \
    ptrdiff_t npoints, const G *x, const G *y, const G *z, ptrdiff_t nselements, const int *s0, const int *s1,    \
        const int *s2, ptrdiff_t nspoints, const G *sx, const G *sy, const G *sz, T *out
#define EDF_PASS npoints, x, y, z, nselements, s0, s1, s2, nspoints, sx, sy, sz, out

int ssdf_edf_f(EDF_ARGS(float, float)) { return edf_select_host<float>(EDF_PASS); }
int ssdf_edf_d(EDF_ARGS(double, double)) { return edf_select_host<double>(EDF_PASS); }

int ssdf_b200_edf_ff(EDF_ARGS(float, float)) { return dense_host<float>(0, EDF_PASS, nullptr); }
int ssdf_b200_edf_dd(EDF_ARGS(double, double)) { return dense_host<double>(0, EDF_PASS, nullptr); }
int ssdf_b200_edf_celllist_ff(EDF_ARGS(float, float)) { return dense_host<float>(1, EDF_PASS, nullptr); }
int ssdf_b200_edf_celllist_dd(EDF_ARGS(double, double)) { return dense_host<double>(1, EDF_PASS, nullptr); }

int ssdf_b200_edf_bvh_ff(EDF_ARGS(float, float)) {
    return bvh_points_host<float, float>(EDF_PASS, nullptr, nullptr, nullptr, nullptr, SSDF_OUT_EDF,
                                         precision_from_env(SSDF_PREC_F32));
}
int ssdf_b200_edf_bvh_fd(EDF_ARGS(float, double)) {
    return bvh_points_host<float, double>(EDF_PASS, nullptr, nullptr, nullptr, nullptr, SSDF_OUT_EDF,
                                          precision_from_env(SSDF_PREC_F32_FIXUP));
}
int ssdf_b200_edf_bvh_dd(EDF_ARGS(double, double)) {
    return bvh_points_host<double, double>(EDF_PASS, nullptr, nullptr, nullptr, nullptr, SSDF_OUT_EDF,
                                           precision_from_env(SSDF_PREC_F32_FIXUP));
}

int ssdf_b200_edf_index_dd(EDF_ARGS(double, double), int *outtri) {
    return bvh_points_host<double, double>(EDF_PASS, outtri, nullptr, nullptr, nullptr, SSDF_OUT_EDF,
                                           precision_from_env(SSDF_PREC_F32_FIXUP));
}
int ssdf_b200_edf_index_ff(EDF_ARGS(float, float), int *outtri) {
    return bvh_points_host<float, float>(EDF_PASS, outtri, nullptr, nullptr, nullptr, SSDF_OUT_EDF,
                                         precision_from_env(SSDF_PREC_F32));
}
int ssdf_b200_sdf_points_dd(EDF_ARGS(double, double), int *outtri) {
    return bvh_points_host<double, double>(EDF_PASS, outtri, nullptr, nullptr, nullptr, SSDF_OUT_SDF,
                                           precision_from_env(SSDF_PREC_F32_FIXUP));
}

int ssdf_b200_closest_point_bvh_ff(ptrdiff_t npoints, const float *x, const float *y, const float *z,
                                   ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                   ptrdiff_t nspoints, const float *sx, const float *sy, const float *sz, float *outd,
                                   float *outx, float *outy, float *outz, int *outtri) {
    if (npoints > 0 && nselements > 0 && (!outx || !outy || !outz || !outtri))
        return fail(SSDF_ERR_INVALID_ARGUMENT, "null closest-point output array");
    return bvh_points_host<float, float>(npoints, x, y, z, nselements, s0, s1, s2, nspoints, sx, sy, sz, outd, outtri,
                                         outx, outy, outz, SSDF_OUT_CLOSEST, precision_from_env(SSDF_PREC_F32_FIXUP));
}
// float coordinates, double distance: the double distance of the float-valued mesh and points, the
// closest point rounded to float, written where the double distance is below the incoming outd
int ssdf_b200_closest_point_bvh_fd(ptrdiff_t npoints, const float *x, const float *y, const float *z,
                                   ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                   ptrdiff_t nspoints, const float *sx, const float *sy, const float *sz, double *outd,
                                   float *outx, float *outy, float *outz, int *outtri) {
    if (npoints > 0 && nselements > 0 && (!outx || !outy || !outz || !outtri))
        return fail(SSDF_ERR_INVALID_ARGUMENT, "null closest-point output array");
    return bvh_points_host<float, double>(npoints, x, y, z, nselements, s0, s1, s2, nspoints, sx, sy, sz, outd, outtri,
                                          outx, outy, outz, SSDF_OUT_CLOSEST, precision_from_env(SSDF_PREC_F32_FIXUP));
}
int ssdf_b200_closest_point_bvh_dd(ptrdiff_t npoints, const double *x, const double *y, const double *z,
                                   ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                   ptrdiff_t nspoints, const double *sx, const double *sy, const double *sz,
                                   double *outd, double *outx, double *outy, double *outz, int *outtri) {
    if (npoints > 0 && nselements > 0 && (!outx || !outy || !outz || !outtri))
        return fail(SSDF_ERR_INVALID_ARGUMENT, "null closest-point output array");
    return bvh_points_host<double, double>(npoints, x, y, z, nselements, s0, s1, s2, nspoints, sx, sy, sz, outd,
                                           outtri, outx, outy, outz, SSDF_OUT_CLOSEST,
                                           precision_from_env(SSDF_PREC_F32_FIXUP));
}

#define GRID_ARGS(G, T)                                                                                           \
    ptrdiff_t nselements, const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints, const G *sx,           \
        const G *sy, const G *sz, ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz, G xmin, G ymin, G zmin, G xmax, G ymax, \
        G zmax, T *out
#define GRID_PASS nselements, s0, s1, s2, nspoints, sx, sy, sz, nx, ny, nz, xmin, ymin, zmin, xmax, ymax, zmax, out

int ssdf_b200_sample_sqedf_bvh_ff(GRID_ARGS(float, float)) {
    return bvh_grid_host<float, float>(GRID_PASS, nullptr, SSDF_OUT_SQEDF, precision_from_env(SSDF_PREC_F32));
}
int ssdf_b200_sample_sqedf_bvh_dd(GRID_ARGS(double, double)) {
    return bvh_grid_host<double, double>(GRID_PASS, nullptr, SSDF_OUT_SQEDF, precision_from_env(SSDF_PREC_F32_FIXUP));
}
int ssdf_b200_sample_sdf_bvh_ff(GRID_ARGS(float, float)) {
    return bvh_grid_host<float, float>(GRID_PASS, nullptr, SSDF_OUT_SDF, precision_from_env(SSDF_PREC_F32_FIXUP));
}
int ssdf_b200_sample_sdf_bvh_dd(GRID_ARGS(double, double)) {
    return bvh_grid_host<double, double>(GRID_PASS, nullptr, SSDF_OUT_SDF, precision_from_env(SSDF_PREC_F32_FIXUP));
}
int ssdf_b200_sample_sdf_index_bvh_dd(GRID_ARGS(double, double), int *outtri) {
    return bvh_grid_host<double, double>(GRID_PASS, outtri, SSDF_OUT_SDF, precision_from_env(SSDF_PREC_F32_FIXUP));
}

// ---- inside flags (serial/bvh/bvh.cpp:318-365, 1800-1866) ------------------------------------------
// 1 where the signed distance (sample_sdf_bvh's pseudo-normal rule, in double) is negative.

int ssdf_b200_points_inside_bvh_f(EDF_ARGS_NOOUT(float), uint8_t *out) {
    if (npoints > 0 && !out) return fail(SSDF_ERR_INVALID_ARGUMENT, "null output array");
    std::vector<double> d(static_cast<size_t>(npoints > 0 ? npoints : 0));
    SSDF_CHECK((bvh_points_host<float, double>(npoints, x, y, z, nselements, s0, s1, s2, nspoints, sx, sy, sz,
                                               d.data(), nullptr, nullptr, nullptr, nullptr, SSDF_OUT_SDF,
                                               precision_from_env(SSDF_PREC_F32_FIXUP))));
    if (nselements == 0 || nspoints == 0) return SSDF_OK;
    for (ptrdiff_t i = 0; i < npoints; i++) out[i] = d[size_t(i)] < 0 ? 1 : 0;
    return SSDF_OK;
}
int ssdf_b200_points_inside_bvh_d(EDF_ARGS_NOOUT(double), uint8_t *out) {
    if (npoints > 0 && !out) return fail(SSDF_ERR_INVALID_ARGUMENT, "null output array");
    std::vector<double> d(static_cast<size_t>(npoints > 0 ? npoints : 0));
    SSDF_CHECK((bvh_points_host<double, double>(npoints, x, y, z, nselements, s0, s1, s2, nspoints, sx, sy, sz,
                                                d.data(), nullptr, nullptr, nullptr, nullptr, SSDF_OUT_SDF,
                                                precision_from_env(SSDF_PREC_F32_FIXUP))));
    if (nselements == 0 || nspoints == 0) return SSDF_OK;
    for (ptrdiff_t i = 0; i < npoints; i++) out[i] = d[size_t(i)] < 0 ? 1 : 0;
    return SSDF_OK;
}

}  // extern "C"

template <typename G>
static int sample_inside_host(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints,
                       const G *sx, const G *sy, const G *sz, ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz, G xmin, G ymin,
                       G zmin, G xmax, G ymax, G zmax, uint8_t *out) {
    if (nx < 0 || ny < 0 || nz < 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "negative grid size");
    const long long n = (long long)nx * ny * nz;
    if (n > 0 && !out) return fail(SSDF_ERR_INVALID_ARGUMENT, "null output array");
    std::vector<double> d(static_cast<size_t>(n));
    SSDF_CHECK((bvh_grid_host<G, double>(nselements, s0, s1, s2, nspoints, sx, sy, sz, nx, ny, nz, xmin, ymin, zmin,
                                         xmax, ymax, zmax, d.data(), nullptr, SSDF_OUT_SDF,
                                         precision_from_env(SSDF_PREC_F32_FIXUP))));
    if (nselements == 0 || nspoints == 0) return SSDF_OK;
    for (long long i = 0; i < n; i++) out[i] = d[size_t(i)] < 0 ? 1 : 0;
    return SSDF_OK;
}

extern "C" {

int ssdf_b200_sample_inside_bvh_f(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                  ptrdiff_t nspoints, const float *sx, const float *sy, const float *sz, ptrdiff_t nx,
                                  ptrdiff_t ny, ptrdiff_t nz, float xmin, float ymin, float zmin, float xmax,
                                  float ymax, float zmax, uint8_t *out) {
    return sample_inside_host<float>(nselements, s0, s1, s2, nspoints, sx, sy, sz, nx, ny, nz, xmin, ymin, zmin, xmax,
                                     ymax, zmax, out);
}
int ssdf_b200_sample_inside_bvh_d(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                  ptrdiff_t nspoints, const double *sx, const double *sy, const double *sz,
                                  ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz, double xmin, double ymin, double zmin,
                                  double xmax, double ymax, double zmax, uint8_t *out) {
    return sample_inside_host<double>(nselements, s0, s1, s2, nspoints, sx, sy, sz, nx, ny, nz, xmin, ymin, zmin, xmax,
                                      ymax, zmax, out);
}

// ---- grid and box helpers (serial/edf/edf.hpp:500-557) ---------------------------------------------

#define AABB_ARGS(G, T)                                                                                            \
    ptrdiff_t npoints, const G *x, const G *y, const G *z, T *xmin, T *xmax, T *ymin, T *ymax, T *zmin, T *zmax
#define AABB_PASS npoints, x, y, z, xmin, xmax, ymin, ymax, zmin, zmax
int ssdf_b200_compute_aabb_ff(AABB_ARGS(float, float)) { return compute_aabb_host<float, float>(AABB_PASS); }
int ssdf_b200_compute_aabb_fd(AABB_ARGS(float, double)) { return compute_aabb_host<float, double>(AABB_PASS); }
int ssdf_b200_compute_aabb_df(AABB_ARGS(double, float)) { return compute_aabb_host<double, float>(AABB_PASS); }
int ssdf_b200_compute_aabb_dd(AABB_ARGS(double, double)) { return compute_aabb_host<double, double>(AABB_PASS); }

#define BOXSDF_ARGS(G, T)                                                                                          \
    ptrdiff_t npoints, const G *x, const G *y, const G *z, T minx, T maxx, T miny, T maxy, T minz, T maxz, T *out
#define BOXSDF_PASS npoints, x, y, z, minx, maxx, miny, maxy, minz, maxz, out
int ssdf_b200_all_points_aabb_signed_distance_ff(BOXSDF_ARGS(float, float)) {
    return box_sdf_host<float, float>(BOXSDF_PASS);
}
int ssdf_b200_all_points_aabb_signed_distance_fd(BOXSDF_ARGS(float, double)) {
    return box_sdf_host<float, double>(BOXSDF_PASS);
}
int ssdf_b200_all_points_aabb_signed_distance_df(BOXSDF_ARGS(double, float)) {
    return box_sdf_host<double, float>(BOXSDF_PASS);
}
int ssdf_b200_all_points_aabb_signed_distance_dd(BOXSDF_ARGS(double, double)) {
    return box_sdf_host<double, double>(BOXSDF_PASS);
}

int ssdf_points_aabb(ptrdiff_t npoints, const void *x, const void *y, const void *z, int coord_type, int out_type,
                     void *box6, void *stream) {
    cudaStream_t s = (cudaStream_t)stream;
    const int g64 = coord_type == SSDF_F64, t64 = out_type == SSDF_F64;
    if ((coord_type != SSDF_F32 && !g64) || (out_type != SSDF_F32 && !t64))
        return fail(SSDF_ERR_INVALID_ARGUMENT, "ssdf_points_aabb: bad coord_type / out_type");
    if (g64)
        return t64 ? points_aabb_device<double, double>(npoints, (const double *)x, (const double *)y, (const double *)z,
                                                        (double *)box6, s)
                   : points_aabb_device<double, float>(npoints, (const double *)x, (const double *)y, (const double *)z,
                                                       (float *)box6, s);
    return t64 ? points_aabb_device<float, double>(npoints, (const float *)x, (const float *)y, (const float *)z,
                                                   (double *)box6, s)
               : points_aabb_device<float, float>(npoints, (const float *)x, (const float *)y, (const float *)z,
                                                  (float *)box6, s);
}

int ssdf_points_aabb_signed_distance(ptrdiff_t npoints, const void *x, const void *y, const void *z, int coord_type,
                                     const double box6[6], int absolute, void *out, int out_type, void *stream) {
    cudaStream_t s = (cudaStream_t)stream;
    const int g64 = coord_type == SSDF_F64, t64 = out_type == SSDF_F64;
    if ((coord_type != SSDF_F32 && !g64) || (out_type != SSDF_F32 && !t64))
        return fail(SSDF_ERR_INVALID_ARGUMENT, "ssdf_points_aabb_signed_distance: bad coord_type / out_type");
    if (!box6) return fail(SSDF_ERR_INVALID_ARGUMENT, "ssdf_points_aabb_signed_distance: null box");
    if (t64) {
        return g64 ? points_box_sdf_device<double, double>(npoints, (const double *)x, (const double *)y,
                                                           (const double *)z, box6, absolute, (double *)out, s)
                   : points_box_sdf_device<float, double>(npoints, (const float *)x, (const float *)y,
                                                          (const float *)z, box6, absolute, (double *)out, s);
    }
    float b[6];
    for (int k = 0; k < 6; k++) b[k] = float(box6[k]);
    return g64 ? points_box_sdf_device<double, float>(npoints, (const double *)x, (const double *)y, (const double *)z,
                                                      b, absolute, (float *)out, s)
               : points_box_sdf_device<float, float>(npoints, (const float *)x, (const float *)y, (const float *)z, b,
                                                     absolute, (float *)out, s);
}

// ---- handle API ---------------------------------------------------------------------------------------

int ssdf_mesh_create(ssdf_mesh **mesh, ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                     ptrdiff_t nspoints, const void *sx, const void *sy, const void *sz, int coord_type,
                     int device_ptrs, const ssdf_build_opts *opts, void *stream) {
    if (!mesh) return fail(SSDF_ERR_INVALID_ARGUMENT, "null mesh handle pointer");
    *mesh = nullptr;
    if (coord_type != SSDF_F32 && coord_type != SSDF_F64) return fail(SSDF_ERR_INVALID_ARGUMENT, "bad coord_type");
    ssdf_build_opts o;
    if (opts) {
        o = *opts;
    } else {
        o.leaf_size = 0, o.keep_fp64 = 1, o.normals = 1, o.treelet_opt = kResidentTreeletRounds;
    }
    if (!device_ptrs) SSDF_CHECK(check_mesh_host(nselements, s0, s1, s2, nspoints, sx, sy, sz));
    cudaStream_t s = (cudaStream_t)stream;
    ssdf_mesh *h = new ssdf_mesh();
    cudaGetDevice(&h->device);
    const int st = mesh_build(&h->storage, &h->m, nselements, s0, s1, s2, nspoints, sx, sy, sz,
                              coord_type == SSDF_F64, device_ptrs, o, s);
    if (st != SSDF_OK) {
        delete h;
        return st;
    }
    *mesh = h;
    return SSDF_OK;
}

int ssdf_mesh_destroy(ssdf_mesh *mesh) {
    if (!mesh) return SSDF_OK;
    // queries still running on any stream may read the mesh: wait for its device first (its storage is
    // pool memory, which cudaFree releases without waiting)
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != mesh->device) cudaSetDevice(mesh->device);
    const cudaError_t e = cudaDeviceSynchronize();
    mesh_free(mesh->storage);
    if (prev != mesh->device) cudaSetDevice(prev);
    delete mesh;
    if (e != cudaSuccess) return cuda_fail(e, "ssdf_mesh_destroy", __FILE__, __LINE__);
    return SSDF_OK;
}

int ssdf_mesh_destroy_async(ssdf_mesh *mesh, void *stream) {
    if (!mesh) return SSDF_OK;
    mesh_free_async(mesh->storage, (cudaStream_t)stream);
    delete mesh;
    return SSDF_OK;
}

int ssdf_mesh_filter_info(const ssdf_mesh *mesh, float *tau_rel, int *float_filter, int64_t *slivers) {
    if (!mesh) return fail(SSDF_ERR_INVALID_ARGUMENT, "null mesh");
    if (tau_rel) *tau_rel = mesh->m.tau_rel_min;
    if (float_filter) *float_filter = mesh->m.filt32 && !fixup_runs_f64(mesh->m) ? 1 : 0;
    if (slivers) *slivers = mesh->m.nill;
    return SSDF_OK;
}

int ssdf_mesh_stats(const ssdf_mesh *mesh, int64_t *nodes, int64_t *leaves, int64_t *depth, int64_t *bytes) {
    if (!mesh) return fail(SSDF_ERR_INVALID_ARGUMENT, "null mesh");
    if (nodes) *nodes = mesh->m.nnodes;
    if (leaves) *leaves = mesh->m.nleaves;
    if (depth) *depth = mesh->m.depth;
    if (bytes) *bytes = (int64_t)mesh_bytes(mesh->storage);
    return SSDF_OK;
}

}  // extern "C"

namespace ssdf_b200 {

static int fill_query(const ssdf_mesh *mesh, const ssdf_query_opts *opts, QueryArgs *a) {
    if (!mesh) return fail(SSDF_ERR_INVALID_ARGUMENT, "null mesh");
    if (!opts) return fail(SSDF_ERR_INVALID_ARGUMENT, "null query options");
    if (opts->output < SSDF_OUT_EDF || opts->output > SSDF_OUT_CLOSEST) return fail(SSDF_ERR_INVALID_ARGUMENT, "bad output");
    if (opts->precision < SSDF_PREC_F32 || opts->precision > SSDF_PREC_F32_FIXUP)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "bad precision");
    memset(a, 0, sizeof(*a));
    a->m = mesh->m;
    a->output = opts->output;
    a->coord_f64 = opts->coord_type == SSDF_F64;
    a->out_f64 = opts->out_type == SSDF_F64;
    // the mesh's own minimum (wider for meshes of a few large triangles); the environment may only widen it
    a->tau_rel = std::max(tau_rel_from_env(), mesh->m.tau_rel_min);
    a->warp_budget = env_int("SSDF_B200_WARP_BUDGET", -1);
    a->seed = env_int("SSDF_B200_SEED", 1) != 0 ? 1 : 0;
    return SSDF_OK;
}

int fill_point_args(ssdf_mesh *mesh, ptrdiff_t npoints, const void *x, const void *y, const void *z, void *out,
                    int *outtri, void *outx, void *outy, void *outz, const ssdf_query_opts *opts, QueryArgs *a) {
    SSDF_CHECK(fill_query(mesh, opts, a));
    if (npoints < 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "negative npoints");
    if (npoints > 0 && (!x || !y || !z || !out)) return fail(SSDF_ERR_INVALID_ARGUMENT, "null point or output array");
    a->is_grid = 0;
    a->npoints = npoints;
    a->x = x, a->y = y, a->z = z;
    a->out = out;
    a->outtri = outtri;
    a->outx = outx, a->outy = outy, a->outz = outz;
    return SSDF_OK;
}

int fill_grid_args(ssdf_mesh *mesh, ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz, const double lo[3], const double hi[3],
                   void *out, int *outtri, const ssdf_query_opts *opts, QueryArgs *a) {
    SSDF_CHECK(fill_query(mesh, opts, a));
    if (nx < 0 || ny < 0 || nz < 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "negative grid size");
    if ((long long)nx * ny * nz > 0 && (!lo || !hi || !out))
        return fail(SSDF_ERR_INVALID_ARGUMENT, "null grid bounds or output array");
    if (opts->output == SSDF_OUT_CLOSEST) return fail(SSDF_ERR_INVALID_ARGUMENT, "closest-point output is for point lists");
    a->is_grid = 1;
    a->nx = nx, a->ny = ny, a->nz = nz;
    const long long n[3] = {nx, ny, nz};
    for (int d = 0; d < 3 && lo && hi; d++) {
        // h = (max - min) / (n - 1) in G precision (serial/bvh/bvh.cpp:1665-1667)
        a->lo64[d] = lo[d];
        a->h64[d] = n[d] > 1 ? (hi[d] - lo[d]) / double(n[d] - 1) : 0.0;
        a->lo32[d] = float(lo[d]);
        a->h32[d] = n[d] > 1 ? (float(hi[d]) - float(lo[d])) / float(n[d] - 1) : 0.f;
    }
    a->out = out;
    a->outtri = outtri;
    set_grid_steps(a);
    return SSDF_OK;
}

}  // namespace ssdf_b200

extern "C" {

int ssdf_edf_device(int method, ptrdiff_t npoints, const void *x, const void *y, const void *z, ptrdiff_t nselements,
                    const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints, const void *sx, const void *sy,
                    const void *sz, int coord_type, void *out, int *outtri, void *stream) {
    if (method != 0 && method != 1) return fail(SSDF_ERR_INVALID_ARGUMENT, "ssdf_edf_device: method 0 (edf) or 1 (celllist)");
    if (coord_type != SSDF_F32 && coord_type != SSDF_F64) return fail(SSDF_ERR_INVALID_ARGUMENT, "bad coord_type");
    if (npoints < 0 || nselements < 0 || nspoints < 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "negative size");
    if (npoints == 0 || nselements == 0 || nspoints == 0) return SSDF_OK;
    if (!x || !y || !z || !out || !s0 || !s1 || !s2 || !sx || !sy || !sz)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "null array");
    const int f64 = coord_type == SSDF_F64;
    const cudaStream_t st = (cudaStream_t)stream;
    return method == 0 ? brute_force_edf(f64, npoints, x, y, z, nselements, s0, s1, s2, nspoints, sx, sy, sz, out, outtri, st)
                       : celllist_edf(f64, npoints, x, y, z, nselements, s0, s1, s2, nspoints, sx, sy, sz, out, outtri, st);
}

int ssdf_query_points(ssdf_mesh *mesh, ptrdiff_t npoints, const void *x, const void *y, const void *z, void *out,
                      int *outtri, void *outx, void *outy, void *outz, const ssdf_query_opts *opts, void *stream) {
    QueryArgs a;
    SSDF_CHECK(fill_point_args(mesh, npoints, x, y, z, out, outtri, outx, outy, outz, opts, &a));
    if (npoints == 0) return SSDF_OK;
    return launch_query(a, opts->precision, (cudaStream_t)stream);
}

int ssdf_query_grid(ssdf_mesh *mesh, ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz, const double lo[3], const double hi[3],
                    void *out, int *outtri, const ssdf_query_opts *opts, void *stream) {
    QueryArgs a;
    SSDF_CHECK(fill_grid_args(mesh, nx, ny, nz, lo, hi, out, outtri, opts, &a));
    if ((long long)nx * ny * nz == 0) return SSDF_OK;
    return launch_query(a, opts->precision, (cudaStream_t)stream);
}

// The fix-up grid query without any allocation (its overflow list lives in a fixed device array
// of the library): for callers that must not allocate device memory while they query.
int ssdf_query_grid_noalloc(ssdf_mesh *mesh, ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz, const double lo[3],
                            const double hi[3], void *out, int *outtri, const ssdf_query_opts *opts, void *stream) {
    QueryArgs a;
    SSDF_CHECK(fill_grid_args(mesh, nx, ny, nz, lo, hi, out, outtri, opts, &a));
    if (opts->precision != SSDF_PREC_F32_FIXUP)
        return fail(SSDF_ERR_INVALID_ARGUMENT,
                    "ssdf_query_grid_noalloc runs the fix-up arithmetic (SSDF_PREC_F32_FIXUP) only");
    if ((long long)nx * ny * nz == 0) return SSDF_OK;
    return launch_query_noalloc(a, (cudaStream_t)stream);
}

long long ssdf_query_grid_noalloc_max(void) { return noalloc_max_queries(); }

int ssdf_last_query_counts(int64_t *triangle_tests, int64_t *box_tests, int64_t *fixup_queries,
                           int64_t *fallback_queries) {
    return query_counts(triangle_tests, box_tests, fixup_queries, fallback_queries);
}

}  // extern "C"
