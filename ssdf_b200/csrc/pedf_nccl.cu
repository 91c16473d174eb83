// pedf_nccl.cu -- ssdf::pedf and ssdf::pedf_update (distributed/psdf.hpp:149-302, 304-482) over an
// NCCL communicator, on device arrays.
//
// The reference exchanges surface parts with MPI and queries on the host. Here one process per GPU
// holds its points and its part of the surface in device memory, the exchanges are NCCL collectives
// on the caller's stream, and the distances come from this library's BVH query:
//   pedf, SSDF_USE_ALLGATHER=1 (default): every rank's part is gathered (sizes all-gathered, then one
//     broadcast per part inside an NCCL group) with its triangle indices shifted by the vertices of
//     the ranks before it, and out = min(out, distance to the whole surface);
//   pedf, SSDF_USE_ALLGATHER=0: the parts are broadcast one after the other and out is updated with
//     each (the reference's low-memory mode);
//   pedf_update: the box of this rank's points grown by their distances is all-gathered, every rank
//     sends each other rank the corners of its triangles meeting that rank's box (send / receive
//     pairs inside an NCCL group, counts exchanged first), and out is updated with the received
//     triangles (exchange.cu holds the selection kernels).
// The result is that of the single-process drop-in on the whole surface, bit for bit: the query takes
// the lexicographic minimum over every triangle it meets, whatever their order.
//
// NCCL is opened at the first call (dlopen of libnccl.so.2: the library a process has already loaded
// under that name, for instance PyTorch's, or the system's), so the library itself does not depend on
// NCCL and loads where there is none; these entry points then return SSDF_ERR_NOT_SUPPORTED.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "internal.h"

namespace ssdf_b200 {
namespace {

// The drop-in edf's arithmetic for an out of this type, or SSDF_B200_PRECISION's.
int out_precision(bool out_f64) {
    const char *v = env_str("SSDF_B200_PRECISION");
    if (v && !strcmp(v, "f64")) return SSDF_PREC_F64;
    if (v && !strcmp(v, "f32")) return SSDF_PREC_F32;
    if (v && (!strcmp(v, "f32x") || !strcmp(v, "fixup"))) return SSDF_PREC_F32_FIXUP;
    return out_f64 ? SSDF_PREC_F32_FIXUP : SSDF_PREC_F32;
}

struct NcclApi {
    decltype(&ncclAllGather) all_gather = nullptr;
    decltype(&ncclBroadcast) broadcast = nullptr;
    decltype(&ncclSend) send = nullptr;
    decltype(&ncclRecv) recv = nullptr;
    decltype(&ncclGroupStart) group_start = nullptr;
    decltype(&ncclGroupEnd) group_end = nullptr;
    decltype(&ncclCommCount) count = nullptr;
    decltype(&ncclCommUserRank) user_rank = nullptr;
    decltype(&ncclGetErrorString) error_string = nullptr;
    std::string why;
};

const NcclApi &nccl() {
    static NcclApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h) {
            api.why = std::string("libnccl.so.2 not found: ") + dlerror();
            return;
        }
        auto sym = [&](const char *n) { return dlsym(h, n); };
        api.all_gather = (decltype(api.all_gather))sym("ncclAllGather");
        api.broadcast = (decltype(api.broadcast))sym("ncclBroadcast");
        api.send = (decltype(api.send))sym("ncclSend");
        api.recv = (decltype(api.recv))sym("ncclRecv");
        api.group_start = (decltype(api.group_start))sym("ncclGroupStart");
        api.group_end = (decltype(api.group_end))sym("ncclGroupEnd");
        api.count = (decltype(api.count))sym("ncclCommCount");
        api.user_rank = (decltype(api.user_rank))sym("ncclCommUserRank");
        api.error_string = (decltype(api.error_string))sym("ncclGetErrorString");
        if (!api.all_gather || !api.broadcast || !api.send || !api.recv || !api.group_start || !api.group_end ||
            !api.count || !api.user_rank || !api.error_string)
            api.why = "libnccl.so.2 lacks a needed symbol";
    });
    return api;
}

#define NCCL_TRY(call)                                                                                       \
    do {                                                                                                     \
        const ncclResult_t r_ = (call);                                                                      \
        if (r_ != ncclSuccess)                                                                               \
            return fail(SSDF_ERR_CUDA, std::string("NCCL: ") + #call + ": " + nccl().error_string(r_));     \
    } while (0)

// Device buffers released (stream-ordered) when the call returns.
struct Pool {
    cudaStream_t s;
    std::vector<void *> p;
    ~Pool() {
        for (void *q : p) cudaFreeAsync(q, s);
    }
    template <typename X>
    int get(X **out, size_t n) {
        *out = nullptr;
        if (n == 0) n = 1;
        const cudaError_t e = cudaMallocAsync((void **)out, sizeof(X) * n, s);
        if (e != cudaSuccess) return cuda_fail(e, "pedf scratch", __FILE__, __LINE__);
        p.push_back(*out);
        return SSDF_OK;
    }
};

template <typename G>
ncclDataType_t nccl_type() {
    return sizeof(G) == 8 ? ncclFloat64 : ncclFloat32;
}

// dst[i] = src[i] + shift, i < n (one part's indices into the gathered vertex numbering)
__global__ void k_shift(long long n, const int *__restrict__ src, int shift, int *__restrict__ dst) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[i] + shift;
}

// corners [m][9] -> soup: indices 3t, 3t + 1, 3t + 2 and vertex SoA in corner order
template <typename G>
__global__ void k_corner_soup(long long m, const G *__restrict__ c, int *__restrict__ s0, int *__restrict__ s1,
                              int *__restrict__ s2, G *__restrict__ vx, G *__restrict__ vy, G *__restrict__ vz) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= m) return;
    s0[t] = int(3 * t), s1[t] = int(3 * t + 1), s2[t] = int(3 * t + 2);
    for (int k = 0; k < 3; k++) {
        vx[3 * t + k] = c[9 * t + 3 * k];
        vy[3 * t + k] = c[9 * t + 3 * k + 1];
        vz[3 * t + k] = c[9 * t + 3 * k + 2];
    }
}

inline unsigned nblk(long long n) { return unsigned((n + 255) / 256); }

// out = min(out, distance to the triangles), on this library's BVH, in the drop-in edf's arithmetic for
// out's type (SSDF_B200_PRECISION overrides); waits for the query.
template <typename G, typename T>
int edf_inout(long long np, const G *x, const G *y, const G *z, T *out, long long nt, const int *s0, const int *s1,
              const int *s2, long long nv, const G *sx, const G *sy, const G *sz, cudaStream_t s) {
    if (np == 0 || nt == 0 || nv == 0) return SSDF_OK;
    const int prec = out_precision(sizeof(T) == 8);
    const int ct = sizeof(G) == 8 ? SSDF_F64 : SSDF_F32;
    ssdf_build_opts bo;
    bo.leaf_size = 0, bo.keep_fp64 = prec != SSDF_PREC_F32, bo.normals = 0, bo.treelet_opt = 1;
    ssdf_mesh *m = nullptr;
    SSDF_CHECK(ssdf_mesh_create(&m, ptrdiff_t(nt), s0, s1, s2, ptrdiff_t(nv), sx, sy, sz, ct, 1, &bo, s));
    ssdf_query_opts qo;
    memset(&qo, 0, sizeof(qo));
    qo.precision = prec, qo.output = SSDF_OUT_EDF, qo.coord_type = ct, qo.out_type = sizeof(T) == 8 ? SSDF_F64 : SSDF_F32;
    int st = ssdf_query_points(m, ptrdiff_t(np), x, y, z, out, nullptr, nullptr, nullptr, nullptr, &qo, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    ssdf_mesh_destroy(m);
    if (st == SSDF_OK && e != cudaSuccess) st = cuda_fail(e, "pedf query", __FILE__, __LINE__);
    return st;
}

// Sizes (triangles, vertices) of every rank's part, all-gathered.
int part_sizes(ncclComm_t comm, int world, long long nt, long long nv, std::vector<long long> &sizes, Pool &pool,
               cudaStream_t s) {
    long long *d = nullptr;
    SSDF_CHECK(pool.get(&d, 2 * size_t(world) + 2));
    const long long mine[2] = {nt, nv};
    SSDF_CUDA(cudaMemcpyAsync(d + 2 * world, mine, sizeof(mine), cudaMemcpyHostToDevice, s));
    NCCL_TRY(nccl().all_gather(d + 2 * world, d, 2, ncclInt64, comm, s));
    sizes.assign(2 * size_t(world), 0);
    SSDF_CUDA(cudaMemcpyAsync(sizes.data(), d, sizeof(long long) * 2 * world, cudaMemcpyDeviceToHost, s));
    SSDF_CUDA(cudaStreamSynchronize(s));
    return SSDF_OK;
}

template <typename G, typename T>
int pedf_impl(ncclComm_t comm, int use_allgather, long long np, const G *x, const G *y, const G *z, long long nt,
              const int *s0, const int *s1, const int *s2, long long nv, const G *sx, const G *sy, const G *sz,
              T *out, cudaStream_t s) {
    const NcclApi &api = nccl();
    int world = 0, me = 0;
    NCCL_TRY(api.count(comm, &world));
    NCCL_TRY(api.user_rank(comm, &me));
    Pool pool{s, {}};
    std::vector<long long> sz_;
    SSDF_CHECK(part_sizes(comm, world, nt, nv, sz_, pool, s));
    // this rank's part, packed: indices s0 | s1 | s2, vertices x | y | z
    int *lidx = nullptr;
    G *lv = nullptr;
    SSDF_CHECK(pool.get(&lidx, 3 * size_t(nt)));
    SSDF_CHECK(pool.get(&lv, 3 * size_t(nv)));
    if (nt > 0) {
        SSDF_CUDA(cudaMemcpyAsync(lidx, s0, sizeof(int) * nt, cudaMemcpyDeviceToDevice, s));
        SSDF_CUDA(cudaMemcpyAsync(lidx + nt, s1, sizeof(int) * nt, cudaMemcpyDeviceToDevice, s));
        SSDF_CUDA(cudaMemcpyAsync(lidx + 2 * nt, s2, sizeof(int) * nt, cudaMemcpyDeviceToDevice, s));
    }
    if (nv > 0) {
        SSDF_CUDA(cudaMemcpyAsync(lv, sx, sizeof(G) * nv, cudaMemcpyDeviceToDevice, s));
        SSDF_CUDA(cudaMemcpyAsync(lv + nv, sy, sizeof(G) * nv, cudaMemcpyDeviceToDevice, s));
        SSDF_CUDA(cudaMemcpyAsync(lv + 2 * nv, sz, sizeof(G) * nv, cudaMemcpyDeviceToDevice, s));
    }
    long long NT = 0, NV = 0;
    std::vector<long long> toff(world), voff(world);
    for (int r = 0; r < world; r++) toff[r] = NT, voff[r] = NV, NT += sz_[2 * r], NV += sz_[2 * r + 1];
    if (NT >= 0x7fffffffll || NV >= 0x7fffffffll) return fail(SSDF_ERR_NOT_SUPPORTED, "pedf: more than 2^31 - 1 elements");
    if (use_allgather) {
        int *gidx = nullptr, *S = nullptr;
        G *gv = nullptr, *V = nullptr;
        SSDF_CHECK(pool.get(&gidx, 3 * size_t(NT)));
        SSDF_CHECK(pool.get(&gv, 3 * size_t(NV)));
        SSDF_CHECK(pool.get(&S, 3 * size_t(NT)));
        SSDF_CHECK(pool.get(&V, 3 * size_t(NV)));
        NCCL_TRY(api.group_start());
        for (int r = 0; r < world; r++) {
            const long long ntr = sz_[2 * r], nvr = sz_[2 * r + 1];
            if (ntr > 0) NCCL_TRY(api.broadcast(lidx, gidx + 3 * toff[r], size_t(3 * ntr), ncclInt32, r, comm, s));
            if (nvr > 0) NCCL_TRY(api.broadcast(lv, gv + 3 * voff[r], size_t(3 * nvr), nccl_type<G>(), r, comm, s));
        }
        NCCL_TRY(api.group_end());
        // gathered numbering: rank r's triangles (indices shifted by the vertices before it), in rank order
        for (int r = 0; r < world; r++) {
            const long long ntr = sz_[2 * r], nvr = sz_[2 * r + 1];
            for (int k = 0; k < 3 && ntr > 0; k++)
                k_shift<<<nblk(ntr), 256, 0, s>>>(ntr, gidx + 3 * toff[r] + k * ntr, int(voff[r]), S + k * NT + toff[r]);
            for (int k = 0; k < 3 && nvr > 0; k++)
                SSDF_CUDA(cudaMemcpyAsync(V + k * NV + voff[r], gv + 3 * voff[r] + k * nvr, sizeof(G) * nvr,
                                          cudaMemcpyDeviceToDevice, s));
        }
        SSDF_CUDA(cudaGetLastError());
        return edf_inout<G, T>(np, x, y, z, out, NT, S, S + NT, S + 2 * NT, NV, V, V + NV, V + 2 * NV, s);
    }
    // broadcast mode: one part after the other, out carrying the minimum
    for (int r = 0; r < world; r++) {
        const long long ntr = sz_[2 * r], nvr = sz_[2 * r + 1];
        if (ntr == 0 || nvr == 0) continue;
        int *pidx = nullptr;
        G *pv = nullptr;
        SSDF_CHECK(pool.get(&pidx, 3 * size_t(ntr)));
        SSDF_CHECK(pool.get(&pv, 3 * size_t(nvr)));
        NCCL_TRY(api.group_start());
        NCCL_TRY(api.broadcast(lidx, pidx, size_t(3 * ntr), ncclInt32, r, comm, s));
        NCCL_TRY(api.broadcast(lv, pv, size_t(3 * nvr), nccl_type<G>(), r, comm, s));
        NCCL_TRY(api.group_end());
        SSDF_CHECK((edf_inout<G, T>(np, x, y, z, out, ntr, pidx, pidx + ntr, pidx + 2 * ntr, nvr, pv, pv + nvr,
                                    pv + 2 * nvr, s)));
    }
    return SSDF_OK;
}

template <typename G, typename T>
int pedf_update_impl(ncclComm_t comm, long long np, const G *x, const G *y, const G *z, long long nt, const int *s0,
                     const int *s1, const int *s2, long long nv, const G *sx, const G *sy, const G *sz, T *out,
                     cudaStream_t s) {
    const NcclApi &api = nccl();
    int world = 0, me = 0;
    NCCL_TRY(api.count(comm, &world));
    NCCL_TRY(api.user_rank(comm, &me));
    Pool pool{s, {}};
    const int ct = sizeof(G) == 8 ? SSDF_F64 : SSDF_F32, ot = sizeof(T) == 8 ? SSDF_F64 : SSDF_F32;
    // 1. grown boxes of every rank's points
    G *boxes = nullptr;
    SSDF_CHECK(pool.get(&boxes, 6 * size_t(world) + 6));
    SSDF_CHECK(ssdf_grown_box(ptrdiff_t(np), x, y, z, out, ct, ot, boxes + 6 * world, s));
    NCCL_TRY(api.all_gather(boxes + 6 * world, boxes, 6, nccl_type<G>(), comm, s));
    // 2. this rank's triangles meeting each box, box after box
    std::vector<long long> send(world, 0), recv(world, 0);
    SSDF_CHECK(ssdf_triangles_meeting_boxes(ptrdiff_t(nt), s0, s1, s2, ptrdiff_t(nv), sx, sy, sz, ct, world, boxes,
                                            nullptr, 0, send.data(), s));
    long long total = 0;
    for (long long c : send) total += c;
    G *corners = nullptr;
    SSDF_CHECK(pool.get(&corners, 9 * size_t(total)));
    if (total > 0)
        SSDF_CHECK(ssdf_triangles_meeting_boxes(ptrdiff_t(nt), s0, s1, s2, ptrdiff_t(nv), sx, sy, sz, ct, world, boxes,
                                                corners, total, send.data(), s));
    // 3. counts: every rank's row all-gathered; this rank receives column `me`
    long long *cnt = nullptr;
    SSDF_CHECK(pool.get(&cnt, size_t(world) * world + world));
    SSDF_CUDA(cudaMemcpyAsync(cnt + size_t(world) * world, send.data(), sizeof(long long) * world,
                              cudaMemcpyHostToDevice, s));
    NCCL_TRY(api.all_gather(cnt + size_t(world) * world, cnt, size_t(world), ncclInt64, comm, s));
    std::vector<long long> all(size_t(world) * world);
    SSDF_CUDA(cudaMemcpyAsync(all.data(), cnt, sizeof(long long) * all.size(), cudaMemcpyDeviceToHost, s));
    SSDF_CUDA(cudaStreamSynchronize(s));
    long long M = 0;
    std::vector<long long> soff(world), roff(world);
    for (int r = 0, o = 0; r < world; r++) soff[r] = o, o += int(send[r]);
    for (int r = 0; r < world; r++) recv[r] = all[size_t(r) * world + me], roff[r] = M, M += recv[r];
    if (M >= 0x7fffffffll / 3) return fail(SSDF_ERR_NOT_SUPPORTED, "pedf_update: too many candidate triangles");
    // 4. the candidates: send / receive pairs in one group
    G *got = nullptr;
    SSDF_CHECK(pool.get(&got, 9 * size_t(M)));
    NCCL_TRY(api.group_start());
    for (int r = 0; r < world; r++) {
        if (send[r] > 0) NCCL_TRY(api.send(corners + 9 * soff[r], size_t(9 * send[r]), nccl_type<G>(), r, comm, s));
        if (recv[r] > 0) NCCL_TRY(api.recv(got + 9 * roff[r], size_t(9 * recv[r]), nccl_type<G>(), r, comm, s));
    }
    NCCL_TRY(api.group_end());
    if (M == 0) return SSDF_OK;
    // 5. out = min(out, distance to the received triangles)
    int *S = nullptr;
    G *V = nullptr;
    SSDF_CHECK(pool.get(&S, 3 * size_t(M)));
    SSDF_CHECK(pool.get(&V, 9 * size_t(M)));
    k_corner_soup<G><<<nblk(M), 256, 0, s>>>(M, got, S, S + M, S + 2 * M, V, V + 3 * M, V + 6 * M);
    SSDF_CUDA(cudaGetLastError());
    return edf_inout<G, T>(np, x, y, z, out, M, S, S + M, S + 2 * M, 3 * M, V, V + 3 * M, V + 6 * M, s);
}

template <typename F>
int with_types(int coord_type, int out_type, F f) {
    if (coord_type == SSDF_F64 && out_type == SSDF_F64) return f((double *)nullptr, (double *)nullptr);
    if (coord_type == SSDF_F32 && out_type == SSDF_F64) return f((float *)nullptr, (double *)nullptr);
    if (coord_type == SSDF_F32 && out_type == SSDF_F32) return f((float *)nullptr, (float *)nullptr);
    return fail(SSDF_ERR_INVALID_ARGUMENT, "pedf: <double, double>, <float, double> or <float, float>");
}

int check_args(void *comm, ptrdiff_t np, const void *x, const void *y, const void *z, ptrdiff_t nt, const int *s0,
               const int *s1, const int *s2, ptrdiff_t nv, const void *sx, const void *sy, const void *sz, void *out) {
    if (!nccl().why.empty()) return fail(SSDF_ERR_NOT_SUPPORTED, "pedf over NCCL: " + nccl().why);
    if (!comm || np < 0 || nt < 0 || nv < 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "pedf: bad arguments");
    if (np > 0 && (!x || !y || !z || !out)) return fail(SSDF_ERR_INVALID_ARGUMENT, "pedf: null point array");
    if (nt > 0 && (!s0 || !s1 || !s2 || !sx || !sy || !sz || nv == 0))
        return fail(SSDF_ERR_INVALID_ARGUMENT, "pedf: null surface array");
    return SSDF_OK;
}

}  // namespace
}  // namespace ssdf_b200

using namespace ssdf_b200;

extern "C" {

int ssdf_pedf_nccl(void *comm, ptrdiff_t npoints, const void *x, const void *y, const void *z, ptrdiff_t nselements,
                   const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints, const void *sx, const void *sy,
                   const void *sz, int coord_type, int out_type, void *out, void *stream) {
    SSDF_CHECK(check_args(comm, npoints, x, y, z, nselements, s0, s1, s2, nspoints, sx, sy, sz, out));
    const int allgather = env_int("SSDF_USE_ALLGATHER", 1) != 0;
    return with_types(coord_type, out_type, [&](auto *g, auto *t) {
        using G = std::remove_pointer_t<decltype(g)>;
        using T = std::remove_pointer_t<decltype(t)>;
        return pedf_impl<G, T>((ncclComm_t)comm, allgather, npoints, (const G *)x, (const G *)y, (const G *)z,
                               nselements, s0, s1, s2, nspoints, (const G *)sx, (const G *)sy, (const G *)sz, (T *)out,
                               (cudaStream_t)stream);
    });
}

int ssdf_pedf_update_nccl(void *comm, ptrdiff_t npoints, const void *x, const void *y, const void *z,
                          ptrdiff_t nselements, const int *s0, const int *s1, const int *s2, ptrdiff_t nspoints,
                          const void *sx, const void *sy, const void *sz, int coord_type, int out_type, void *out,
                          void *stream) {
    SSDF_CHECK(check_args(comm, npoints, x, y, z, nselements, s0, s1, s2, nspoints, sx, sy, sz, out));
    return with_types(coord_type, out_type, [&](auto *g, auto *t) {
        using G = std::remove_pointer_t<decltype(g)>;
        using T = std::remove_pointer_t<decltype(t)>;
        return pedf_update_impl<G, T>((ncclComm_t)comm, npoints, (const G *)x, (const G *)y, (const G *)z,
                                      nselements, s0, s1, s2, nspoints, (const G *)sx, (const G *)sy, (const G *)sz,
                                      (T *)out, (cudaStream_t)stream);
    });
}

}  // extern "C"
