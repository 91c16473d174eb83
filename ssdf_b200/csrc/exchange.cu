// exchange.cu -- the selection steps of pedf_update (distributed/psdf.hpp:327-470) on the device.
//
// pedf_update sends each rank only the triangles that can improve its points' current distances:
//   1. every rank grows the box of its points by their distances, [min(p - r), max(p + r)] per axis in
//      the coordinates' type (psdf.hpp:327-361); the boxes are all-gathered by the caller;
//   2. for each rank's box, the local triangles whose corner box meets it (closed intervals,
//      psdf.hpp:378-389, 391-452) are compacted, in triangle order, into one array of corner triples,
//      box after box, ready for an all-to-all.
// The reference sends each rank the unique vertices and re-indexed triangles; this sends the corners
// of each triangle (the distances are the same).
//
// The box is a min/max reduction that skips NaN values as std::min / std::max do when the running
// value comes first, so the result does not depend on the order of the reduction. The compaction is a
// flag pass, an exclusive scan and a scatter per box, so the order is the triangles' own.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <string>
#include <vector>

#include "internal.h"

namespace ssdf_b200 {
namespace {

constexpr int kExThreads = 256;
constexpr int kExBlocks = 296;  // two waves of reduction blocks on 148 SMs

template <typename G>
__device__ __forceinline__ G lowest_g();
template <>
__device__ __forceinline__ float lowest_g<float>() {
    return -FLT_MAX;
}
template <>
__device__ __forceinline__ double lowest_g<double>() {
    return -DBL_MAX;
}

// Per-block partial boxes of the points grown by their distances: part[6 b .. 6 b + 5] = min x, y, z,
// max x, y, z of the block's points (a NaN never replaces the running value).
template <typename G, typename T>
__global__ void __launch_bounds__(kExThreads) k_grown_partial(long long n, const G *__restrict__ x,
                                                              const G *__restrict__ y, const G *__restrict__ z,
                                                              const T *__restrict__ out, G *__restrict__ part) {
    G v[6];
    for (int d = 0; d < 3; d++) v[d] = -lowest_g<G>(), v[3 + d] = lowest_g<G>();
    for (long long i = blockIdx.x * (long long)kExThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kExThreads) {
        const G r = G(out[i]);
        const G p[3] = {x[i], y[i], z[i]};
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const G lo = p[d] - r, hi = p[d] + r;
            v[d] = lo < v[d] ? lo : v[d];
            v[3 + d] = v[3 + d] < hi ? hi : v[3 + d];
        }
    }
    __shared__ G s[6][kExThreads];
    for (int k = 0; k < 6; k++) s[k][threadIdx.x] = v[k];
    __syncthreads();
    for (int w = kExThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int k = 0; k < 6; k++) {
                const G o = s[k][threadIdx.x + w], m = s[k][threadIdx.x];
                s[k][threadIdx.x] = k < 3 ? (o < m ? o : m) : (m < o ? o : m);
            }
        __syncthreads();
    }
    if (threadIdx.x < 6) part[6 * blockIdx.x + threadIdx.x] = s[threadIdx.x][0];
}

template <typename G>
__global__ void k_grown_final(int nparts, const G *__restrict__ part, G *__restrict__ box) {
    if (threadIdx.x >= 6) return;
    const int k = threadIdx.x;
    G m = k < 3 ? -lowest_g<G>() : lowest_g<G>();
    for (int b = 0; b < nparts; b++) {
        const G o = part[6 * b + k];
        m = k < 3 ? (o < m ? o : m) : (m < o ? o : m);
    }
    box[k] = m;
}

// flag[t] = 1 when triangle t's corner box meets the box (closed intervals); err[0] = the lowest
// triangle with a vertex index out of range.
template <typename G>
__global__ void k_meets(int nt, int nv, const int *__restrict__ s0, const int *__restrict__ s1,
                        const int *__restrict__ s2, const G *__restrict__ sx, const G *__restrict__ sy,
                        const G *__restrict__ sz, const G *__restrict__ box, int *__restrict__ flag,
                        int *__restrict__ err) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const int id[3] = {s0[t], s1[t], s2[t]};
    if (id[0] < 0 || id[0] >= nv || id[1] < 0 || id[1] >= nv || id[2] < 0 || id[2] >= nv) {
        atomicMin(err, t);
        flag[t] = 0;
        return;
    }
    const G *c[3] = {sx, sy, sz};
    bool meets = true;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const G a = c[d][id[0]], b = c[d][id[1]], e = c[d][id[2]];
        G lo = a, hi = a;
        lo = b < lo ? b : lo, hi = hi < b ? b : hi;
        lo = e < lo ? e : lo, hi = hi < e ? e : hi;
        meets = meets && !(hi < box[d] || lo > box[3 + d]);
    }
    flag[t] = meets ? 1 : 0;
}

// The corners (x0 y0 z0 x1 y1 z1 x2 y2 z2) of every flagged triangle at dst[9 (pos[t])].
template <typename G>
__global__ void k_scatter_corners(int nt, const int *__restrict__ s0, const int *__restrict__ s1,
                                  const int *__restrict__ s2, const G *__restrict__ sx, const G *__restrict__ sy,
                                  const G *__restrict__ sz, const int *__restrict__ flag, const int *__restrict__ pos,
                                  G *__restrict__ dst) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt || !flag[t]) return;
    G *o = dst + 9 * size_t(pos[t]);
    const int id[3] = {s0[t], s1[t], s2[t]};
#pragma unroll
    for (int v = 0; v < 3; v++) o[3 * v] = sx[id[v]], o[3 * v + 1] = sy[id[v]], o[3 * v + 2] = sz[id[v]];
}

template <typename G, typename T>
int grown_box_impl(long long n, const G *x, const G *y, const G *z, const T *out, G *box, cudaStream_t stream) {
    const int blocks = int(std::min<long long>(kExBlocks, std::max<long long>(1, (n + kExThreads - 1) / kExThreads)));
    G *part = nullptr;
    SSDF_CUDA(cudaMallocAsync(&part, sizeof(G) * 6 * size_t(blocks), stream));
    k_grown_partial<G, T><<<blocks, kExThreads, 0, stream>>>(n, x, y, z, out, part);
    k_grown_final<G><<<1, 32, 0, stream>>>(blocks, part, box);
    const cudaError_t e = cudaGetLastError();
    cudaFreeAsync(part, stream);
    if (e != cudaSuccess) return cuda_fail(e, "grown box", __FILE__, __LINE__);
    return SSDF_OK;
}

template <typename G>
int meeting_impl(int nt, int nv, const int *s0, const int *s1, const int *s2, const G *sx, const G *sy, const G *sz,
                 int nboxes, const G *boxes, G *corners, long long capacity, long long *counts, cudaStream_t stream) {
    int *flags = nullptr, *err = nullptr;
    SSDF_CUDA(cudaMallocAsync(&flags, sizeof(int) * (2 * size_t(nt) * nboxes + 1), stream));
    int *pos = flags + size_t(nt) * nboxes;
    err = pos + size_t(nt) * nboxes;
    std::vector<int> last(2 * size_t(nboxes));
    int herr = 0x7fffffff;
    cudaError_t e = cudaMemcpyAsync(err, &herr, sizeof(int), cudaMemcpyHostToDevice, stream);
    int st = SSDF_OK;
    for (int b = 0; b < nboxes && e == cudaSuccess && st == SSDF_OK; b++) {
        int *f = flags + size_t(nt) * b, *p = pos + size_t(nt) * b;
        k_meets<G><<<grid_blocks(nt, kExThreads), kExThreads, 0, stream>>>(nt, nv, s0, s1, s2, sx, sy, sz, boxes + 6 * b,
                                                                          f, err);
        e = cudaGetLastError();
        if (e == cudaSuccess) st = exclusive_scan_i32(f, p, nt, stream);
        if (e == cudaSuccess && st == SSDF_OK)
            e = cudaMemcpyAsync(&last[2 * b], p + nt - 1, sizeof(int), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess && st == SSDF_OK)
            e = cudaMemcpyAsync(&last[2 * b + 1], f + nt - 1, sizeof(int), cudaMemcpyDeviceToHost, stream);
    }
    if (e == cudaSuccess && st == SSDF_OK) e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && st == SSDF_OK) e = cudaStreamSynchronize(stream);
    long long total = 0;
    if (e == cudaSuccess && st == SSDF_OK) {
        if (herr != 0x7fffffff)
            st = fail(SSDF_ERR_INVALID_ARGUMENT, "triangle " + std::to_string(herr) + " has a vertex index out of range");
        for (int b = 0; b < nboxes; b++) total += (counts[b] = (long long)last[2 * b] + last[2 * b + 1]);
        if (st == SSDF_OK && corners && total > capacity)
            st = fail(SSDF_ERR_INVALID_ARGUMENT, "corner array holds " + std::to_string(capacity) + " triangles, " +
                                                     std::to_string(total) + " needed");
    }
    long long base = 0;
    for (int b = 0; b < nboxes && corners && e == cudaSuccess && st == SSDF_OK; b++) {
        k_scatter_corners<G><<<grid_blocks(nt, kExThreads), kExThreads, 0, stream>>>(
            nt, s0, s1, s2, sx, sy, sz, flags + size_t(nt) * b, pos + size_t(nt) * b, corners + 9 * size_t(base));
        e = cudaGetLastError();
        base += counts[b];
    }
    if (e == cudaSuccess && st == SSDF_OK && corners) e = cudaStreamSynchronize(stream);
    cudaFreeAsync(flags, stream);
    if (e != cudaSuccess && st == SSDF_OK) st = cuda_fail(e, "triangles meeting boxes", __FILE__, __LINE__);
    return st;
}

}  // namespace
}  // namespace ssdf_b200

using namespace ssdf_b200;

extern "C" {

int ssdf_grown_box(ptrdiff_t npoints, const void *x, const void *y, const void *z, const void *out, int coord_type,
                   int out_type, void *box6, void *stream) {
    if (npoints < 0 || !box6 || (coord_type != SSDF_F32 && coord_type != SSDF_F64) ||
        (out_type != SSDF_F32 && out_type != SSDF_F64))
        return fail(SSDF_ERR_INVALID_ARGUMENT, "ssdf_grown_box: bad arguments");
    if (npoints > 0 && (!x || !y || !z || !out)) return fail(SSDF_ERR_INVALID_ARGUMENT, "ssdf_grown_box: null array");
    const cudaStream_t s = (cudaStream_t)stream;
    if (coord_type == SSDF_F64)
        return out_type == SSDF_F64
                   ? grown_box_impl<double, double>(npoints, (const double *)x, (const double *)y, (const double *)z,
                                                    (const double *)out, (double *)box6, s)
                   : grown_box_impl<double, float>(npoints, (const double *)x, (const double *)y, (const double *)z,
                                                   (const float *)out, (double *)box6, s);
    return out_type == SSDF_F64
               ? grown_box_impl<float, double>(npoints, (const float *)x, (const float *)y, (const float *)z,
                                               (const double *)out, (float *)box6, s)
               : grown_box_impl<float, float>(npoints, (const float *)x, (const float *)y, (const float *)z,
                                              (const float *)out, (float *)box6, s);
}

int ssdf_triangles_meeting_boxes(ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                                 ptrdiff_t nspoints, const void *sx, const void *sy, const void *sz, int coord_type,
                                 int nboxes, const void *boxes, void *corners, long long capacity, long long *counts,
                                 void *stream) {
    if (nselements < 0 || nspoints < 0 || nboxes < 0 || !counts || (coord_type != SSDF_F32 && coord_type != SSDF_F64))
        return fail(SSDF_ERR_INVALID_ARGUMENT, "ssdf_triangles_meeting_boxes: bad arguments");
    for (int b = 0; b < nboxes; b++) counts[b] = 0;
    if (nselements == 0 || nboxes == 0) return SSDF_OK;
    if (!s0 || !s1 || !s2 || !sx || !sy || !sz || !boxes)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "ssdf_triangles_meeting_boxes: null array");
    if (nselements >= 0x7fffffffll / 2 / (nboxes > 0 ? nboxes : 1) || nspoints >= 0x7fffffffll)
        return fail(SSDF_ERR_NOT_SUPPORTED, "ssdf_triangles_meeting_boxes: too many triangles or boxes");
    const cudaStream_t s = (cudaStream_t)stream;
    if (coord_type == SSDF_F64)
        return meeting_impl<double>(int(nselements), int(nspoints), s0, s1, s2, (const double *)sx, (const double *)sy,
                                    (const double *)sz, nboxes, (const double *)boxes, (double *)corners, capacity,
                                    counts, s);
    return meeting_impl<float>(int(nselements), int(nspoints), s0, s1, s2, (const float *)sx, (const float *)sy,
                               (const float *)sz, nboxes, (const float *)boxes, (float *)corners, capacity, counts, s);
}

}  // extern "C"
