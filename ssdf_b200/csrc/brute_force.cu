// brute_force.cu -- ssdf::edf on the GPU: every triangle against every point, exact arithmetic.
//
// The reference's edf (serial/ssdf.hpp:447-619) sorts and sweeps on three axes; its value is the
// brute-force minimum (its pruning only skips triangles that cannot improve). Here:
//   - triangle records (vertices + box, caller's order) are staged tile by tile into shared memory
//     with bulk TMA copies (cp.async.bulk + mbarrier, double-buffered, bounded waits);
//   - one thread per point walks the tile; a warp skips a triangle's Ericson test when none of
//     its points can improve on its box distance (warp-uniform branch);
//   - for few points a warp takes one point, its lanes split the triangles and the lexicographic
//     (d^2, index) minimum is reduced with warp shuffles.
// Arithmetic is T's (float or double) with the reference's expression: the result is bitwise
// sqrt(min(out^2, min_t d2_t)) in T, the reference's value; the closest triangle is the lowest
// index at the minimum.
#include <cuda_runtime.h>

#include <cfloat>

#include "device_geom.cuh"
#include "internal.h"
#include "tma.cuh"

namespace ssdf_b200 {

namespace {

constexpr int kRec = 16;  // ax ay az bx by bz cx cy cz lox hix loy hiy loz hiz -
constexpr int kBruteThreads = 256;

template <typename T>
__device__ __forceinline__ T rel_margin() {
    return T(1) + T(1) / T(65536);
}

template <typename T>
__global__ void k_brute_records(int nt, int nv, const int *__restrict__ s0, const int *__restrict__ s1,
                                const int *__restrict__ s2, const T *__restrict__ sx, const T *__restrict__ sy,
                                const T *__restrict__ sz, T *__restrict__ rec, int *__restrict__ err,
                                int *__restrict__ scale_bits) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    T *r = rec + size_t(kRec) * t;
    const int id[3] = {s0[t], s1[t], s2[t]};
    if (id[0] < 0 || id[0] >= nv || id[1] < 0 || id[1] >= nv || id[2] < 0 || id[2] >= nv) {
        atomicMin(err, t);
        for (int k = 0; k < kRec; k++) r[k] = T(0);
        return;
    }
    float amax = 0.f;
    for (int v = 0; v < 3; v++) {
        r[3 * v + 0] = sx[id[v]];
        r[3 * v + 1] = sy[id[v]];
        r[3 * v + 2] = sz[id[v]];
    }
    for (int d = 0; d < 3; d++) {
        const T lo = fmin(fmin(r[d], r[3 + d]), r[6 + d]);
        const T hi = fmax(fmax(r[d], r[3 + d]), r[6 + d]);
        r[9 + 2 * d] = lo;
        r[10 + 2 * d] = hi;
        amax = fmaxf(amax, fmaxf(fabsf(float(lo)), fabsf(float(hi))));
    }
    r[15] = T(0);
    atomicMax(scale_bits, __float_as_int(amax));
}

template <typename T>
__device__ __forceinline__ T abs_margin(float scale);
template <>
__device__ __forceinline__ double abs_margin<double>(float scale) {
    const double s = double(scale) * 0x1p-40;
    return s * s;
}
template <>
__device__ __forceinline__ float abs_margin<float>(float scale) {
    const float s = scale * 0x1p-16f;
    return s * s;
}

// One thread per point; triangle tiles of TILE records double-buffered in shared memory.
// COUNT: the counting instantiation (box and Ericson tests into counters[0..1]).
template <typename T, int TILE, bool COUNT>
__global__ void __launch_bounds__(kBruteThreads) k_brute_tile(int npoints, const T *__restrict__ x,
                                                              const T *__restrict__ y, const T *__restrict__ z,
                                                              int nt, const T *__restrict__ rec, T *__restrict__ out,
                                                              int *__restrict__ outtri,
                                                              const int *__restrict__ scale_bits,
                                                              int *__restrict__ err,
                                                              unsigned long long *__restrict__ counters) {
    unsigned long long n_tri = 0, n_box = 0;
    // The kernel has no static shared memory, so the dynamic window starts at the CTA's shared
    // base: two mbarriers in its first 16 bytes, tile buffers from byte 128 (TMA needs 16).
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw);
    T *buf = reinterpret_cast<T *>(smem_raw + 128);
    const int p = blockIdx.x * kBruteThreads + threadIdx.x;
    const bool valid = p < npoints;
    const T margin = abs_margin<T>(__int_as_float(*scale_bits));
    T px = T(0), py = T(0), pz = T(0), best = T(0);
    if (valid) {
        px = x[p], py = y[p], pz = z[p];
        const T o = out[p];
        best = o * o;
    }
    T thr = best * rel_margin<T>() + margin;
    int bid = -1;
    const int ntiles = (nt + TILE - 1) / TILE;
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    auto issue = [&](int it) {
        const int b = it & 1;
        const int cnt = min(TILE, nt - it * TILE);
        const uint32_t bytes = uint32_t(cnt) * kRec * sizeof(T);
        mbar_arrive_expect_tx(&bar[b], bytes);
        bulk_copy_g2s(buf + size_t(b) * TILE * kRec, rec + size_t(it) * TILE * kRec, bytes, &bar[b]);
    };
    if (threadIdx.x == 0) {
        issue(0);
        if (ntiles > 1) issue(1);
    }
    int it = 0;
    bool timed_out = false;
    for (; it < ntiles; it++) {
        const int b = it & 1;
        const bool ok = mbar_wait(&bar[b], uint32_t((it >> 1) & 1));
        if (__syncthreads_or(!ok)) {
            timed_out = true;
            break;
        }
        const T *tile = buf + size_t(b) * TILE * kRec;
        const int cnt = min(TILE, nt - it * TILE);
        for (int k = 0; k < cnt; k++) {
            const T *r = tile + kRec * k;
            const T db = box_dist_sq<T>(px, py, pz, r[9], r[10], r[11], r[12], r[13], r[14]);
            const bool want = valid && db < thr;
            if (COUNT) n_box += valid ? 1 : 0;
            if (!__any_sync(0xffffffffu, want)) continue;
            if (want) {
                if (COUNT) n_tri++;
                const T d2 = tri_dist_sq_exact<T>(px, py, pz, r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7], r[8]);
                if (d2 < best) {
                    best = d2;
                    bid = it * TILE + k;
                    thr = best * rel_margin<T>() + margin;
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0 && it + 2 < ntiles) issue(it + 2);
    }
    if (timed_out) {
        if (threadIdx.x == 0) {
            atomicExch(err + 1, 1);
            // let the copies this block still has in flight land before it exits (bounded)
            mbar_wait(&bar[it & 1], uint32_t((it >> 1) & 1));
            if (it + 1 < ntiles) mbar_wait(&bar[(it + 1) & 1], uint32_t(((it + 1) >> 1) & 1));
        }
        return;
    }
    if (valid) {
        out[p] = sqrt(best);
        if (outtri && bid >= 0) outtri[p] = bid;
    }
    if (COUNT) flush_pair_counts(counters, n_tri, n_box);
}

// One warp per point: lanes take triangles lane, lane + 32, ...; shuffle-reduced lexicographic min.
template <typename T, bool COUNT>
__global__ void __launch_bounds__(kBruteThreads) k_brute_warp(int npoints, const T *__restrict__ x,
                                                              const T *__restrict__ y, const T *__restrict__ z,
                                                              int nt, const T *__restrict__ rec, T *__restrict__ out,
                                                              int *__restrict__ outtri,
                                                              const int *__restrict__ scale_bits,
                                                              unsigned long long *__restrict__ counters) {
    unsigned long long n_tri = 0, n_box = 0;
    const int warp = (blockIdx.x * kBruteThreads + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= npoints) return;
    const T margin = abs_margin<T>(__int_as_float(*scale_bits));
    const T px = x[warp], py = y[warp], pz = z[warp];
    const T o = out[warp];
    T best = o * o;
    const T init = best;
    T thr = best * rel_margin<T>() + margin;
    int bid = -1;
    for (int t = lane; t < nt; t += 32) {
        const T *r = rec + size_t(kRec) * t;
        const T db = box_dist_sq<T>(px, py, pz, __ldg(r + 9), __ldg(r + 10), __ldg(r + 11), __ldg(r + 12),
                                    __ldg(r + 13), __ldg(r + 14));
        if (COUNT) n_box++;
        if (!(db < thr)) continue;
        if (COUNT) n_tri++;
        const T d2 = tri_dist_sq_exact<T>(px, py, pz, __ldg(r), __ldg(r + 1), __ldg(r + 2), __ldg(r + 3),
                                          __ldg(r + 4), __ldg(r + 5), __ldg(r + 6), __ldg(r + 7), __ldg(r + 8));
        if (d2 < best) {
            best = d2;
            bid = t;
            thr = best * rel_margin<T>() + margin;
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        const T ob = __shfl_xor_sync(0xffffffffu, best, off);
        const int oi = __shfl_xor_sync(0xffffffffu, bid, off);
        if (ob < best || (ob == best && oi >= 0 && (bid < 0 || oi < bid))) {
            best = ob;
            bid = oi;
        }
    }
    (void)init;
    if (lane == 0) {
        out[warp] = sqrt(best);
        if (outtri && bid >= 0) outtri[warp] = bid;
    }
    if (COUNT) flush_pair_counts(counters, n_tri, n_box);
}

template <typename T>
int brute_impl(ptrdiff_t npoints, const T *x, const T *y, const T *z, ptrdiff_t nt, const int *s0, const int *s1,
               const int *s2, ptrdiff_t nv, const T *sx, const T *sy, const T *sz, T *out, int *outtri,
               cudaStream_t stream) {
    constexpr int TILE = sizeof(T) == 8 ? 128 : 256;
    T *rec = nullptr;
    int *flags = nullptr;  // [0] first bad triangle, [1] timed out, [2] coordinate scale bits
    SSDF_CUDA(cudaMallocAsync(&rec, sizeof(T) * kRec * size_t(nt), stream));
    cudaError_t e = cudaMallocAsync(&flags, 4 * sizeof(int), stream);
    if (e != cudaSuccess) {
        cudaFreeAsync(rec, stream);
        return cuda_fail(e, "brute force flags", __FILE__, __LINE__);
    }
    int st = SSDF_OK;
    const int h0[4] = {0x7fffffff, 0, 0, 0};
    e = cudaMemcpyAsync(flags, h0, sizeof(h0), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess) {
        k_brute_records<T><<<grid_blocks(nt, 256), 256, 0, stream>>>(int(nt), int(nv), s0, s1, s2, sx, sy, sz, rec,
                                                                     flags, flags + 2);
        e = cudaGetLastError();
    }
    const bool count = env_int("SSDF_B200_COUNT", 0) != 0;
    unsigned long long *counters = nullptr, hc[2] = {0, 0};
    if (e == cudaSuccess && count) {
        e = cudaMallocAsync(&counters, 2 * sizeof(unsigned long long), stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(counters, 0, 2 * sizeof(unsigned long long), stream);
    }
    if (e == cudaSuccess) {
        if (npoints < 148 * 64) {
            const long long threads = (long long)npoints * 32;
            if (count)
                k_brute_warp<T, true><<<grid_blocks(threads, kBruteThreads), kBruteThreads, 0, stream>>>(
                    int(npoints), x, y, z, int(nt), rec, out, outtri, flags + 2, counters);
            else
                k_brute_warp<T, false><<<grid_blocks(threads, kBruteThreads), kBruteThreads, 0, stream>>>(
                    int(npoints), x, y, z, int(nt), rec, out, outtri, flags + 2, counters);
        } else {
            const size_t smem = 128 + 2 * size_t(TILE) * kRec * sizeof(T);
            auto kern = count ? k_brute_tile<T, TILE, true> : k_brute_tile<T, TILE, false>;
            e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
            if (e == cudaSuccess)
                kern<<<grid_blocks(npoints, kBruteThreads), kBruteThreads, smem, stream>>>(
                    int(npoints), x, y, z, int(nt), rec, out, outtri, flags + 2, flags, counters);
        }
        if (e == cudaSuccess) e = cudaGetLastError();
    }
    int h[4] = {0x7fffffff, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, flags, sizeof(h), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && counters) e = cudaMemcpyAsync(hc, counters, sizeof(hc), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (counters) {
        cudaFreeAsync(counters, stream);
        if (e == cudaSuccess) set_last_counts(hc[0], hc[1], 0, 0);
    }
    if (e != cudaSuccess) st = cuda_fail(e, "brute-force edf", __FILE__, __LINE__);
    else if (h[0] != 0x7fffffff)
        st = fail(SSDF_ERR_INVALID_ARGUMENT, "triangle " + std::to_string(h[0]) + " has a vertex index out of range");
    else if (h[1])
        st = fail(SSDF_ERR_INTERNAL, "brute-force edf: a tile copy did not complete (bounded wait gave up)");
    cudaFreeAsync(rec, stream);
    cudaFreeAsync(flags, stream);
    return st;
}

}  // namespace

int brute_force_edf(int f64, ptrdiff_t npoints, const void *x, const void *y, const void *z, ptrdiff_t nt,
                    const int *s0, const int *s1, const int *s2, ptrdiff_t nv, const void *sx, const void *sy,
                    const void *sz, void *out, int *outtri, cudaStream_t stream) {
    if (npoints <= 0 || nt <= 0 || nv <= 0) return SSDF_OK;
    if (npoints > 0x7fffffff / 32 || nt > kMaxTriangles)
        return fail(SSDF_ERR_NOT_SUPPORTED, "brute-force edf: too many points or triangles for one launch");
    if (f64)
        return brute_impl<double>(npoints, (const double *)x, (const double *)y, (const double *)z, nt, s0, s1, s2, nv,
                                  (const double *)sx, (const double *)sy, (const double *)sz, (double *)out, outtri,
                                  stream);
    return brute_impl<float>(npoints, (const float *)x, (const float *)y, (const float *)z, nt, s0, s1, s2, nv,
                             (const float *)sx, (const float *)sy, (const float *)sz, (float *)out, outtri, stream);
}

}  // namespace ssdf_b200
