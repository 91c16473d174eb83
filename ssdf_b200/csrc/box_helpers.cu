// box_helpers.cu -- the grid and box helpers that set up a distance query: the bounding box of a
// point set (ssdf::compute_aabb, serial/edf/edf.hpp:500-539) and every point's signed distance to a
// box (ssdf::all_points_aabb_signed_distance, serial/edf/edf.hpp:541-557, over
// point_aabb_signed_distance, serial/edf/edf.hpp:193-221). The reference's driver uses the pair to
// start `out` at |distance to the query points' own box| (drivers/sdf.exe.cpp:316-326).
//
// Both are memory-bound streams over the SoA coordinates: the box is a two-pass min/max reduction
// (per-block partials, then one block; deterministic, no float atomics), the signed distance one
// coalesced pass. Values are bitwise the reference's: min/max select, and the distance is evaluated
// term by term in T with the library-wide -fmad=false and IEEE square root.
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"

namespace ssdf_b200 {
namespace {

constexpr int kBoxThreads = 256;

template <typename T>
__device__ __forceinline__ T pos_inf();
template <>
__device__ __forceinline__ float pos_inf<float>() {
    return __int_as_float(0x7f800000);
}
template <>
__device__ __forceinline__ double pos_inf<double>() {
    return __longlong_as_double(0x7ff0000000000000ll);
}

// std::min(m, v) / std::max(m, v) as the reference's reduction applies them: a NaN v never replaces m.
template <typename T>
__device__ __forceinline__ T sel_min(T m, T v) {
    return v < m ? v : m;
}
template <typename T>
__device__ __forceinline__ T sel_max(T m, T v) {
    return m < v ? v : m;
}

// Six running extremes in the reference's output order: xmin, xmax, ymin, ymax, zmin, zmax.
template <typename T>
struct Box6 {
    T v[6];
    __device__ __forceinline__ void init() {
        v[0] = v[2] = v[4] = pos_inf<T>();
        v[1] = v[3] = v[5] = -pos_inf<T>();
    }
    __device__ __forceinline__ void add(T x, T y, T z) {
        v[0] = sel_min(v[0], x), v[1] = sel_max(v[1], x);
        v[2] = sel_min(v[2], y), v[3] = sel_max(v[3], y);
        v[4] = sel_min(v[4], z), v[5] = sel_max(v[5], z);
    }
    __device__ __forceinline__ void merge(const Box6 &o) {
        v[0] = sel_min(v[0], o.v[0]), v[1] = sel_max(v[1], o.v[1]);
        v[2] = sel_min(v[2], o.v[2]), v[3] = sel_max(v[3], o.v[3]);
        v[4] = sel_min(v[4], o.v[4]), v[5] = sel_max(v[5], o.v[5]);
    }
};

// Block-wide merge; thread 0 returns the block's box.
template <typename T>
__device__ Box6<T> block_merge(Box6<T> b) {
    __shared__ T s[6][kBoxThreads / 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        Box6<T> o;
#pragma unroll
        for (int k = 0; k < 6; k++) o.v[k] = __shfl_xor_sync(0xffffffffu, b.v[k], off);
        b.merge(o);
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < 6; k++) s[k][w] = b.v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int j = 1; j < kBoxThreads / 32; j++) {
            Box6<T> o;
#pragma unroll
            for (int k = 0; k < 6; k++) o.v[k] = s[k][j];
            b.merge(o);
        }
    }
    return b;
}

// Pass 1: per-block boxes of the points converted to T (T(x[i]), serial/edf/edf.hpp:521-523).
template <typename G, typename T>
__global__ void __launch_bounds__(kBoxThreads) k_aabb_partial(long long n, const G *__restrict__ x,
                                                              const G *__restrict__ y, const G *__restrict__ z,
                                                              T *__restrict__ partial) {
    Box6<T> b;
    b.init();
    for (long long i = blockIdx.x * (long long)kBoxThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kBoxThreads)
        b.add(T(__ldg(x + i)), T(__ldg(y + i)), T(__ldg(z + i)));
    b = block_merge(b);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < 6; k++) partial[6 * blockIdx.x + k] = b.v[k];
}

// Pass 2: one block merges the partials, seeded with the first point as the reference's reduction
// is (serial/edf/edf.hpp:512-517).
template <typename G, typename T>
__global__ void __launch_bounds__(kBoxThreads) k_aabb_final(int nparts, const G *__restrict__ x,
                                                            const G *__restrict__ y, const G *__restrict__ z,
                                                            const T *__restrict__ partial, T *__restrict__ box) {
    Box6<T> b;
    b.init();
    for (int j = threadIdx.x; j < nparts; j += kBoxThreads) {
        Box6<T> o;
#pragma unroll
        for (int k = 0; k < 6; k++) o.v[k] = partial[6 * j + k];
        b.merge(o);
    }
    b = block_merge(b);
    if (threadIdx.x == 0) {
        const T x0 = T(x[0]), y0 = T(y[0]), z0 = T(z[0]);
        Box6<T> seed;
        seed.v[0] = seed.v[1] = x0, seed.v[2] = seed.v[3] = y0, seed.v[4] = seed.v[5] = z0;
        seed.merge(b);
#pragma unroll
        for (int k = 0; k < 6; k++) box[k] = seed.v[k];
    }
}

// Signed distance to the box [minx, maxx] x [miny, maxy] x [minz, maxz], negative inside, term by
// term as serial/edf/edf.hpp:203-220 (std::max / std::min<T>(0, .) as their select forms).
template <typename T>
__device__ __forceinline__ T point_box_sdf(T px, T py, T pz, T minx, T maxx, T miny, T maxy, T minz, T maxz) {
    const T hx = (maxx - minx) * T(0.5), hy = (maxy - miny) * T(0.5), hz = (maxz - minz) * T(0.5);
    const T cx = (maxx + minx) * T(0.5), cy = (maxy + miny) * T(0.5), cz = (maxz + minz) * T(0.5);
    const T qx = fabs(px - cx) - hx, qy = fabs(py - cy) - hy, qz = fabs(pz - cz) - hz;
    const T ox = qx > T(0) ? qx : T(0), oy = qy > T(0) ? qy : T(0), oz = qz > T(0) ? qz : T(0);
    const T outside = sqrt(ox * ox + oy * oy + oz * oz);
    const T myz = qy < qz ? qz : qy;
    const T mxyz = qx < myz ? myz : qx;
    const T inside = mxyz < T(0) ? mxyz : T(0);
    return outside + inside;
}

template <typename G, typename T>
__global__ void __launch_bounds__(kBoxThreads) k_box_sdf(long long n, const G *__restrict__ x, const G *__restrict__ y,
                                                         const G *__restrict__ z, T minx, T maxx, T miny, T maxy,
                                                         T minz, T maxz, int absolute, T *__restrict__ out) {
    for (long long i = blockIdx.x * (long long)kBoxThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kBoxThreads) {
        const T d = point_box_sdf<T>(T(__ldg(x + i)), T(__ldg(y + i)), T(__ldg(z + i)), minx, maxx, miny, maxy, minz, maxz);
        out[i] = absolute ? fabs(d) : d;
    }
}

// Blocks of a streaming pass: at most eight per SM, the grid striding over the rest.
int stream_blocks(long long n) {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 1;
    }
    const long long need = (n + kBoxThreads - 1) / kBoxThreads;
    return int(std::max(1ll, std::min<long long>(need, 8ll * sms)));
}

}  // namespace

// Device arrays in, the six extremes (xmin, xmax, ymin, ymax, zmin, zmax; T) out to device `box6`.
template <typename G, typename T>
int points_aabb_device(long long n, const G *x, const G *y, const G *z, T *box6, cudaStream_t stream) {
    if (n <= 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "compute_aabb of no points");
    if (!x || !y || !z || !box6) return fail(SSDF_ERR_INVALID_ARGUMENT, "compute_aabb: null array");
    const int nb = stream_blocks(n);
    T *partial = nullptr;
    SSDF_CUDA(cudaMallocAsync(&partial, sizeof(T) * 6 * size_t(nb), stream));
    k_aabb_partial<G, T><<<nb, kBoxThreads, 0, stream>>>(n, x, y, z, partial);
    k_aabb_final<G, T><<<1, kBoxThreads, 0, stream>>>(nb, x, y, z, partial, box6);
    const cudaError_t e = cudaGetLastError();
    cudaFreeAsync(partial, stream);
    if (e != cudaSuccess) return cuda_fail(e, "compute_aabb launch", __FILE__, __LINE__);
    return SSDF_OK;
}

template <typename G, typename T>
int points_box_sdf_device(long long n, const G *x, const G *y, const G *z, const T box6[6], int absolute, T *out,
                          cudaStream_t stream) {
    if (n < 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "negative point count");
    if (n == 0) return SSDF_OK;
    if (!x || !y || !z || !out || !box6) return fail(SSDF_ERR_INVALID_ARGUMENT, "box signed distance: null array");
    k_box_sdf<G, T><<<stream_blocks(n), kBoxThreads, 0, stream>>>(n, x, y, z, box6[0], box6[1], box6[2], box6[3],
                                                                  box6[4], box6[5], absolute, out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "box signed distance launch", __FILE__, __LINE__);
    return SSDF_OK;
}

template int points_aabb_device<float, float>(long long, const float *, const float *, const float *, float *, cudaStream_t);
template int points_aabb_device<float, double>(long long, const float *, const float *, const float *, double *, cudaStream_t);
template int points_aabb_device<double, double>(long long, const double *, const double *, const double *, double *, cudaStream_t);
template int points_aabb_device<double, float>(long long, const double *, const double *, const double *, float *, cudaStream_t);
template int points_box_sdf_device<float, float>(long long, const float *, const float *, const float *, const float *,
                                                 int, float *, cudaStream_t);
template int points_box_sdf_device<float, double>(long long, const float *, const float *, const float *,
                                                  const double *, int, double *, cudaStream_t);
template int points_box_sdf_device<double, double>(long long, const double *, const double *, const double *,
                                                   const double *, int, double *, cudaStream_t);
template int points_box_sdf_device<double, float>(long long, const double *, const double *, const double *,
                                                  const float *, int, float *, cudaStream_t);

}  // namespace ssdf_b200
