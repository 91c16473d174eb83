// radix_sort.cu -- stable LSD radix sort of (key, value) pairs and an exclusive scan, on the device.
//
// One pass per 8-bit digit: a per-tile digit histogram (256 keys per tile), an exclusive scan of
// the digit-major histogram table (giving each (digit, tile) its output offset), then a stable
// scatter that ranks equal digits inside a warp with __match_any_sync and across the tile's warps
// through a shared-memory table. Used by the BVH builder (30-bit Morton keys), the pseudo-normal
// pass (vertex ids, 64-bit edge keys) and the cell list (cell ids).
#include <cuda_runtime.h>

#include "internal.h"

namespace ssdf_b200 {

namespace {

constexpr int kTile = 256;
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanBlock = kScanThreads * kScanItems;

template <typename K>
__global__ void __launch_bounds__(kTile) k_digit_hist(const K *__restrict__ keys, int n, int shift, int ntiles,
                                                      int *__restrict__ table) {
    __shared__ int hist[256];
    hist[threadIdx.x] = 0;
    __syncthreads();
    const int i = blockIdx.x * kTile + threadIdx.x;
    if (i < n) atomicAdd(&hist[int((keys[i] >> shift) & 0xff)], 1);
    __syncthreads();
    table[threadIdx.x * ntiles + blockIdx.x] = hist[threadIdx.x];
}

template <typename K>
__global__ void __launch_bounds__(kTile) k_scatter(const K *__restrict__ kin, const int *__restrict__ vin,
                                                   K *__restrict__ kout, int *__restrict__ vout, int n, int shift,
                                                   int ntiles, const int *__restrict__ offsets) {
    constexpr int kWarps = kTile / 32;
    __shared__ int cnt[kWarps][256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int w = 0; w < kWarps; w++) cnt[w][threadIdx.x] = 0;
    __syncthreads();
    const int i = blockIdx.x * kTile + threadIdx.x;
    const bool valid = i < n;
    K key = 0;
    int val = 0, d = 0;
    if (valid) {
        key = kin[i];
        val = vin[i];
        d = int((key >> shift) & 0xff);
    }
    const unsigned peers = __match_any_sync(0xffffffffu, valid ? d : 0x10000 + lane);
    const unsigned lt = (1u << lane) - 1u;
    const int rank = __popc(peers & lt);
    if (valid && (__ffs(peers) - 1) == lane) cnt[warp][d] = __popc(peers);
    __syncthreads();
    {
        int run = 0;
        for (int w = 0; w < kWarps; w++) {
            const int c = cnt[w][threadIdx.x];
            cnt[w][threadIdx.x] = run;
            run += c;
        }
    }
    __syncthreads();
    if (valid) {
        const int pos = offsets[d * ntiles + blockIdx.x] + cnt[warp][d] + rank;
        kout[pos] = key;
        vout[pos] = val;
    }
}

// Block-local exclusive scan of kScanBlock items; block totals to `sums` (if not null).
__global__ void __launch_bounds__(kScanThreads) k_scan_block(const int *__restrict__ in, int *__restrict__ out,
                                                             int n, int *__restrict__ sums) {
    __shared__ int warp_tot[kScanThreads / 32];
    const int base = blockIdx.x * kScanBlock + threadIdx.x * kScanItems;
    int v[kScanItems];
    int tsum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        v[k] = (base + k < n) ? in[base + k] : 0;
        tsum += v[k];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = tsum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int w = warp_tot[lane];
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        warp_tot[lane] = wi - w;
        if (lane == 31 && sums) sums[blockIdx.x] = wi;
    }
    __syncthreads();
    int run = warp_tot[warp] + incl - tsum;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
}

__global__ void k_add_block_offsets(int *__restrict__ out, int n, const int *__restrict__ offs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += offs[i / kScanBlock];
}

}  // namespace

// Exclusive scan of n ints (out may alias in). Scratch is stream-ordered.
int exclusive_scan_i32(const int *in, int *out, int n, cudaStream_t stream) {
    if (n <= 0) return SSDF_OK;
    const int nblocks = (n + kScanBlock - 1) / kScanBlock;
    if (nblocks == 1) {
        k_scan_block<<<1, kScanThreads, 0, stream>>>(in, out, n, nullptr);
        SSDF_CUDA(cudaGetLastError());
        return SSDF_OK;
    }
    int *sums = nullptr;
    SSDF_CUDA(cudaMallocAsync(&sums, sizeof(int) * nblocks, stream));
    k_scan_block<<<nblocks, kScanThreads, 0, stream>>>(in, out, n, sums);
    SSDF_CUDA(cudaGetLastError());
    int st = exclusive_scan_i32(sums, sums, nblocks, stream);
    if (st == SSDF_OK) {
        k_add_block_offsets<<<grid_blocks(n, 256), 256, 0, stream>>>(out, n, sums);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) st = cuda_fail(e, "k_add_block_offsets", __FILE__, __LINE__);
    }
    cudaFreeAsync(sums, stream);
    return st;
}

template <typename K>
static int radix_sort_pairs(K *keys, int *vals, int n, int key_bits, cudaStream_t stream) {
    if (n <= 1) return SSDF_OK;
    const int ntiles = (n + kTile - 1) / kTile;
    const int passes = (key_bits + 7) / 8;
    K *k2 = nullptr;
    int *v2 = nullptr, *table = nullptr;
    int st = SSDF_OK;
    if (cudaMallocAsync(&k2, sizeof(K) * size_t(n), stream) != cudaSuccess ||
        cudaMallocAsync(&v2, sizeof(int) * size_t(n), stream) != cudaSuccess ||
        cudaMallocAsync(&table, sizeof(int) * size_t(256) * ntiles, stream) != cudaSuccess) {
        st = fail(SSDF_ERR_OUT_OF_MEMORY, "radix sort scratch");
    }
    K *kin = keys, *kout = k2;
    int *vin = vals, *vout = v2;
    for (int p = 0; p < passes && st == SSDF_OK; p++) {
        const int shift = 8 * p;
        k_digit_hist<K><<<ntiles, kTile, 0, stream>>>(kin, n, shift, ntiles, table);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            st = cuda_fail(e, "k_digit_hist", __FILE__, __LINE__);
            break;
        }
        st = exclusive_scan_i32(table, table, 256 * ntiles, stream);
        if (st != SSDF_OK) break;
        k_scatter<K><<<ntiles, kTile, 0, stream>>>(kin, vin, kout, vout, n, shift, ntiles, table);
        e = cudaGetLastError();
        if (e != cudaSuccess) {
            st = cuda_fail(e, "k_scatter", __FILE__, __LINE__);
            break;
        }
        K *tk = kin;
        kin = kout;
        kout = tk;
        int *tv = vin;
        vin = vout;
        vout = tv;
    }
    if (st == SSDF_OK && kin != keys) {
        cudaError_t e = cudaMemcpyAsync(keys, kin, sizeof(K) * size_t(n), cudaMemcpyDeviceToDevice, stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(vals, vin, sizeof(int) * size_t(n), cudaMemcpyDeviceToDevice, stream);
        if (e != cudaSuccess) st = cuda_fail(e, "radix sort copy-back", __FILE__, __LINE__);
    }
    if (k2) cudaFreeAsync(k2, stream);
    if (v2) cudaFreeAsync(v2, stream);
    if (table) cudaFreeAsync(table, stream);
    return st;
}

int radix_sort_pairs_u32(uint32_t *keys, int *vals, int n, int key_bits, cudaStream_t stream) {
    return radix_sort_pairs<uint32_t>(keys, vals, n, key_bits, stream);
}
int radix_sort_pairs_u64(uint64_t *keys, int *vals, int n, int key_bits, cudaStream_t stream) {
    return radix_sort_pairs<uint64_t>(keys, vals, n, key_bits, stream);
}

}  // namespace ssdf_b200
