// Streamed download of a grid query into host arrays.
//
// The drop-in grid entry points (ssdf::sample_sdf_bvh and the other host-array grid calls,
// serial/bvh/bvh.cpp) build the BVH, query every node and hand the values back in the caller's
// arrays. The query kernel and the device-to-host copy of its results would run one after the other;
// here the copy of each slab chunk starts as soon as the kernel has finished that chunk:
//
//   - a grid launch's blocks are slab-major (columns of 8 x 4 x grid_block_planes nodes, x fastest,
//     then y, then z), so the blocks of whole z-slabs cover one contiguous range of the output;
//   - the last block of a chunk to finish raises the chunk's flag in page-locked host memory
//     (signal_chunk in bvh_query.cu), and this thread, which would otherwise wait for the launch,
//     polls the flags and issues one cudaMemcpyAsync per finished chunk on a second stream;
//   - a page-locked output array receives that copy directly; an ordinary (pageable) one, as the
//     reference's callers pass (std::vector, numpy), receives it through one of a few page-locked
//     staging slots that this thread copies into the array once the slot's copy has landed, while
//     the launch and the next copies go on;
//   - the fix-up arithmetic finishes a few queries in its second stage, after the chunk that holds
//     them may have been copied: their final values are gathered on the device once the launch is
//     done and written into the host arrays after every chunk copy has landed.
//
// The host arrays end up with the same bits as a launch followed by one copy.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace ssdf_b200 {

namespace {

constexpr int kMaxChunks = 64;
constexpr int kTargetChunks = 16;
// Below this many nodes the copy is short next to the launch overhead it would hide.
constexpr long long kStreamMinQueries = 1ll << 22;

// Pageable outputs go through this many page-locked staging slots of one chunk each: a chunk's DMA
// lands in a free slot, and the calling thread copies the slot into the caller's array while the
// launch and the next DMAs go on.
constexpr int kStageSlots = 4;

struct ThreadResources {
    int device = -1;
    cudaStream_t copy = nullptr;  // chunk copies
    int *flags = nullptr;         // [kMaxChunks], page-locked, mapped
    int *dflags = nullptr;        // the flags' device address
    char *stage = nullptr;        // kStageSlots staging slots, page-locked (grown on demand)
    size_t stage_bytes = 0;
    cudaEvent_t landed[kStageSlots] = {};  // a slot's DMA has completed
};
thread_local ThreadResources t_res;

int thread_resources(ThreadResources **out) {
    int dev = 0;
    SSDF_CUDA(cudaGetDevice(&dev));
    ThreadResources &r = t_res;
    if (r.device != dev) {  // one set per thread; a thread that changes device gets a new set
        r = ThreadResources{};
        SSDF_CUDA(cudaStreamCreateWithFlags(&r.copy, cudaStreamNonBlocking));
        SSDF_CUDA(cudaHostAlloc((void **)&r.flags, sizeof(int) * kMaxChunks, cudaHostAllocMapped));
        SSDF_CUDA(cudaHostGetDevicePointer((void **)&r.dflags, r.flags, 0));
        for (int i = 0; i < kStageSlots; i++)
            SSDF_CUDA(cudaEventCreateWithFlags(&r.landed[i], cudaEventDisableTiming));
        r.device = dev;
    }
    *out = &r;
    return SSDF_OK;
}

// Staging slots of at least `slot` bytes each (kept for the thread's later calls).
int stage_reserve(ThreadResources *r, size_t slot) {
    const size_t need = slot * kStageSlots;
    if (r->stage_bytes >= need) return SSDF_OK;
    if (r->stage) SSDF_CUDA(cudaFreeHost(r->stage));
    r->stage = nullptr;
    r->stage_bytes = 0;
    SSDF_CUDA(cudaHostAlloc((void **)&r->stage, need, cudaHostAllocDefault));
    r->stage_bytes = need;
    return SSDF_OK;
}

bool page_locked(const void *p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();  // an unknown pointer is not an error here
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

// The final values of the second stage's queries, packed for one copy: values (as out's type), then
// triangle indices.
__global__ void k_gather_fallback(int count, const int *__restrict__ ids, const void *__restrict__ out, int out_f64,
                                  const int *__restrict__ tri, void *__restrict__ vals, int *__restrict__ tris) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int q = ids[i];
    if (out_f64)
        ((double *)vals)[i] = ((const double *)out)[q];
    else
        ((float *)vals)[i] = ((const float *)out)[q];
    if (tri) tris[i] = tri[q];
}

// Contiguous element range [lo, hi) of chunk c.
struct ChunkPlan {
    long long planes_per_chunk, plane_elems, nz;
    int nchunks, chunk_blocks;
    long long lo(int c) const { return std::min(nz, c * planes_per_chunk) * plane_elems; }
    long long hi(int c) const { return std::min(nz, (c + 1) * planes_per_chunk) * plane_elems; }
};

ChunkPlan plan_chunks(const QueryArgs &a) {
    const long long slab = grid_block_planes(a.grid_steps);  // z-planes of one row of grid blocks
    const long long bxn = grid_blocks_x(a.nx), byn = grid_blocks_y(a.ny);
    const long long slabs = grid_blocks_z(a.nz, a.grid_steps);
    const long long per = (slabs + kTargetChunks - 1) / kTargetChunks;
    ChunkPlan p;
    p.planes_per_chunk = per * slab;
    p.plane_elems = a.nx * a.ny;
    p.nz = a.nz;
    p.nchunks = int((slabs + per - 1) / per);
    p.chunk_blocks = int(per * bxn * byn);
    return p;
}

}  // namespace

// A host copy of at least 8 MB split across up to 8 threads: one thread's memcpy bandwidth would
// otherwise cap the served query rate (staging of large requests, tens of MB per batch at high load)
// and lengthen the streamed download's last copy after the query has ended.
void par_memcpy(void *dst, const void *src, size_t bytes) {
    constexpr size_t kChunk = size_t(4) << 20;
    if (bytes < 2 * kChunk) {
        memcpy(dst, src, bytes);
        return;
    }
    const size_t parts = std::min<size_t>(8, bytes / kChunk);
    const size_t step = (bytes + parts - 1) / parts;
    std::vector<std::thread> th;
    for (size_t k = 1; k < parts; k++) {
        const size_t off = k * step, len = std::min(step, bytes - off);
        th.emplace_back([=] { memcpy(static_cast<char *>(dst) + off, static_cast<const char *>(src) + off, len); });
    }
    memcpy(dst, src, std::min(step, bytes));
    for (auto &t : th) t.join();
}

bool streamed_download_applies(long long n, const void *host_out, const int *host_tri) {
    (void)host_out;
    (void)host_tri;
    return n >= kStreamMinQueries && env_int("SSDF_B200_STREAM_DOWNLOAD", 1) != 0;
}

int launch_query_streamed(const QueryArgs &args, int precision, void *host_out, int *host_tri, cudaStream_t stream) {
    QueryArgs a = args;
    if (!a.is_grid) return fail(SSDF_ERR_INVALID_ARGUMENT, "streamed download serves grids");
    const long long n = a.nx * a.ny * a.nz;
    if (n <= 0) return SSDF_OK;
    const ChunkPlan plan = plan_chunks(a);
    if (plan.nchunks > kMaxChunks || plan.chunk_blocks <= 0 || query_blocks(a) > 0x7fffffffll)
        return fail(SSDF_ERR_NOT_SUPPORTED, "grid too large for the streamed download");
    ThreadResources *r = nullptr;
    SSDF_CHECK(thread_resources(&r));
    const size_t esz = a.out_f64 ? sizeof(double) : sizeof(float);
    // A page-locked array takes its chunks' DMA directly; an ordinary (pageable) one through a staging
    // slot that this thread copies out once the slot's DMA has landed.
    const bool out_direct = page_locked(host_out);
    const bool tri_direct = !host_tri || page_locked(host_tri);
    const bool staged = !out_direct || !tri_direct;
    const size_t chunk_elems = size_t(plan.planes_per_chunk * plan.plane_elems);
    const size_t out_part = out_direct ? 0 : chunk_elems * esz;
    const size_t slot_bytes = out_part + (tri_direct ? 0 : chunk_elems * sizeof(int));
    if (staged) SSDF_CHECK(stage_reserve(r, slot_bytes));  // before the launch: growing it may block
    int *counts = nullptr;
    SSDF_CUDA(cudaMallocAsync(&counts, sizeof(int) * kMaxChunks, stream));
    struct Cleanup {
        int *counts;
        int *fb = nullptr;
        cudaStream_t s;
        cudaEvent_t done = nullptr;
        ~Cleanup() {
            if (fb) cudaFreeAsync(fb, s);
            cudaFreeAsync(counts, s);
            if (done) cudaEventDestroy(done);
        }
    } cl{counts, nullptr, stream};
    SSDF_CUDA(cudaMemsetAsync(counts, 0, sizeof(int) * kMaxChunks, stream));
    // the previous call on this thread has returned, so nothing reads the flags any more
    memset(r->flags, 0, sizeof(int) * kMaxChunks);
    a.chunk_counts = counts;
    a.chunk_flags = r->dflags;
    a.chunk_blocks = plan.chunk_blocks;
    SSDF_CUDA(cudaEventCreateWithFlags(&cl.done, cudaEventDisableTiming));
    SSDF_CHECK(launch_query_keep(a, precision, stream, &cl.fb));
    SSDF_CUDA(cudaEventRecord(cl.done, stream));

    // copy each chunk once its flag is up, or once the launch has ended (a counting or budgeted launch
    // raises no flags)
    const volatile int *flags = r->flags;
    std::vector<char> sent(size_t(plan.nchunks), 0);
    int slot_chunk[kStageSlots];
    for (int i = 0; i < kStageSlots; i++) slot_chunk[i] = -1;
    int issued = 0, delivered = 0, st = SSDF_OK;
    while (delivered < plan.nchunks && st == SSDF_OK) {
        const cudaError_t q = cudaEventQuery(cl.done);
        if (q != cudaSuccess && q != cudaErrorNotReady) {
            st = cuda_fail(q, "streamed grid query", __FILE__, __LINE__);
            break;
        }
        const bool ended = q == cudaSuccess;
        bool progress = false;
        for (int c = 0; c < plan.nchunks && issued < plan.nchunks && st == SSDF_OK; c++) {
            if (sent[c] || !(ended || flags[c])) continue;
            int slot = -1;
            if (staged) {
                for (int i = 0; i < kStageSlots && slot < 0; i++)
                    if (slot_chunk[i] < 0) slot = i;
                if (slot < 0) break;  // every slot in use: copy some out first
            }
            const long long lo = plan.lo(c), hi = plan.hi(c);
            const size_t cnt = size_t(hi - lo);
            char *stage = staged ? r->stage + size_t(slot) * slot_bytes : nullptr;
            void *to_out = out_direct ? (void *)((char *)host_out + lo * esz) : (void *)stage;
            cudaError_t e = cudaMemcpyAsync(to_out, (const char *)a.out + lo * esz, cnt * esz, cudaMemcpyDeviceToHost,
                                            r->copy);
            if (e == cudaSuccess && host_tri) {
                void *to_tri = tri_direct ? (void *)(host_tri + lo) : (void *)(stage + out_part);
                e = cudaMemcpyAsync(to_tri, a.outtri + lo, sizeof(int) * cnt, cudaMemcpyDeviceToHost, r->copy);
            }
            if (e == cudaSuccess && staged) e = cudaEventRecord(r->landed[slot], r->copy);
            if (e != cudaSuccess) st = cuda_fail(e, "chunk copy", __FILE__, __LINE__);
            sent[c] = 1;
            issued++;
            progress = true;
            if (staged)
                slot_chunk[slot] = c;
            else
                delivered++;
        }
        // staged chunks whose DMA has landed: into the caller's arrays
        for (int i = 0; i < kStageSlots && st == SSDF_OK; i++) {
            if (slot_chunk[i] < 0) continue;
            const cudaError_t e = cudaEventQuery(r->landed[i]);
            if (e == cudaErrorNotReady) continue;
            if (e != cudaSuccess) {
                st = cuda_fail(e, "chunk copy", __FILE__, __LINE__);
                break;
            }
            const int c = slot_chunk[i];
            const long long lo = plan.lo(c);
            const size_t cnt = size_t(plan.hi(c) - lo);
            const char *stage = r->stage + size_t(i) * slot_bytes;
            if (!out_direct) par_memcpy((char *)host_out + lo * esz, stage, cnt * esz);
            if (!tri_direct) par_memcpy(host_tri + lo, stage + out_part, sizeof(int) * cnt);
            slot_chunk[i] = -1;
            delivered++;
            progress = true;
        }
        if (!progress) std::this_thread::yield();
    }
    if (st == SSDF_OK) cudaGetLastError();  // a not-ready poll is no error
    // the second stage's queries: their final values, gathered once the launch is done
    int nfb = 0;
    void *vals = nullptr;
    int *tris = nullptr;
    std::vector<char> hvals;
    std::vector<int> hids, htris;
    if (st == SSDF_OK && cl.fb) {
        cudaError_t e = cudaMemcpyAsync(&nfb, cl.fb, sizeof(int), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) st = cuda_fail(e, "second-stage count", __FILE__, __LINE__);
        if (st == SSDF_OK && nfb > 0) {
            e = cudaMallocAsync(&vals, esz * size_t(nfb), stream);
            if (e == cudaSuccess && host_tri) e = cudaMallocAsync((void **)&tris, sizeof(int) * size_t(nfb), stream);
            if (e == cudaSuccess) {
                k_gather_fallback<<<unsigned((nfb + 255) / 256), 256, 0, stream>>>(nfb, cl.fb + 1, a.out, a.out_f64,
                                                                                   host_tri ? a.outtri : nullptr,
                                                                                   vals, tris);
                e = cudaGetLastError();
            }
            hvals.resize(esz * size_t(nfb));
            hids.resize(size_t(nfb));
            if (host_tri) htris.resize(size_t(nfb));
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(hids.data(), cl.fb + 1, sizeof(int) * size_t(nfb), cudaMemcpyDeviceToHost, stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(hvals.data(), vals, esz * size_t(nfb), cudaMemcpyDeviceToHost, stream);
            if (e == cudaSuccess && host_tri)
                e = cudaMemcpyAsync(htris.data(), tris, sizeof(int) * size_t(nfb), cudaMemcpyDeviceToHost, stream);
            if (vals) cudaFreeAsync(vals, stream);
            if (tris) cudaFreeAsync(tris, stream);
            if (e != cudaSuccess) st = cuda_fail(e, "second-stage gather", __FILE__, __LINE__);
        }
    }
    // every chunk copy has landed before the second stage's values overwrite theirs
    const cudaError_t ec = cudaStreamSynchronize(r->copy);
    const cudaError_t es = cudaStreamSynchronize(stream);
    if (st == SSDF_OK && ec != cudaSuccess) st = cuda_fail(ec, "chunk copies", __FILE__, __LINE__);
    if (st == SSDF_OK && es != cudaSuccess) st = cuda_fail(es, "streamed grid query", __FILE__, __LINE__);
    if (st == SSDF_OK) {
        for (int i = 0; i < nfb; i++) {
            const size_t q = size_t(hids[size_t(i)]);
            memcpy((char *)host_out + q * esz, hvals.data() + size_t(i) * esz, esz);
            if (host_tri) host_tri[q] = htris[size_t(i)];
        }
    }
    return st;
}

}  // namespace ssdf_b200
