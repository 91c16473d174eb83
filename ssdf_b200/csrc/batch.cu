// batch.cu -- many (mesh, query set) jobs in one persistent launch, replayed as a CUDA graph.
//
// No reference counterpart: ssdf answers one mesh per call and rebuilds its BVH each time
// (serial/bvh/bvh.cu:80-158). Here resident meshes (ssdf_mesh) of very different sizes are queried
// together: the host writes a job table (one QueryArgs per job, largest first, with each job's first
// 128-query block), the persistent kernel's blocks pull (job, block) items from an atomic counter,
// and the fix-up window stage finishes every job's overflowed queries. The table lives in device
// memory and the kernels read it there, so the captured graph (two memsets + two kernels) replays
// for any batch composition; only the table is rewritten (from pinned memory) before each replay.
//
// A fix-up batch keeps a second table for the jobs whose meshes the FP64 kernel answers faster or
// alone (made mostly of slivers, or outside the float filter's preconditions: fixup_runs_f64): the
// persistent FP64 kernel runs those after the fix-up kernels, in the same graph, so every job of the
// batch gets the arithmetic it would get alone.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.h"

using namespace ssdf_b200;

struct ssdf_batch {
    int max_jobs = 0;
    int precision = SSDF_PREC_F32_FIXUP;
    int traversal = 0;  // 0 auto, 1 warp, 2 thread
    int arity = 0;      // 0 auto, 2, 4
    std::vector<QueryArgs> jobs;
    // device tables: [0] the batch's own arithmetic, [1] the FP64 jobs of a fix-up batch
    BatchHeader *d_hdr = nullptr;  // [2]
    QueryArgs *d_jobs = nullptr, *d_jobs64 = nullptr;
    long long *d_first = nullptr, *d_first64 = nullptr;
    unsigned long long *d_next = nullptr;  // [2]
    int *d_fbcount = nullptr;
    int *d_fb = nullptr;
    size_t fb_cap = 0;  // ints
    // pinned staging
    BatchHeader *h_hdr = nullptr;  // [2]
    QueryArgs *h_jobs = nullptr, *h_jobs64 = nullptr;
    long long *h_first = nullptr, *h_first64 = nullptr;
    // captured graphs, one per (warp, wide, budget, FP64 table) key: a run reuses the graph of its key
    cudaGraphExec_t exec[16] = {};
    int sms = 0;
    long long last_total = 0;
};

static void batch_free(ssdf_batch *b) {
    for (auto &g : b->exec)
        if (g) cudaGraphExecDestroy(g);
    cudaFree(b->d_hdr);
    cudaFree(b->d_jobs);
    cudaFree(b->d_jobs64);
    cudaFree(b->d_first);
    cudaFree(b->d_first64);
    cudaFree(b->d_next);
    cudaFree(b->d_fbcount);
    cudaFree(b->d_fb);
    cudaFreeHost(b->h_hdr);
    cudaFreeHost(b->h_jobs);
    cudaFreeHost(b->h_jobs64);
    cudaFreeHost(b->h_first);
    cudaFreeHost(b->h_first64);
}

// The launch sequence of one run with the given traversal and arity: counters reset, then the
// persistent kernel and the window stage, then (f64) the persistent FP64 kernel over the second
// table. It reads the job tables from device memory only.
static int enqueue_run(ssdf_batch *b, bool warp, bool wide, bool budget, bool f64, cudaStream_t s) {
    BatchLaunch L;
    L.budget = budget;
    L.hdr = b->d_hdr;
    L.jobs = b->d_jobs;
    L.first_block = b->d_first;
    L.next_item = b->d_next;
    L.sms = b->sms;
    L.warp = warp;
    L.wide = wide;
    L.grid = b->sms * batch_blocks_per_sm(b->precision, warp, wide);
    cudaError_t e = cudaMemsetAsync(b->d_next, 0, 2 * sizeof(unsigned long long), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_fbcount, 0, sizeof(int) * b->max_jobs, s);
    if (e != cudaSuccess) return cuda_fail(e, "batch reset", __FILE__, __LINE__);
    SSDF_CHECK(launch_batch(L, b->precision, s));
    if (!f64) return SSDF_OK;
    BatchLaunch D = L;
    D.budget = false;
    D.hdr = b->d_hdr + 1;
    D.jobs = b->d_jobs64;
    D.first_block = b->d_first64;
    D.next_item = b->d_next + 1;
    D.grid = b->sms * batch_blocks_per_sm(SSDF_PREC_F64, warp, wide);
    return launch_batch(D, SSDF_PREC_F64, s);
}

// The packet budget exists for the fix-up kernel's packet walks (binary and 4-wide).
static bool budget_applies(const ssdf_batch *b, bool warp, bool wide) {
    (void)wide;
    return b->precision == SSDF_PREC_F32_FIXUP && warp;
}

static int graph_key(bool warp, bool wide, bool budget, bool f64) {
    return (warp ? 1 : 0) | (wide ? 2 : 0) | (budget ? 4 : 0) | (f64 ? 8 : 0);
}

// Captures (once) the graph of a (traversal, arity, budget, FP64 table) key on a private stream,
// thread-local mode.
static int capture_key(ssdf_batch *b, bool warp, bool wide, bool budget, bool f64) {
    const int key = graph_key(warp, wide, budget, f64);
    if (b->exec[key]) return SSDF_OK;
    cudaStream_t cap;
    SSDF_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    int st = SSDF_OK;
    if (e == cudaSuccess) {
        st = enqueue_run(b, warp, wide, budget, f64, cap);
        e = cudaStreamEndCapture(cap, &g);
    }
    if (e == cudaSuccess && st == SSDF_OK) e = cudaGraphInstantiate(&b->exec[key], g, 0);
    if (g) cudaGraphDestroy(g);
    cudaStreamDestroy(cap);
    if (st != SSDF_OK) return st;
    if (e != cudaSuccess) return cuda_fail(e, "batch graph capture", __FILE__, __LINE__);
    return SSDF_OK;
}

namespace ssdf_b200 {
// Captures every graph a run of this batch can use, so that later runs capture nothing. A capture
// running in one thread while another thread synchronises the device fails; the server calls this
// before its threads start.
int batch_capture_graphs(ssdf_batch *b) {
    for (int warp = 0; warp < 2; warp++)
        for (int wide = 0; wide < 2; wide++) {
            if ((b->traversal == 1 && !warp) || (b->traversal == 2 && warp)) continue;
            if ((b->arity == 2 && wide) || (b->arity == 4 && !wide)) continue;
            for (int f64 = 0; f64 < (b->precision == SSDF_PREC_F32_FIXUP ? 2 : 1); f64++) {
                SSDF_CHECK(capture_key(b, warp != 0, wide != 0, false, f64 != 0));
                if (budget_applies(b, warp != 0, wide != 0))
                    SSDF_CHECK(capture_key(b, warp != 0, wide != 0, true, f64 != 0));
            }
        }
    return SSDF_OK;
}
}  // namespace ssdf_b200

extern "C" {

int ssdf_batch_create(ssdf_batch **out, int max_jobs, int precision, int traversal, int arity) {
    if (!out || max_jobs <= 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "ssdf_batch_create: bad arguments");
    if (precision < SSDF_PREC_F32 || precision > SSDF_PREC_F32_FIXUP)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "ssdf_batch_create: bad precision");
    *out = nullptr;
    ssdf_batch *b = new ssdf_batch();
    b->max_jobs = max_jobs;
    b->precision = precision;
    b->traversal = traversal;
    b->arity = arity;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_hdr, 2 * sizeof(BatchHeader));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_jobs, sizeof(QueryArgs) * max_jobs);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_jobs64, sizeof(QueryArgs) * max_jobs);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_first, sizeof(long long) * max_jobs);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_first64, sizeof(long long) * max_jobs);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_next, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_fbcount, sizeof(int) * max_jobs);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_hdr, 2 * sizeof(BatchHeader));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_jobs, sizeof(QueryArgs) * max_jobs);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_jobs64, sizeof(QueryArgs) * max_jobs);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_first, sizeof(long long) * max_jobs);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_first64, sizeof(long long) * max_jobs);
    if (e == cudaSuccess) memset(b->h_hdr, 0, 2 * sizeof(BatchHeader));
    if (e != cudaSuccess) {
        batch_free(b);
        delete b;
        return cuda_fail(e, "ssdf_batch_create", __FILE__, __LINE__);
    }
    *out = b;
    return SSDF_OK;
}

int ssdf_batch_destroy(ssdf_batch *b) {
    if (!b) return SSDF_OK;
    cudaDeviceSynchronize();
    batch_free(b);
    delete b;
    return SSDF_OK;
}

int ssdf_batch_clear(ssdf_batch *b) {
    if (!b) return fail(SSDF_ERR_INVALID_ARGUMENT, "null batch");
    b->jobs.clear();
    return SSDF_OK;
}

int ssdf_batch_size(const ssdf_batch *b) { return b ? int(b->jobs.size()) : 0; }

static int batch_add(ssdf_batch *b, const QueryArgs &a, const ssdf_query_opts *opts) {
    if (opts->precision != b->precision)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "a batch runs one arithmetic: job precision differs from the batch's");
    if (int(b->jobs.size()) >= b->max_jobs) return fail(SSDF_ERR_INVALID_ARGUMENT, "batch is full");
    if (b->precision == SSDF_PREC_F64 && !a.m.nodes64)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "mesh built without double data (keep_fp64=0)");
    if (b->precision == SSDF_PREC_F32_FIXUP && (!a.m.tris64 || !a.m.nodes64 || !a.m.filt32))
        return fail(SSDF_ERR_INVALID_ARGUMENT, "fix-up queries need the double triangles and BVH (keep_fp64=1)");
    if (a.output == SSDF_OUT_SDF && (!a.m.face_n || !a.m.tris64))
        return fail(SSDF_ERR_INVALID_ARGUMENT, "signed queries need a mesh built with normals=1 and keep_fp64=1");
    if (b->precision == SSDF_PREC_F32 && (a.output == SSDF_OUT_SDF || a.output == SSDF_OUT_CLOSEST))
        return fail(SSDF_ERR_INVALID_ARGUMENT, "SSDF_PREC_F32 serves the edf and sqedf outputs");
    const long long n = a.is_grid ? a.nx * a.ny * a.nz : a.npoints;
    if (n >= 0x7fffffffll) return fail(SSDF_ERR_NOT_SUPPORTED, "more than 2^31 - 1 queries in one job");
    if (n > 0) b->jobs.push_back(a);
    return SSDF_OK;
}

int ssdf_batch_add_grid(ssdf_batch *b, ssdf_mesh *mesh, ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz, const double lo[3],
                        const double hi[3], void *out, int *outtri, const ssdf_query_opts *opts) {
    if (!b || !opts) return fail(SSDF_ERR_INVALID_ARGUMENT, "null batch or options");
    QueryArgs a;
    SSDF_CHECK(fill_grid_args(mesh, nx, ny, nz, lo, hi, out, outtri, opts, &a));
    return batch_add(b, a, opts);
}

int ssdf_batch_add_grid_slab(ssdf_batch *b, ssdf_mesh *mesh, ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz,
                             const double lo[3], const double hi[3], ptrdiff_t z0, ptrdiff_t nz_slab, void *out,
                             int *outtri, const ssdf_query_opts *opts) {
    if (!b || !opts) return fail(SSDF_ERR_INVALID_ARGUMENT, "null batch or options");
    if (z0 < 0 || nz_slab < 0 || z0 + nz_slab > nz)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "ssdf_batch_add_grid_slab: planes outside the grid");
    QueryArgs a;
    SSDF_CHECK(fill_grid_args(mesh, nx, ny, nz, lo, hi, out, outtri, opts, &a));
    a.nz = nz_slab;  // the grid's origin and spacing stay those of the whole grid
    a.z0 = z0;
    set_grid_steps(&a);
    return batch_add(b, a, opts);
}

int ssdf_batch_add_points(ssdf_batch *b, ssdf_mesh *mesh, ptrdiff_t npoints, const void *x, const void *y,
                          const void *z, void *out, int *outtri, const ssdf_query_opts *opts) {
    if (!b || !opts) return fail(SSDF_ERR_INVALID_ARGUMENT, "null batch or options");
    QueryArgs a;
    SSDF_CHECK(fill_point_args(mesh, npoints, x, y, z, out, outtri, nullptr, nullptr, nullptr, opts, &a));
    return batch_add(b, a, opts);
}

// Sizes the fix-up overflow lists for runs of up to max_queries queries, so that such runs never
// reallocate them (a reallocation synchronises the device).
int ssdf_batch_reserve(ssdf_batch *b, long long max_queries, void *stream_) {
    if (!b || max_queries < 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "ssdf_batch_reserve: bad arguments");
    const size_t need = b->precision == SSDF_PREC_F32_FIXUP ? 2 * size_t(max_queries) : 0;
    if (need <= b->fb_cap) return SSDF_OK;
    SSDF_CUDA(cudaStreamSynchronize((cudaStream_t)stream_));
    cudaFree(b->d_fb);
    b->d_fb = nullptr;
    b->fb_cap = 0;
    SSDF_CUDA(cudaMalloc(&b->d_fb, sizeof(int) * need));
    b->fb_cap = need;
    return SSDF_OK;
}

// One persistent launch over every job (+ the fix-up window stage). use_graph: capture the launch
// sequence once (per traversal mode and arity) and replay it afterwards.
int ssdf_batch_run(ssdf_batch *b, int use_graph, void *stream_) {
    if (!b) return fail(SSDF_ERR_INVALID_ARGUMENT, "null batch");
    cudaStream_t stream = (cudaStream_t)stream_;
    const int njobs = int(b->jobs.size());
    if (njobs == 0) return SSDF_OK;
    // point jobs of kSortMinPoints or more are visited in Morton order (computed before the launch,
    // outside any graph; freed in stream order behind it), which lets them walk as warp packets
    const bool sort_points = b->traversal != 2 && env_int("SSDF_B200_SORT_POINTS", 1) != 0;
    bool any_grid = false, any_sorted = false;
    for (const auto &j : b->jobs) {
        any_grid |= j.is_grid != 0;
        any_sorted |= sort_points && !j.is_grid && j.npoints >= kSortMinPoints;
    }
    const bool warp = b->traversal == 1 ? true : b->traversal == 2 ? false : default_warp(any_grid || any_sorted);
    const bool wide = b->arity == 4 ? true : b->arity == 2 ? false : default_wide();
    // the FP64 table of a fix-up batch: jobs whose meshes the FP64 kernel answers (fixup_runs_f64)
    const bool fixup = b->precision == SSDF_PREC_F32_FIXUP;
    auto to_f64 = [&](const QueryArgs &a) { return fixup && fixup_runs_f64(a.m); };
    // largest jobs first: the tail of each launch is then made of small items
    std::vector<int> order(njobs);
    for (int i = 0; i < njobs; i++) order[i] = i;
    auto cost = [&](const QueryArgs &a) { return double(query_blocks(a)) * std::log2(2.0 + a.m.nt); };
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost(b->jobs[x]) > cost(b->jobs[y]); });
    // fix-up overflow lists: one slice of (ids, thresholds) per job of the first table
    size_t need = 0;
    if (fixup)
        for (const auto &j : b->jobs)
            if (!to_f64(j)) need += 2 * size_t(j.is_grid ? j.nx * j.ny * j.nz : j.npoints);
    if (need > b->fb_cap) SSDF_CHECK(ssdf_batch_reserve(b, (long long)(need / 2), stream));
    // the staging buffers may still feed the previous run's copies
    SSDF_CUDA(cudaStreamSynchronize(stream));
    struct Orders {  // the runs' visiting orders, freed in stream order when the call returns
        std::vector<int *> p;
        cudaStream_t s;
        ~Orders() {
            for (int *q : p) cudaFreeAsync(q, s);
        }
    } orders{{}, stream};
    long long total = 0, total64 = 0, nq = 0, one_step = 0;
    for (auto &j : b->jobs) {
        nq += j.is_grid ? j.nx * j.ny * j.nz : j.npoints;
        if (j.is_grid) j.grid_steps = 1;
        one_step += query_blocks(j);
    }
    // the batch fills the GPU as a whole: its grid jobs walk columns of as many steps as its total
    // work leaves four waves of blocks for
    const int steps = grid_steps_for(one_step);
    size_t off = 0;
    int k = 0, k64 = 0;
    for (int r = 0; r < njobs; r++) {
        QueryArgs a = b->jobs[order[r]];
        a.warp_budget = resolve_warp_budget(a.warp_budget, nq, a.m.nt);
        if (a.is_grid) a.grid_steps = steps;
        if (sort_points && !a.is_grid && a.npoints >= kSortMinPoints) {
            int *ord = nullptr;
            SSDF_CHECK(morton_point_order(a.npoints, a.x, a.y, a.z, a.coord_f64, a.m.nodes32, &ord, stream));
            orders.p.push_back(ord);
            a.order = ord;
        }
        a.counters = nullptr;
        if (to_f64(a)) {
            a.fallback_count = nullptr;
            a.fallback_ids = nullptr;
            a.fallback_thr = nullptr;
            a.warp_budget = 0;
            b->h_jobs64[k64] = a;
            b->h_first64[k64++] = total64;
            total64 += query_blocks(a);
            continue;
        }
        if (fixup) {
            const size_t n = size_t(a.is_grid ? a.nx * a.ny * a.nz : a.npoints);
            a.fallback_count = b->d_fbcount + k;
            a.fallback_ids = b->d_fb + off;
            a.fallback_thr = reinterpret_cast<float *>(b->d_fb + off + n);
            off += 2 * n;
        } else {
            a.fallback_count = nullptr;
            a.fallback_ids = nullptr;
            a.fallback_thr = nullptr;
        }
        b->h_jobs[k] = a;
        b->h_first[k++] = total;
        total += query_blocks(a);
    }
    b->h_hdr[0] = BatchHeader{k, 0, total};
    b->h_hdr[1] = BatchHeader{k64, 0, total64};
    b->last_total = total + total64;
    SSDF_CUDA(cudaMemcpyAsync(b->d_hdr, b->h_hdr, 2 * sizeof(BatchHeader), cudaMemcpyHostToDevice, stream));
    if (k > 0) {
        SSDF_CUDA(cudaMemcpyAsync(b->d_jobs, b->h_jobs, sizeof(QueryArgs) * k, cudaMemcpyHostToDevice, stream));
        SSDF_CUDA(cudaMemcpyAsync(b->d_first, b->h_first, sizeof(long long) * k, cudaMemcpyHostToDevice, stream));
    }
    if (k64 > 0) {
        SSDF_CUDA(cudaMemcpyAsync(b->d_jobs64, b->h_jobs64, sizeof(QueryArgs) * k64, cudaMemcpyHostToDevice, stream));
        SSDF_CUDA(
            cudaMemcpyAsync(b->d_first64, b->h_first64, sizeof(long long) * k64, cudaMemcpyHostToDevice, stream));
    }
    bool budget = false;
    for (int j = 0; j < k; j++) budget |= b->h_jobs[j].warp_budget > 0;
    budget = budget && budget_applies(b, warp, wide);
    const bool f64 = k64 > 0;
    if (!use_graph) return enqueue_run(b, warp, wide, budget, f64, stream);
    SSDF_CHECK(capture_key(b, warp, wide, budget, f64));
    SSDF_CUDA(cudaGraphLaunch(b->exec[graph_key(warp, wide, budget, f64)], stream));
    return SSDF_OK;
}

// Work items (128-query blocks) of the last run.
long long ssdf_batch_last_blocks(const ssdf_batch *b) { return b ? b->last_total : 0; }

}  // extern "C"
