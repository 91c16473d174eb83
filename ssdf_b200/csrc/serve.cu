// serve.cu -- a request loop with continuous batching over resident meshes.
//
// No reference counterpart (ssdf answers one blocking call at a time). Requests name a registered
// mesh and carry a host point list or a node grid; they are answered asynchronously:
//   * admission: a mesh is built on the device when a request first needs it and stays resident
//     while the resident bytes fit the memory budget; beyond it the least recently used meshes that
//     no in-flight batch holds are evicted (and rebuilt if asked for again);
//   * admission: with a queued-query limit, a request that would bring the queries waiting to be
//     packed above it is refused at once with SSDF_ERR_BUSY (counted), so the queue, and with it the
//     latency of accepted requests, stays bounded under overload;
//   * parts: a request larger than split_queries is answered as parts -- z-slabs of a grid (keeping
//     the whole grid's node coordinates, so each value is the one a whole-grid query gives) or runs
//     of a point list; the scheduler takes one part of each waiting request in turn, so a small
//     request goes into the next batch beside a large one instead of behind it;
//   * continuous batching: a scheduler thread packs the requests that are waiting into one batch
//     (ssdf_batch_* -- one persistent launch, replayed as a CUDA graph) up to a query budget, stages
//     the point lists through pinned memory, and launches it on a free slot (4 by default), each
//     with its own stream and buffers; requests that arrive while batches run go into the next
//     one, whose upload and kernels overlap the others' (a batch whose last packets still walk
//     leaves the rest of the GPU to the next batch);
//   * completion: one thread per slot waits for that slot's event, copies results to the callers'
//     buffers, stamps latencies and wakes waiters, so no batch waits behind a slower one;
//   * tracing: with SSDF_B200_SERVE_TRACE=<file> every batch appends one line -- its slot, request and
//     query counts, and the times (ms since creation) its oldest request was submitted, packing
//     began, the launch was enqueued, the GPU finished and the results were delivered.
// Each result is computed by the same kernel as an alone query, so it is bitwise the same in any mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <list>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "internal.h"

using namespace ssdf_b200;
using Clock = std::chrono::steady_clock;

namespace {

struct HostMeshCopy {
    std::vector<int> s0, s1, s2;
    std::vector<double> sx, sy, sz;
};

struct Resident {
    ssdf_mesh *mesh = nullptr;
    size_t bytes = 0;
    int pins = 0;  // in-flight batches holding it
    std::list<int>::iterator lru;
};

struct Request {
    long long ticket = 0;
    int mesh_id = 0;
    bool grid = false;
    long long n = 0;
    const double *x = nullptr, *y = nullptr, *z = nullptr;
    long long nx = 0, ny = 0, nz = 0;
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    double *out = nullptr;
    int *outtri = nullptr;
    Clock::time_point submitted;
    int status = SSDF_OK;
    bool done = false;
    // parts: units are z-planes of a grid or points of a list
    long long units = 0;       // nz or n
    long long unit_size = 1;   // queries per unit (nx * ny for a grid)
    long long part_units = 0;  // units per part
    long long next = 0;        // first unit not yet packed
    int parts_out = 0;         // parts packed and not yet delivered
    long long queries() const { return units * unit_size; }
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t event = nullptr;
    ssdf_batch *batch = nullptr;
    double *d_pts = nullptr, *d_out = nullptr;
    int *d_tri = nullptr;
    double *h_pts = nullptr, *h_out = nullptr;
    int *h_tri = nullptr;
    std::vector<std::shared_ptr<Request>> reqs;  // one per job (a part of a request)
    std::vector<long long> offsets;              // the job's first value in the slot's buffers
    std::vector<long long> part_first, part_units;
    std::vector<int> meshes;
    bool busy = false;      // packed or in flight
    bool inflight = false;  // launched; its completer waits on the event
    // trace stamps of the batch in flight
    Clock::time_point t_pack, t_launch, t_gpu;
    long long queries = 0;
};

}  // namespace

struct ssdf_server {
    ssdf_server_opts opts;
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_slot;
    std::vector<HostMeshCopy> meshes;
    std::unordered_map<int, Resident> resident;
    std::list<int> lru;  // front = most recent
    size_t resident_bytes = 0;
    std::deque<std::shared_ptr<Request>> pending;  // requests with parts not yet packed
    long long queued_queries = 0;                  // queries of those parts
    long long rejected = 0;
    std::unordered_map<long long, std::shared_ptr<Request>> tickets;
    long long next_ticket = 1;
    std::vector<Slot> slots;
    std::thread scheduler;
    std::vector<std::thread> completers;  // one per slot
    cudaStream_t build_stream = nullptr;  // mesh builds, apart from the two batch slots
    bool stop = false;
    int device = 0;
    // stats
    std::vector<double> latencies_ms;
    long long queries_done = 0, batches = 0, evictions = 0, builds = 0;
    Clock::time_point first_submit, last_done;
    bool any_submit = false;
    // optional per-batch trace (SSDF_B200_SERVE_TRACE = file path): one line per batch
    FILE *trace = nullptr;
    Clock::time_point t0;
};

namespace {

int build_resident(ssdf_server *s, int id, Resident *r) {
    const HostMeshCopy &h = s->meshes[id];
    ssdf_build_opts bo;
    bo.leaf_size = s->opts.leaf_size;
    bo.keep_fp64 = 1;
    bo.normals = 1;
    bo.treelet_opt = kResidentTreeletRounds;
    ssdf_mesh *m = nullptr;
    SSDF_CHECK(ssdf_mesh_create(&m, ptrdiff_t(h.s0.size()), h.s0.data(), h.s1.data(), h.s2.data(),
                                ptrdiff_t(h.sx.size()), h.sx.data(), h.sy.data(), h.sz.data(), SSDF_F64, 0, &bo,
                                s->build_stream));
    int64_t bytes = 0;
    ssdf_mesh_stats(m, nullptr, nullptr, nullptr, &bytes);
    r->mesh = m;
    r->bytes = size_t(bytes);
    return SSDF_OK;
}

// Evicts least recently used meshes, other than `keep` and those an in-flight batch holds, while
// the resident bytes exceed the budget (caller holds s->mu). Runs on every admission and again
// whenever a batch releases its meshes, so a budget overrun while everything was pinned does not
// outlive the batches that caused it.
void evict_over_budget(ssdf_server *s, int keep) {
    auto li = s->lru.end();
    while (s->resident_bytes > s->opts.memory_budget && li != s->lru.begin()) {
        --li;
        const int victim = *li;
        Resident &v = s->resident[victim];
        if (victim == keep || v.pins > 0) continue;
        s->resident_bytes -= v.bytes;
        // no batch holds it, so nothing in flight reads it: a stream-ordered free on the build stream,
        // without the device-wide wait of ssdf_mesh_destroy (which would stall every slot)
        ssdf_mesh_destroy_async(v.mesh, s->build_stream);
        li = s->lru.erase(li);
        s->resident.erase(victim);
        s->evictions++;
    }
}

// Makes mesh `id` resident (caller holds s->mu); evicts unpinned LRU meshes over the budget.
int admit(ssdf_server *s, int id) {
    auto it = s->resident.find(id);
    if (it != s->resident.end()) {
        s->lru.erase(it->second.lru);
        s->lru.push_front(id);
        it->second.lru = s->lru.begin();
        return SSDF_OK;
    }
    Resident r;
    SSDF_CHECK(build_resident(s, id, &r));
    s->builds++;
    s->resident_bytes += r.bytes;
    s->lru.push_front(id);
    r.lru = s->lru.begin();
    s->resident[id] = r;
    evict_over_budget(s, id);
    return SSDF_OK;
}

void finish(ssdf_server *s, Slot &sl, int status) {
    // copy results to the callers, then stamp latencies: a request counts as served once its results
    // are in the caller's arrays (caller holds no lock)
    for (size_t k = 0; k < sl.reqs.size(); k++) {
        Request &r = *sl.reqs[k];
        const long long first = sl.part_first[k] * r.unit_size, n = sl.part_units[k] * r.unit_size;
        if (status == SSDF_OK) {
            par_memcpy(r.out + first, sl.h_out + sl.offsets[k], sizeof(double) * size_t(n));
            if (r.outtri) par_memcpy(r.outtri + first, sl.h_tri + sl.offsets[k], sizeof(int) * size_t(n));
        }
    }
    const auto now = Clock::now();
    std::lock_guard<std::mutex> lock(s->mu);
    for (auto &rp : sl.reqs) {
        if (status != SSDF_OK) rp->status = status;
        rp->parts_out--;
        if (rp->parts_out > 0 || rp->next < rp->units || rp->done) continue;
        rp->done = true;  // its last part: the request's results are all in the caller's arrays
        s->latencies_ms.push_back(std::chrono::duration<double, std::milli>(now - rp->submitted).count());
        s->queries_done += rp->queries();
    }
    for (int id : sl.meshes) {
        auto it = s->resident.find(id);
        if (it != s->resident.end()) it->second.pins--;
    }
    if (s->trace) {
        auto ms = [&](Clock::time_point t) { return std::chrono::duration<double, std::milli>(t - s->t0).count(); };
        Clock::time_point oldest = now;
        for (auto &rp : sl.reqs) oldest = std::min(oldest, rp->submitted);
        fprintf(s->trace, "slot %d reqs %zu queries %lld oldest_submit %.3f pack %.3f launched %.3f gpu_done %.3f "
                          "delivered %.3f\n",
                int(&sl - s->slots.data()), sl.reqs.size(), sl.queries, ms(oldest), ms(sl.t_pack), ms(sl.t_launch),
                ms(sl.t_gpu), ms(Clock::now()));
    }
    evict_over_budget(s, -1);
    s->last_done = now;
    sl.reqs.clear();
    sl.offsets.clear();
    sl.part_first.clear();
    sl.part_units.clear();
    sl.meshes.clear();
    sl.busy = false;
    sl.inflight = false;
    s->cv_done.notify_all();
    s->cv_slot.notify_all();
    s->cv_work.notify_all();
}

void scheduler_loop(ssdf_server *s) {
    cudaSetDevice(s->device);
    const long long cap = s->opts.max_batch_queries;
    while (true) {
        std::unique_lock<std::mutex> lock(s->mu);
        auto free_slot = [&]() -> Slot * {
            for (auto &x : s->slots)
                if (!x.busy) return &x;
            return nullptr;
        };
        s->cv_work.wait(lock, [&] { return s->stop || (!s->pending.empty() && free_slot()); });
        if (s->stop) return;
        Slot &sl = *free_slot();
        sl.t_pack = Clock::now();
        // pack waiting requests' parts up to the query and job budgets, one part of each request in
        // turn (oldest first), until nothing more fits
        long long used = 0, used_pts = 0;
        bool progress = true;
        while (progress && int(sl.reqs.size()) < s->opts.max_batch_jobs) {
            progress = false;
            for (auto it = s->pending.begin();
                 it != s->pending.end() && int(sl.reqs.size()) < s->opts.max_batch_jobs;) {
                auto r = *it;
                const long long units = std::min(r->part_units, r->units - r->next);
                const long long n = units * r->unit_size;
                if (used + n > cap) {
                    ++it;
                    continue;
                }
                const int st = admit(s, r->mesh_id);
                if (st != SSDF_OK) {  // this and its remaining parts fail; parts in flight finish
                    r->status = st;
                    s->queued_queries -= (r->units - r->next) * r->unit_size;
                    r->next = r->units;
                    if (r->parts_out == 0) r->done = true;
                    it = s->pending.erase(it);
                    s->cv_done.notify_all();
                    continue;
                }
                s->resident[r->mesh_id].pins++;
                sl.meshes.push_back(r->mesh_id);
                sl.offsets.push_back(used);
                sl.part_first.push_back(r->next);
                sl.part_units.push_back(units);
                sl.reqs.push_back(r);
                r->next += units;
                r->parts_out++;
                s->queued_queries -= n;
                used += n;
                if (!r->grid) used_pts += n;
                progress = true;
                if (r->next == r->units)
                    it = s->pending.erase(it);
                else
                    ++it;
            }
        }
        if (sl.reqs.empty()) continue;
        sl.busy = true;
        // jobs: device meshes resolved under the lock (they stay pinned)
        std::vector<ssdf_mesh *> ms;
        for (auto &r : sl.reqs) ms.push_back(s->resident[r->mesh_id].mesh);
        lock.unlock();
        // stage point lists into pinned memory, then upload
        int st = ssdf_batch_clear(sl.batch);
        ssdf_query_opts qo;
        memset(&qo, 0, sizeof(qo));
        qo.precision = s->opts.precision;
        qo.output = SSDF_OUT_SDF;
        qo.coord_type = SSDF_F64;
        qo.out_type = SSDF_F64;
        long long poff = 0;
        for (size_t k = 0; k < sl.reqs.size() && st == SSDF_OK; k++) {
            Request &r = *sl.reqs[k];
            double *out = sl.d_out + sl.offsets[k];
            int *tri = sl.d_tri + sl.offsets[k];
            const long long first = sl.part_first[k], units = sl.part_units[k];
            if (r.grid) {
                st = ssdf_batch_add_grid_slab(sl.batch, ms[k], r.nx, r.ny, r.nz, r.lo, r.hi, first, units, out, tri,
                                              &qo);
            } else {
                double *hx = sl.h_pts + 3 * poff;
                par_memcpy(hx, r.x + first, sizeof(double) * size_t(units));
                par_memcpy(hx + units, r.y + first, sizeof(double) * size_t(units));
                par_memcpy(hx + 2 * units, r.z + first, sizeof(double) * size_t(units));
                double *dx = sl.d_pts + 3 * poff;
                st = ssdf_batch_add_points(sl.batch, ms[k], units, dx, dx + units, dx + 2 * units, out, tri, &qo);
                poff += units;
            }
        }
        cudaError_t e = cudaSuccess;
        if (st == SSDF_OK && used_pts > 0)
            e = cudaMemcpyAsync(sl.d_pts, sl.h_pts, sizeof(double) * 3 * size_t(used_pts), cudaMemcpyHostToDevice,
                                sl.stream);
        if (st == SSDF_OK && e == cudaSuccess) st = ssdf_batch_run(sl.batch, 1, sl.stream);
        if (st == SSDF_OK && e == cudaSuccess)
            e = cudaMemcpyAsync(sl.h_out, sl.d_out, sizeof(double) * size_t(used), cudaMemcpyDeviceToHost, sl.stream);
        if (st == SSDF_OK && e == cudaSuccess)
            e = cudaMemcpyAsync(sl.h_tri, sl.d_tri, sizeof(int) * size_t(used), cudaMemcpyDeviceToHost, sl.stream);
        if (st == SSDF_OK && e == cudaSuccess) e = cudaEventRecord(sl.event, sl.stream);
        if (e != cudaSuccess && st == SSDF_OK) st = cuda_fail(e, "serving batch", __FILE__, __LINE__);
        sl.t_launch = Clock::now();
        sl.queries = used;
        lock.lock();
        s->batches++;
        if (st != SSDF_OK) {
            lock.unlock();
            finish(s, sl, st);
            continue;
        }
        sl.inflight = true;
        s->cv_slot.notify_all();
    }
}

// Delivers the batches of one slot: waits for its launch, then for its event.
void completer_loop(ssdf_server *s, int idx) {
    cudaSetDevice(s->device);
    Slot &sl = s->slots[idx];
    while (true) {
        {
            std::unique_lock<std::mutex> lock(s->mu);
            s->cv_slot.wait(lock, [&] { return s->stop || sl.inflight; });
            if (!sl.inflight) return;
        }
        const cudaError_t e = cudaEventSynchronize(sl.event);
        sl.t_gpu = Clock::now();
        finish(s, sl, e == cudaSuccess ? SSDF_OK : SSDF_ERR_CUDA);
    }
}

}  // namespace

extern "C" {

int ssdf_server_create(ssdf_server **out, const ssdf_server_opts *opts) {
    if (!out || !opts || opts->max_batch_queries <= 0 || opts->max_batch_jobs <= 0)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "ssdf_server_create: bad arguments");
    *out = nullptr;
    ssdf_server *s = new ssdf_server();
    s->opts = *opts;
    cudaGetDevice(&s->device);
    const size_t cap = size_t(opts->max_batch_queries);
    if (opts->slots < 0 || opts->slots > 16) {
        delete s;
        return fail(SSDF_ERR_INVALID_ARGUMENT, "ssdf_server_create: slots must be 0 (default 8) or 1..16");
    }
    if (s->opts.split_queries == 0) s->opts.split_queries = std::min(1 << 18, opts->max_batch_queries);
    if (s->opts.split_queries < 0 || s->opts.split_queries > opts->max_batch_queries || opts->max_queued_queries < 0) {
        delete s;
        return fail(SSDF_ERR_INVALID_ARGUMENT,
                    "ssdf_server_create: split_queries must be 0..max_batch_queries, max_queued_queries >= 0");
    }
    s->slots = std::vector<Slot>(opts->slots ? opts->slots : 8);
    int st = SSDF_OK;
    if (cudaStreamCreateWithFlags(&s->build_stream, cudaStreamNonBlocking) != cudaSuccess)
        st = fail(SSDF_ERR_CUDA, "ssdf_server_create: build stream");
    for (size_t k = 0; k < s->slots.size() && st == SSDF_OK; k++) {
        Slot &sl = s->slots[k];
        cudaError_t e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.event, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMalloc(&sl.d_pts, sizeof(double) * 3 * cap);
        if (e == cudaSuccess) e = cudaMalloc(&sl.d_out, sizeof(double) * cap);
        if (e == cudaSuccess) e = cudaMalloc(&sl.d_tri, sizeof(int) * cap);
        if (e == cudaSuccess) e = cudaMallocHost(&sl.h_pts, sizeof(double) * 3 * cap);
        if (e == cudaSuccess) e = cudaMallocHost(&sl.h_out, sizeof(double) * cap);
        if (e == cudaSuccess) e = cudaMallocHost(&sl.h_tri, sizeof(int) * cap);
        if (e != cudaSuccess) st = cuda_fail(e, "ssdf_server_create", __FILE__, __LINE__);
        if (st == SSDF_OK) st = ssdf_batch_create(&sl.batch, opts->max_batch_jobs, opts->precision, 0, 0);
        // overflow lists sized once: a run that grew them would wait for the other slot's batch
        if (st == SSDF_OK) st = ssdf_batch_reserve(sl.batch, (long long)cap, sl.stream);
        if (st == SSDF_OK) st = batch_capture_graphs(sl.batch);  // no capture once the threads run
    }
    if (st != SSDF_OK) {
        ssdf_server_destroy(s);
        return st;
    }
    s->t0 = Clock::now();
    if (const char *tp = env_str("SSDF_B200_SERVE_TRACE")) s->trace = fopen(tp, "w");
    s->scheduler = std::thread(scheduler_loop, s);
    for (int k = 0; k < int(s->slots.size()); k++) s->completers.emplace_back(completer_loop, s, k);
    *out = s;
    return SSDF_OK;
}

int ssdf_server_destroy(ssdf_server *s) {
    if (!s) return SSDF_OK;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    s->cv_slot.notify_all();
    if (s->scheduler.joinable()) s->scheduler.join();
    for (auto &t : s->completers)
        if (t.joinable()) t.join();
    cudaDeviceSynchronize();
    for (auto &kv : s->resident) ssdf_mesh_destroy(kv.second.mesh);
    for (auto &sl : s->slots) {
        if (sl.batch) ssdf_batch_destroy(sl.batch);
        cudaFree(sl.d_pts);
        cudaFree(sl.d_out);
        cudaFree(sl.d_tri);
        cudaFreeHost(sl.h_pts);
        cudaFreeHost(sl.h_out);
        cudaFreeHost(sl.h_tri);
        if (sl.event) cudaEventDestroy(sl.event);
        if (sl.stream) cudaStreamDestroy(sl.stream);
    }
    if (s->build_stream) cudaStreamDestroy(s->build_stream);
    if (s->trace) fclose(s->trace);
    delete s;
    return SSDF_OK;
}

int ssdf_server_add_mesh(ssdf_server *s, ptrdiff_t nselements, const int *s0, const int *s1, const int *s2,
                         ptrdiff_t nspoints, const double *sx, const double *sy, const double *sz, int *mesh_id) {
    if (!s || !mesh_id || nselements <= 0 || nspoints <= 0 || !s0 || !s1 || !s2 || !sx || !sy || !sz)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "ssdf_server_add_mesh: bad arguments");
    for (ptrdiff_t t = 0; t < nselements; t++)
        if (s0[t] < 0 || s0[t] >= nspoints || s1[t] < 0 || s1[t] >= nspoints || s2[t] < 0 || s2[t] >= nspoints)
            return fail(SSDF_ERR_INVALID_ARGUMENT, "triangle " + std::to_string(t) + " has a vertex index out of range");
    HostMeshCopy h;
    h.s0.assign(s0, s0 + nselements);
    h.s1.assign(s1, s1 + nselements);
    h.s2.assign(s2, s2 + nselements);
    h.sx.assign(sx, sx + nspoints);
    h.sy.assign(sy, sy + nspoints);
    h.sz.assign(sz, sz + nspoints);
    std::lock_guard<std::mutex> lock(s->mu);
    s->meshes.push_back(std::move(h));
    *mesh_id = int(s->meshes.size()) - 1;
    return SSDF_OK;
}

static int submit(ssdf_server *s, std::shared_ptr<Request> r, long long *ticket) {
    r->units = r->grid ? r->nz : r->n;
    r->unit_size = r->grid ? r->nx * r->ny : 1;
    const long long n = r->queries();
    if (r->units <= 0 || r->unit_size <= 0 || n >= 0x7fffffffll)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "request size must be 1 .. 2^31 - 1 queries");
    if (r->unit_size > s->opts.max_batch_queries)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "one z-plane of the grid exceeds max_batch_queries (" +
                                                   std::to_string(s->opts.max_batch_queries) + ")");
    r->part_units = std::max(1ll, (long long)s->opts.split_queries / r->unit_size);
    std::lock_guard<std::mutex> lock(s->mu);
    if (r->mesh_id < 0 || r->mesh_id >= int(s->meshes.size()))
        return fail(SSDF_ERR_INVALID_ARGUMENT, "unknown mesh id");
    if (s->opts.max_queued_queries > 0 && s->queued_queries > 0 &&
        s->queued_queries + n > s->opts.max_queued_queries) {
        s->rejected++;
        return fail(SSDF_ERR_BUSY, "server queue over its admission limit (" +
                                       std::to_string(s->opts.max_queued_queries) + " queued queries)");
    }
    s->queued_queries += n;
    r->ticket = s->next_ticket++;
    r->submitted = Clock::now();
    if (!s->any_submit) s->first_submit = r->submitted, s->any_submit = true;
    s->tickets[r->ticket] = r;
    s->pending.push_back(r);
    *ticket = r->ticket;
    s->cv_work.notify_one();
    return SSDF_OK;
}

int ssdf_server_submit_points(ssdf_server *s, int mesh_id, ptrdiff_t npoints, const double *x, const double *y,
                              const double *z, double *out, int *outtri, long long *ticket) {
    if (!s || !x || !y || !z || !out || !ticket) return fail(SSDF_ERR_INVALID_ARGUMENT, "null argument");
    auto r = std::make_shared<Request>();
    r->mesh_id = mesh_id;
    r->n = npoints;
    r->x = x, r->y = y, r->z = z;
    r->out = out;
    r->outtri = outtri;
    return submit(s, r, ticket);
}

int ssdf_server_submit_grid(ssdf_server *s, int mesh_id, ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz,
                            const double lo[3], const double hi[3], double *out, int *outtri, long long *ticket) {
    if (!s || !lo || !hi || !out || !ticket) return fail(SSDF_ERR_INVALID_ARGUMENT, "null argument");
    auto r = std::make_shared<Request>();
    r->mesh_id = mesh_id;
    r->grid = true;
    r->nx = nx, r->ny = ny, r->nz = nz;
    for (int d = 0; d < 3; d++) r->lo[d] = lo[d], r->hi[d] = hi[d];
    r->out = out;
    r->outtri = outtri;
    return submit(s, r, ticket);
}

int ssdf_server_wait(ssdf_server *s, long long ticket, double timeout_s) {
    if (!s) return fail(SSDF_ERR_INVALID_ARGUMENT, "null server");
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return fail(SSDF_ERR_INVALID_ARGUMENT, "unknown ticket");
    auto r = it->second;
    const bool ok = s->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), [&] { return r->done; });
    if (!ok) return fail(SSDF_ERR_INTERNAL, "request not finished within the timeout");
    s->tickets.erase(ticket);
    return r->status;
}

int ssdf_server_stats(ssdf_server *s, ssdf_server_report *st) {
    if (!s || !st) return fail(SSDF_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    memset(st, 0, sizeof(*st));
    std::vector<double> v = s->latencies_ms;
    st->completed = (long long)v.size();
    if (!v.empty()) {
        std::sort(v.begin(), v.end());
        auto pct = [&](double p) { return v[std::min(v.size() - 1, size_t(p * double(v.size() - 1) + 0.5))]; };
        st->p50_ms = pct(0.50);
        st->p99_ms = pct(0.99);
        st->max_ms = v.back();
    }
    st->queries = s->queries_done;
    st->batches = s->batches;
    st->evictions = s->evictions;
    st->builds = s->builds;
    st->resident_bytes = (long long)s->resident_bytes;
    st->resident_meshes = (long long)s->resident.size();
    st->rejected = s->rejected;
    if (s->any_submit)
        st->seconds = std::chrono::duration<double>(s->last_done - s->first_submit).count();
    return SSDF_OK;
}

int ssdf_server_reset_stats(ssdf_server *s) {
    if (!s) return fail(SSDF_ERR_INVALID_ARGUMENT, "null server");
    std::lock_guard<std::mutex> lock(s->mu);
    s->latencies_ms.clear();
    s->queries_done = s->batches = s->evictions = s->builds = s->rejected = 0;
    s->any_submit = false;
    return SSDF_OK;
}

}  // extern "C"
