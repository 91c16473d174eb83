// internal.h -- shared declarations of the library's host runtime and kernels.
#pragma once

#include <cmath>

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <string>

#include "../../include/ssdf_b200.h"

namespace ssdf_b200 {

// ---- error plumbing ------------------------------------------------------------------------------
void set_error(const std::string &msg);
int fail(int status, const std::string &msg);
int cuda_fail(cudaError_t err, const char *what, const char *file, int line);

#define SSDF_CUDA(call)                                                             \
    do {                                                                            \
        cudaError_t ssdf_err_ = (call);                                             \
        if (ssdf_err_ != cudaSuccess)                                               \
            return ::ssdf_b200::cuda_fail(ssdf_err_, #call, __FILE__, __LINE__);    \
    } while (0)

#define SSDF_CHECK(call)                           \
    do {                                           \
        int ssdf_st_ = (call);                     \
        if (ssdf_st_ != SSDF_OK) return ssdf_st_;  \
    } while (0)

// ---- device layouts ------------------------------------------------------------------------------
//
// BVH: binary, child-box layout. Every internal node holds both children's boxes and references,
// so one visit tests two boxes from one 64-byte (FP32) or 128-byte (FP64) record:
//   FP32 node (4 x float4): (c0.lox, c0.hix, c0.loy, c0.hiy), (c1.lox, c1.hix, c1.loy, c1.hiy),
//                           (c0.loz, c0.hiz, c1.loz, c1.hiz), (ref0, ref1, -, -) as int bits
//   FP64 node (8 x double2): c0 x, c0 y, c0 z, c1 x, c1 y, c1 z as (lo, hi), (ref0, ref1) as
//                            int bits, padding
//   4-wide FP32 node (8 x float4): lo x / hi x / lo y / hi y / lo z / hi z of children 0..3, then
//                           the 4 references as int bits, padding
//   4-wide FP64 node (14 x double2): the same six rows as pairs of double2, the 4 references as
//                            int bits in one double2, padding
// A reference >= 0 is an internal node; < 0 is a leaf ~((first << 5) | (count - 1)) over the
// triangle records in leaf order; kEmptyRef is an empty slot (its box is inverted).
// Triangles in leaf order:
//   FP32 record (3 x float4): (ax, ay, az, bx), (by, bz, cx, cy), (cz, id bits, -, -)
//   FP64 record (5 x double2): (ax, ay), (az, bx), (by, bz), (cx, cy), (cz, id)
// where id is the triangle's index in the caller's s0/s1/s2 and a, b, c its vertices s0, s1, s2.
constexpr int kEmptyRef = -2147483647 - 1;  // INT_MIN
constexpr int kLeafCountBits = 5;
constexpr int kMaxLeafSize = 16;
constexpr int kMaxTriangles = 1 << 26;
constexpr int kStackSize = 64;

__host__ __device__ inline int leaf_ref(int first, int count) { return ~((first << kLeafCountBits) | (count - 1)); }
__host__ __device__ inline int leaf_first(int ref) { return (~ref) >> kLeafCountBits; }
__host__ __device__ inline int leaf_count(int ref) { return ((~ref) & ((1 << kLeafCountBits) - 1)) + 1; }

struct DeviceMesh {
    int nt = 0;            // triangles
    int nv = 0;            // vertices
    int nnodes = 0;        // node records (>= 1)
    int depth = 0;         // max internal-node depth of the BVH (root = 1)
    int leaf_size = 4;
    int nleaves = 0;
    const float4 *nodes32 = nullptr;   // [4 * nnodes]
    const double2 *nodes64 = nullptr;  // [8 * nnodes] or null
    // 4-wide BVH over the same leaves (collapsed from the binary one)
    int nnodes4 = 0;
    int depth4 = 0;
    const float4 *nodes4_32 = nullptr;   // [8 * nnodes4]
    const double2 *nodes4_64 = nullptr;  // [14 * nnodes4] or null
    const float4 *tris32 = nullptr;    // [3 * nt], leaf order
    const double2 *tris64 = nullptr;   // [5 * nt], leaf order, or null
    // the fix-up path's FP32 filter records, [3 * nt], leaf order, with the double data or null:
    // (ax, ay, az, ab.ab), (abx, aby, abz, ac.ac), (acx, acy, acz, ab.ac) of the triangle, or of a
    // well-conditioned proxy containing an ill-conditioned one, marked by the sign bit of ab.ab
    // (mesh_build.cu, filter_record)
    const float4 *filt32 = nullptr;
    // sign data, caller's triangle order
    const int *s0 = nullptr, *s1 = nullptr, *s2 = nullptr;  // [nt]
    const double *face_n = nullptr;    // [3 * nt]
    const double *edge_n = nullptr;    // [9 * nt]
    const double *vertex_n = nullptr;  // [3 * nv]
    // scale of the coordinates (max |coordinate| over the mesh), for the fix-up window
    float coord_scale = 0.f;
    // triangles the fix-up filter sees through a proxy (ill-conditioned; 0 without the double data)
    int nill = 0;
    // the fix-up window's smallest relative width for this mesh (at least 2^-16; wider when its
    // records are large against coord_scale), and whether the float filter can serve it at all
    // (coordinates within 2^28, no record that float rounding made degenerate, needle-like or
    // too small); see set_filter_window
    float tau_rel_min = 1.0f / 65536.0f;
    int filter_ok = 0;
};

// Largest coordinate magnitude of a mesh, or of a query point, that the fix-up path's float filter
// takes: every product it forms then stays finite (|p - a| < 2^30, dot products < 2^60, their
// products < 2^120). Points beyond it are answered exactly by the second stage.
constexpr float kFilterMaxCoord = 268435456.0f;  // 2^28
// Sets DeviceMesh::tau_rel_min and ::filter_ok from the largest bound term of the mesh's filter
// records (mesh_build.cu, filter_bound) and whether every record is safe.
void set_filter_window(DeviceMesh *m, float largest_term, bool records_safe);

// Everything a query launch needs; built by the host entry points.
struct QueryArgs {
    DeviceMesh m;
    int output;        // SSDF_OUT_*
    int coord_f64;     // G == double
    int out_f64;       // T == double
    int is_grid;
    long long npoints;
    // point source
    const void *x, *y, *z;
    // grid source: nodes n, origin lo and spacing h in G precision (both views kept)
    long long nx, ny, nz;
    double lo64[3], h64[3];
    float lo32[3], h32[3];
    // outputs
    void *out;
    int *outtri;
    void *outx, *outy, *outz;
    // fix-up window: tau = tau_rel * (coord_scale + d)
    float tau_rel;
    // fix-up path, warp packets: a packet that has tested more than this many triangle records hands
    // its queries to the second stage (a warp per query) with their current windows; 0: no limit;
    // < 0: the default for the launch's size (resolve_warp_budget)
    int warp_budget;
    // overflow list of the FP32 fix-up kernel (query, final window), finished by k_window
    int *fallback_ids;
    float *fallback_thr;
    int *fallback_count;
    // optional counters [4]: triangle tests, box tests, fix-up evaluations, fallbacks
    unsigned long long *counters;
    // 0: environment / default; traversal 1 warp packets, 2 thread per query; arity 2 or 4
    int force_traversal;
    int force_arity;
    // point lists: the visiting order (query index per slot, Morton-sorted), or null (input order)
    const int *order;
    // streamed download of a grid (launch_query_streamed): the blocks of chunk c (blockIdx.x /
    // chunk_blocks, whole slabs of the grid) count themselves in chunk_counts[c] (device memory), and
    // the last one raises chunk_flags[c] (page-locked host memory); null: off
    int *chunk_counts;
    int *chunk_flags;
    int chunk_blocks;
    // grid launches: start each step of a block's column from the triangles found one step below
    int seed;
    // grid launches: z-steps of 2 kQ planes each block walks (1 .. kMaxGridSteps)
    int grid_steps;
    // grid jobs: the z-planes nz of this job are planes z0 .. z0 + nz - 1 of a larger grid with the
    // same origin and spacing (node coordinates use the global plane; outputs are the job's own)
    long long z0;
};

// Job table header of a batch (device memory).
struct BatchHeader {
    int njobs;
    int pad;
    long long total_blocks;
};

// Device pointers and launch shape of one batch launch.
struct BatchLaunch {
    const BatchHeader *hdr;
    const QueryArgs *jobs;
    const long long *first_block;
    unsigned long long *next_item;
    int grid;   // persistent blocks (SMs x resident blocks per SM)
    int sms;
    bool warp, wide;
    bool budget;  // the fix-up packets stop after the jobs' warp_budget (k_query_batch<..., BUDGET>)
};

// ---- mesh build (mesh_build.cu) ------------------------------------------------------------------
struct MeshStorage;  // owns the device allocations behind a DeviceMesh
int mesh_build(MeshStorage **storage, DeviceMesh *mesh, ptrdiff_t nt, const int *s0, const int *s1, const int *s2,
               ptrdiff_t nv, const void *sx, const void *sy, const void *sz, int coord_f64, int device_ptrs,
               const ssdf_build_opts &opts, cudaStream_t stream);
void mesh_free(MeshStorage *storage);                            // after the work using it completed
void mesh_free_async(MeshStorage *storage, cudaStream_t stream);  // in stream order
size_t mesh_bytes(const MeshStorage *storage);

// ---- radix sort (radix_sort.cu) ------------------------------------------------------------------
// Stable LSD sort of (key, value) pairs on the device, keys of `key_bits` low bits. Scratch is
// allocated on `stream` (stream-ordered).
int radix_sort_pairs_u32(uint32_t *keys, int *vals, int n, int key_bits, cudaStream_t stream);
int radix_sort_pairs_u64(uint64_t *keys, int *vals, int n, int key_bits, cudaStream_t stream);
// Exclusive prefix sum of n ints (out may alias in).
int exclusive_scan_i32(const int *in, int *out, int n, cudaStream_t stream);

// ---- queries (bvh_query.cu) ----------------------------------------------------------------------
int launch_query(const QueryArgs &args, int precision, cudaStream_t stream);
// launch_query that, on success with the fix-up arithmetic, hands back the second stage's query list
// (device ints: count, then the query indices) instead of freeing it; *fallback_list stays null for
// the other arithmetics. The caller frees it with cudaFreeAsync on `stream`.
int launch_query_keep(const QueryArgs &args, int precision, cudaStream_t stream, int **fallback_list);
// A grid query whose results go to host arrays: args.out / args.outtri are device buffers of the
// grid's size, and each slab chunk is copied to host_out / host_tri as soon as the kernel has
// finished it (through page-locked staging where an array is pageable), so the download overlaps the
// query. Returns when the host arrays hold the results (the same bits as launch_query followed by a
// copy).
int launch_query_streamed(const QueryArgs &args, int precision, void *host_out, int *host_tri, cudaStream_t stream);
// Host copy split across up to 8 threads (copies of at least 8 MB).
void par_memcpy(void *dst, const void *src, size_t bytes);
// Whether the streamed grid download applies: n queries (at least 2^22) and the switch on.
bool streamed_download_applies(long long n, const void *host_out, const int *host_tri);
int launch_query_noalloc(const QueryArgs &args, cudaStream_t stream);
long long noalloc_max_queries();
int launch_batch(const BatchLaunch &b, int precision, cudaStream_t stream);
// Whether a fix-up request on this mesh runs the FP64 kernel instead (bvh_query.cu).
bool fixup_runs_f64(const DeviceMesh &m);
int batch_capture_graphs(ssdf_batch *b);  // batch.cu
int batch_blocks_per_sm(int precision, bool warp, bool wide);
bool default_warp(int is_grid);
bool default_wide();
// Queries each lane of the query kernels answers (two independent arithmetic chains per node visit).
#ifndef SSDF_B200_QUERIES_PER_LANE
#define SSDF_B200_QUERIES_PER_LANE 1
#endif
constexpr int kQ = SSDF_B200_QUERIES_PER_LANE;
// Grid launches: a block of 128 lanes covers an 8 x 4 column of nodes and walks it upwards in
// QueryArgs::grid_steps steps (1 .. kMaxGridSteps) of 4 kQ z-planes, each step an 8 x 4 x 4kQ brick
// of nodes (each warp a 4 x 4 x 2kQ part of it). A lane starts each step from the closest triangle it
// found one step below, 4 kQ nodes away: a tight upper bound (SSDF_B200_SEED=0 starts from the
// incoming bound alone). Large grids take kDefaultGridSteps; a grid too small to fill the GPU with
// such columns takes fewer (grid_steps_for).
constexpr int kMaxGridSteps = 8;      // the most SSDF_B200_GRID_STEPS may ask for
constexpr int kDefaultGridSteps = 4;   // the most the launch rule picks
__host__ __device__ inline long long grid_blocks_x(long long nx) { return (nx + 7) / 8; }
__host__ __device__ inline long long grid_blocks_y(long long ny) { return (ny + 3) / 4; }
__host__ __device__ inline long long grid_block_planes(int steps) { return 4ll * kQ * steps; }
__host__ __device__ inline long long grid_blocks_z(long long nz, int steps) {
    return (nz + grid_block_planes(steps) - 1) / grid_block_planes(steps);
}
// Blocks of 128 lanes one job needs (grid columns as above, x fastest, then y, then z; or 128 kQ
// consecutive points).
inline long long query_blocks(const QueryArgs &a) {
    if (a.is_grid) return grid_blocks_x(a.nx) * grid_blocks_y(a.ny) * grid_blocks_z(a.nz, a.grid_steps);
    return (a.npoints + 128 * kQ - 1) / (128 * kQ);
}
// Steps per grid block for a launch whose work, at one step per block, is `one_step_blocks` blocks:
// the most steps (up to kMaxGridSteps) that still leave four waves of resident blocks on this
// device (SSDF_B200_GRID_STEPS overrides). bvh_query.cu.
int grid_steps_for(long long one_step_blocks);
// Sets QueryArgs::grid_steps of a grid job from its own size (no-op for point lists).
void set_grid_steps(QueryArgs *a);

// The counts ssdf_last_query_counts reports for this thread's last counting launch (bvh_query.cu).
void set_last_counts(unsigned long long tri, unsigned long long box, unsigned long long fix,
                     unsigned long long fallback);
// Warp-summed, one 64-bit atomic per warp: counts of a counting launch (c[0] triangle tests, c[1]
// box tests). Every lane of the warp must call it.
__device__ __forceinline__ void flush_pair_counts(unsigned long long *c, unsigned long long tri,
                                                  unsigned long long box) {
    for (int o = 16; o > 0; o >>= 1) {
        tri += __shfl_xor_sync(0xffffffffu, tri, o);
        box += __shfl_xor_sync(0xffffffffu, box, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(c, tri);
        atomicAdd(c + 1, box);
    }
}

// ---- brute force and cell list (brute_force.cu, celllist.cu) -------------------------------------
// With SSDF_B200_COUNT set, both run a counting instantiation and leave their triangle (Ericson)
// and box tests in ssdf_last_query_counts.
int brute_force_edf(int f64, ptrdiff_t npoints, const void *x, const void *y, const void *z, ptrdiff_t nt,
                    const int *s0, const int *s1, const int *s2, ptrdiff_t nv, const void *sx, const void *sy,
                    const void *sz, void *out, int *outtri, cudaStream_t stream);
int celllist_edf(int f64, ptrdiff_t npoints, const void *x, const void *y, const void *z, ptrdiff_t nt,
                 const int *s0, const int *s1, const int *s2, ptrdiff_t nv, const void *sx, const void *sy,
                 const void *sz, void *out, int *outtri, cudaStream_t stream);

// ---- box helpers (box_helpers.cu) ----------------------------------------------------------------
// Bounding box of n device points as T (xmin, xmax, ymin, ymax, zmin, zmax into device box6).
template <typename G, typename T>
int points_aabb_device(long long n, const G *x, const G *y, const G *z, T *box6, cudaStream_t stream);
// Signed distance of n device points to the box given as host box6 (|.| when absolute).
template <typename G, typename T>
int points_box_sdf_device(long long n, const G *x, const G *y, const G *z, const T box6[6], int absolute, T *out,
                          cudaStream_t stream);

// ---- level sets and field rebuilds (sdf_rebuild.cu) ----------------------------------------------
// A uniform grid: n[d] samples along axis d at o[d] + i h[d], x fastest (G's o and h, widened).
struct GridDesc {
    long long n[3];
    double o[3], h[3];
};
GridDesc grid_strided(const GridDesc &g, long long stride, bool g64);
GridDesc grid_refined(const GridDesc &g, long long factor, bool g64);
template <typename G, typename T>
int level_set_device(const GridDesc &gd, const T *d_f, T level, long long *ntri, G *x, G *y, G *z, int **d_offsets,
                     cudaStream_t stream);
template <typename G, typename T>
int rebuild_device(const GridDesc &gd, const T *d_f, T level, T band, long long stride, T *d_out, cudaStream_t stream);
template <typename G, typename T>
int refine_device(const GridDesc &gd, const T *d_f, long long factor, T *d_fine, cudaStream_t stream);
template <typename G, typename T>
int round_device(const GridDesc &gd, const T *d_f, T radius, T band, bool open, bool close, long long stride, T *d_out,
                 T *d_f0, cudaStream_t stream);

// Treelet refinement rounds of a resident mesh's BVH (built once, queried many times). Measured on the
// current kernels, queries against 1 round: beam lattice (8e6 points + 512^3 grid, float) 335.6 ->
// 313.1 / 308.7 / 304.8 ms for 2 / 3 / 4 rounds; torus knot 256^3 16.70 -> 16.63 ms (3); 64^3
// icosphere 0.470 -> 0.465 ms; the serving leg's heaviest grid 3.74 -> 3.67 ms. Each round adds about
// 1.5 ms to the torus knot's build, which calls that build per query do not repay
// (call_treelet_rounds).
constexpr int kResidentTreeletRounds = 3;

// ---- small helpers -------------------------------------------------------------------------------
inline int grid_blocks(long long n, int threads) { return int((n + threads - 1) / threads); }
// Default of QueryArgs::warp_budget, for launches (single, or a whole batch) of at most
// kBudgetMaxQueries queries; larger launches run without one. SSDF_B200_WARP_BUDGET sets it for every
// launch (0 = no limit). Measured on B200: with 2048 the 64^3 icosphere grid runs 1.83 -> 1.31 ms and a
// 110^3 grid on an 81,920-triangle sphere 22.2 -> 8.5 ms (packets near the centre, where every
// triangle is almost equidistant, hand their queries to the warp-per-query stage: the launch's tail
// shortens). A launch that fills the GPU many times over gains nothing from a shorter tail and pays
// for the repeated work (the 256-mesh batch: 257 -> 275 ms).
constexpr int kWarpBudget = 2048;
constexpr long long kBudgetMaxQueries = 1ll << 21;
// QueryArgs::warp_budget for a launch of n queries when it was left to the default (< 0): 5.6 sqrt(T)
// records for a mesh of T triangles, within [128, kWarpBudget] -- a packet that has tested that many
// is in a near-equidistant region. Measured on B200 (sphere grids, the best budget of each sweep in
// brackets): 1,280 triangles 48^3 [200]: 0.20 ms against 0.28 ms at 400; 5,120 triangles 64^3 [400]:
// 0.49 ms against 0.58 at 640 and 0.53 at 480; 20,480 triangles 96^3 [600 .. 1,280]: 1.64 ms against
// 1.89 at 2048; the serving leg's 110^3 grid on 81,920 triangles [1,536 .. 2,048]: 8.2 ms against 8.7
// at 1024 and 10.1 at 512.
constexpr int kWarpBudgetMin = 128;
inline int resolve_warp_budget(int b, long long n, int ntri) {
    if (b >= 0) return b;
    if (n > kBudgetMaxQueries) return 0;
    const int v = int(5.6 * std::sqrt(double(ntri > 0 ? ntri : 0)));
    return v < kWarpBudgetMin ? kWarpBudgetMin : (v > kWarpBudget ? kWarpBudget : v);
}
// Point lists of at least this many queries are visited in Morton order (SSDF_B200_SORT_POINTS=0
// keeps input order).
constexpr long long kSortMinPoints = 4096;
// Morton order of n (< 2^31) points over the mesh's root box: *order (n ints, stream-ordered
// allocation the caller frees with cudaFreeAsync) lists the point indices in key order (bvh_query.cu).
int morton_point_order(long long n, const void *x, const void *y, const void *z, int f64, const float4 *nodes32,
                       int **order, cudaStream_t stream);
int env_int(const char *name, int dflt);
const char *env_str(const char *name);
// Treelet refinement rounds for a mesh that one host-array call builds and queries once: none below
// 2^21 queries (SSDF_B200_TREELET overrides). The refinement is latency bound (about 1.1-1.7 ms
// whatever the mesh size) and saves 0-15 % of a query, so a smaller call loses by it. Measured on
// B200: a 5,120-triangle sphere's 64^3 grid call 3.3 -> 2.1 ms without it, 131,072-triangle
// potential_contact 4.0 -> 2.3 ms, 2e6-point closest_within_radius 12.7 -> 11.1 ms; the beam
// lattice's 8e6 points gain 5.4 ms by it.
inline int call_treelet_rounds(long long nqueries) {
    return env_int("SSDF_B200_TREELET", nqueries >= (1ll << 21) ? 1 : 0);
}
cudaStream_t library_stream();  // per-thread non-blocking stream for the blocking entry points
void retain_pool_memory();      // keep freed scratch in the device's default pool (once per device)

}  // namespace ssdf_b200

// The handle behind ssdf_mesh* (include/ssdf_b200.h).
struct ssdf_mesh {
    ssdf_b200::DeviceMesh m;
    ssdf_b200::MeshStorage *storage = nullptr;
    int device = 0;
};

namespace ssdf_b200 {
// QueryArgs of one grid / point job (validation shared by the direct and the batch entry points).
int fill_grid_args(ssdf_mesh *mesh, ptrdiff_t nx, ptrdiff_t ny, ptrdiff_t nz, const double lo[3], const double hi[3],
                   void *out, int *outtri, const ssdf_query_opts *opts, QueryArgs *a);
int fill_point_args(ssdf_mesh *mesh, ptrdiff_t npoints, const void *x, const void *y, const void *z, void *out,
                    int *outtri, void *outx, void *outy, void *outz, const ssdf_query_opts *opts, QueryArgs *a);
}  // namespace ssdf_b200

