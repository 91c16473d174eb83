// mesh_build.cu -- device-resident mesh: triangle records, LBVH, refit, pseudo-normals.
//
// Replaces the reference's per-call host packing + cuBQL build (serial/bvh/bvh.cu:108-130,
// serial/bvh/bvh.cpp:155-165) with a device pipeline that runs once per mesh:
//   1. validate indices, gather vertices, triangle boxes (FP32 and FP64), scene box of centroids;
//   2. 30-bit Morton codes of the centroids, stable radix sort (radix_sort.cu);
//   3. Karras LBVH topology over the sorted primitives (index tie-break for equal codes);
//   4. bottom-up refit with per-node arrival counters;
//   5. optional SAH treelet refinement (treelet_opt.cu);
//   6. node records in the child-box layout, subtrees of <= leaf_size triangles collapsed into
//      leaves, triangle records in leaf order (internal.h documents both layouts);
//   7. optional angle-weighted pseudo-normals (serial/bvh/bvh.cpp:1669-1721), summed in the
//      reference's order so they are bitwise its values up to the last bit of acos.
#include <cuda_runtime.h>

#include <cfloat>
#include <vector>

#include "internal.h"

namespace ssdf_b200 {

// SAH treelet refinement (treelet_opt.cu): restructures the topology in place, refits the boxes and
// re-derives the leaf order (ids, leaf references, first_of) so subtrees stay contiguous ranges.
int treelet_optimize(int n, int *child_l, int *child_r, int *parent_int, int *parent_leaf, int *first_of,
                     float *nbox32, double *nbox64, const float *pbox32, const double *pbox64, int *sorted_ids,
                     cudaStream_t stream);

struct MeshStorage {
    std::vector<void *> blocks;
    size_t bytes = 0;
};

namespace {

template <typename T>
int dalloc(MeshStorage *s, T **p, size_t count, cudaStream_t stream) {
    void *ptr = nullptr;
    const size_t b = sizeof(T) * (count ? count : 1);
    cudaError_t e = cudaMallocAsync(&ptr, b, stream);
    if (e != cudaSuccess) return fail(SSDF_ERR_OUT_OF_MEMORY, "device allocation of " + std::to_string(b) + " bytes");
    s->blocks.push_back(ptr);
    s->bytes += b;
    *p = reinterpret_cast<T *>(ptr);
    return SSDF_OK;
}

// Monotone float <-> int for atomicMin/atomicMax on floats.
__device__ __forceinline__ int f2o(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float o2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

__global__ void k_validate(int nt, int nv, const int *__restrict__ s0, const int *__restrict__ s1,
                           const int *__restrict__ s2, int *__restrict__ bad) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const int a = s0[t], b = s1[t], c = s2[t];
    if (a < 0 || a >= nv || b < 0 || b >= nv || c < 0 || c >= nv) atomicMin(bad, t);
}

template <typename G>
__global__ void k_widen(int nv, const G *__restrict__ sx, const G *__restrict__ sy, const G *__restrict__ sz,
                        double *__restrict__ vx, double *__restrict__ vy, double *__restrict__ vz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    vx[i] = double(sx[i]);
    vy[i] = double(sy[i]);
    vz[i] = double(sz[i]);
}

// Per triangle: FP32 / FP64 boxes, FP32 centroid; scene centroid bounds and coordinate scale.
__global__ void k_prep(int nt, const int *__restrict__ s0, const int *__restrict__ s1, const int *__restrict__ s2,
                       const double *__restrict__ vx, const double *__restrict__ vy, const double *__restrict__ vz,
                       float *__restrict__ box32, double *__restrict__ box64, float *__restrict__ cen,
                       int *__restrict__ scene /* 6 ordered ints: lo xyz, hi xyz */, int *__restrict__ scale) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    float c[3] = {0.f, 0.f, 0.f};
    float amax = 0.f;
    const bool ok = t < nt;
    if (ok) {
        const int id[3] = {s0[t], s1[t], s2[t]};
        double p[3][3];
        for (int v = 0; v < 3; v++) p[v][0] = vx[id[v]], p[v][1] = vy[id[v]], p[v][2] = vz[id[v]];
        for (int d = 0; d < 3; d++) {
            const double lo = fmin(fmin(p[0][d], p[1][d]), p[2][d]);
            const double hi = fmax(fmax(p[0][d], p[1][d]), p[2][d]);
            box64[6 * t + 2 * d] = lo;
            box64[6 * t + 2 * d + 1] = hi;
            const float f0 = float(p[0][d]), f1 = float(p[1][d]), f2 = float(p[2][d]);
            const float flo = fminf(fminf(f0, f1), f2), fhi = fmaxf(fmaxf(f0, f1), f2);
            box32[6 * t + 2 * d] = flo;
            box32[6 * t + 2 * d + 1] = fhi;
            c[d] = 0.5f * (flo + fhi);
            cen[3 * t + d] = c[d];
            amax = fmaxf(amax, fmaxf(fabsf(flo), fabsf(fhi)));
        }
    }
    // warp-level reduction then one atomic per warp
    float lo[3], hi[3];
    for (int d = 0; d < 3; d++) lo[d] = ok ? c[d] : FLT_MAX, hi[d] = ok ? c[d] : -FLT_MAX;
    for (int o = 16; o > 0; o >>= 1) {
        for (int d = 0; d < 3; d++) {
            lo[d] = fminf(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
            hi[d] = fmaxf(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
        }
        amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    }
    if ((threadIdx.x & 31) == 0) {
        for (int d = 0; d < 3; d++) {
            atomicMin(&scene[d], f2o(lo[d]));
            atomicMax(&scene[3 + d], f2o(hi[d]));
        }
        atomicMax(scale, __float_as_int(amax));
    }
}

__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

__global__ void k_morton(int nt, const float *__restrict__ cen, const int *__restrict__ scene,
                         uint32_t *__restrict__ keys, int *__restrict__ vals) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    uint32_t q[3];
    for (int d = 0; d < 3; d++) {
        const float lo = o2f(scene[d]), hi = o2f(scene[3 + d]);
        const float ext = hi - lo;
        float u = ext > 0.f ? (cen[3 * t + d] - lo) / ext : 0.5f;
        u = fminf(fmaxf(u, 0.f), 1.f);
        q[d] = uint32_t(fminf(u * 1024.f, 1023.f));
    }
    keys[t] = (expand_bits(q[0]) << 2) | (expand_bits(q[1]) << 1) | expand_bits(q[2]);
    vals[t] = t;
}

__device__ __forceinline__ int karras_delta(const uint32_t *__restrict__ k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const uint32_t a = k[i], b = k[j];
    if (a == b) return 32 + __clz(i ^ j);
    return __clz(a ^ b);
}

// Internal node i of the n-1: children (>= 0 internal, < 0 leaf -(pos + 1)), range, parents.
__global__ void k_karras(int n, const uint32_t *__restrict__ k, int *__restrict__ child_l, int *__restrict__ child_r,
                         int *__restrict__ first_of, int *__restrict__ last_of, int *__restrict__ parent_int,
                         int *__restrict__ parent_leaf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int d = (karras_delta(k, n, i, i + 1) - karras_delta(k, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = karras_delta(k, n, i, i - d);
    int lmax = 2;
    while (karras_delta(k, n, i, i + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (karras_delta(k, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = karras_delta(k, n, i, j);
    int s = 0, t = l;
    do {
        t = (t + 1) >> 1;
        if (karras_delta(k, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int gamma = i + s * d + min(d, 0);
    const int first = min(i, j), last = max(i, j);
    const int left = (first == gamma) ? -(gamma + 1) : gamma;
    const int right = (last == gamma + 1) ? -(gamma + 2) : gamma + 1;
    child_l[i] = left;
    child_r[i] = right;
    first_of[i] = first;
    last_of[i] = last;
    if (left < 0) parent_leaf[gamma] = i; else parent_int[gamma] = i;
    if (right < 0) parent_leaf[gamma + 1] = i; else parent_int[gamma + 1] = i;
    if (i == 0) parent_int[0] = -1;
}

// Bottom-up refit: the second thread to reach a node unions its two children's boxes.
__global__ void k_refit(int n, const int *__restrict__ sorted_ids, const int *__restrict__ child_l,
                        const int *__restrict__ child_r, const int *__restrict__ parent_int,
                        const int *__restrict__ parent_leaf, const float *__restrict__ pbox32,
                        const double *__restrict__ pbox64, float *nbox32, double *nbox64, int *arrivals) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int node = parent_leaf[p];
    while (node >= 0) {
        __threadfence();
        if (atomicAdd(&arrivals[node], 1) == 0) return;
        __threadfence();
        const int c[2] = {child_l[node], child_r[node]};
        float b32[6];
        double b64[6];
        for (int k = 0; k < 6; k++) b32[k] = (k & 1) ? -FLT_MAX : FLT_MAX, b64[k] = (k & 1) ? -DBL_MAX : DBL_MAX;
        for (int h = 0; h < 2; h++) {
            const float *s32;
            const double *s64;
            if (c[h] < 0) {
                const int prim = sorted_ids[-c[h] - 1];
                s32 = pbox32 + 6 * prim;
                s64 = pbox64 + 6 * prim;
            } else {
                s32 = nbox32 + 6 * c[h];
                s64 = nbox64 + 6 * c[h];
            }
            for (int k = 0; k < 6; k += 2) {
                b32[k] = fminf(b32[k], __ldcg(s32 + k));
                b32[k + 1] = fmaxf(b32[k + 1], __ldcg(s32 + k + 1));
                b64[k] = fmin(b64[k], __ldcg(s64 + k));
                b64[k + 1] = fmax(b64[k + 1], __ldcg(s64 + k + 1));
            }
        }
        for (int k = 0; k < 6; k++) {
            __stcg(nbox32 + 6 * node + k, b32[k]);
            __stcg(nbox64 + 6 * node + k, b64[k]);
        }
        node = parent_int[node];
    }
}

// Subtree sizes after treelet restructuring: recomputed bottom-up the same way.
__global__ void k_counts(int n, const int *__restrict__ child_l, const int *__restrict__ child_r,
                         const int *__restrict__ parent_int, const int *__restrict__ parent_leaf, int *count,
                         int *arrivals) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int node = parent_leaf[p];
    while (node >= 0) {
        __threadfence();
        if (atomicAdd(&arrivals[node], 1) == 0) return;
        __threadfence();
        const int l = child_l[node], r = child_r[node];
        const int cl = l < 0 ? 1 : __ldcg(count + l);
        const int cr = r < 0 ? 1 : __ldcg(count + r);
        __stcg(count + node, cl + cr);
        node = parent_int[node];
    }
}

// Node records. A child with <= L triangles in its subtree becomes a leaf over its range.
__global__ void k_write_nodes(int n, int L, const int *__restrict__ child_l, const int *__restrict__ child_r,
                              const int *__restrict__ first_of, const int *__restrict__ count,
                              const int *__restrict__ sorted_ids, const float *__restrict__ pbox32,
                              const double *__restrict__ pbox64, const float *__restrict__ nbox32,
                              const double *__restrict__ nbox64, float4 *__restrict__ nodes32,
                              double2 *__restrict__ nodes64) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int ref[2];
    const float *b32[2];
    const double *b64[2];
    const int c[2] = {child_l[i], child_r[i]};
    for (int h = 0; h < 2; h++) {
        if (c[h] < 0) {
            const int pos = -c[h] - 1;
            ref[h] = leaf_ref(pos, 1);
            b32[h] = pbox32 + 6 * sorted_ids[pos];
            b64[h] = pbox64 + 6 * sorted_ids[pos];
        } else {
            ref[h] = count[c[h]] <= L ? leaf_ref(first_of[c[h]], count[c[h]]) : c[h];
            b32[h] = nbox32 + 6 * c[h];
            b64[h] = nbox64 + 6 * c[h];
        }
    }
    nodes32[4 * i + 0] = make_float4(b32[0][0], b32[0][1], b32[0][2], b32[0][3]);
    nodes32[4 * i + 1] = make_float4(b32[1][0], b32[1][1], b32[1][2], b32[1][3]);
    nodes32[4 * i + 2] = make_float4(b32[0][4], b32[0][5], b32[1][4], b32[1][5]);
    nodes32[4 * i + 3] = make_float4(__int_as_float(ref[0]), __int_as_float(ref[1]), 0.f, 0.f);
    if (nodes64) {
        for (int h = 0; h < 2; h++)
            for (int d = 0; d < 3; d++) nodes64[8 * i + 3 * h + d] = make_double2(b64[h][2 * d], b64[h][2 * d + 1]);
        nodes64[8 * i + 6] = make_double2(__longlong_as_double((long long)(unsigned)ref[0]),
                                          __longlong_as_double((long long)(unsigned)ref[1]));
        nodes64[8 * i + 7] = make_double2(0.0, 0.0);
    }
}

// A single root holding one leaf over all n <= L triangles (child 1 empty, inverted box).
__global__ void k_write_small_root(int n, const float *__restrict__ box32, const double *__restrict__ box64,
                                   float4 *__restrict__ nodes32, double2 *__restrict__ nodes64) {
    float b[6] = {FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX};
    double e[6] = {DBL_MAX, -DBL_MAX, DBL_MAX, -DBL_MAX, DBL_MAX, -DBL_MAX};
    for (int t = 0; t < n; t++)
        for (int k = 0; k < 6; k += 2) {
            b[k] = fminf(b[k], box32[6 * t + k]), b[k + 1] = fmaxf(b[k + 1], box32[6 * t + k + 1]);
            e[k] = fmin(e[k], box64[6 * t + k]), e[k + 1] = fmax(e[k + 1], box64[6 * t + k + 1]);
        }
    const float inf = __int_as_float(0x7f800000);
    nodes32[0] = make_float4(b[0], b[1], b[2], b[3]);
    nodes32[1] = make_float4(inf, -inf, inf, -inf);
    nodes32[2] = make_float4(b[4], b[5], inf, -inf);
    nodes32[3] = make_float4(__int_as_float(leaf_ref(0, n)), __int_as_float(kEmptyRef), 0.f, 0.f);
    if (nodes64) {
        const double dinf = __longlong_as_double(0x7ff0000000000000ll);
        for (int d = 0; d < 3; d++) {
            nodes64[d] = make_double2(e[2 * d], e[2 * d + 1]);
            nodes64[3 + d] = make_double2(dinf, -dinf);
        }
        nodes64[6] = make_double2(__longlong_as_double((long long)(unsigned)leaf_ref(0, n)),
                                  __longlong_as_double((long long)(unsigned)kEmptyRef));
        nodes64[7] = make_double2(0.0, 0.0);
    }
}

// 4-wide nodes, top-down: a node starts from its binary node's two children and repeatedly opens
// the expandable child (internal, > L triangles) of largest surface area until it has four.
// Internal children become the next level's nodes (slots taken from an atomic counter).
__device__ __forceinline__ float box_area(const float *b) {
    const float dx = b[1] - b[0], dy = b[3] - b[2], dz = b[5] - b[4];
    return dx * dy + dy * dz + dz * dx;
}

__global__ void k_collapse4(const int *__restrict__ n_in_ptr, const int2 *__restrict__ qin, int2 *__restrict__ qout,
                            int *__restrict__ n_out,
                            int *__restrict__ slots, int L, const int *__restrict__ child_l,
                            const int *__restrict__ child_r, const int *__restrict__ first_of,
                            const int *__restrict__ count, const int *__restrict__ sorted_ids,
                            const float *__restrict__ pbox32, const double *__restrict__ pbox64,
                            const float *__restrict__ nbox32, const double *__restrict__ nbox64,
                            float4 *__restrict__ n32, double2 *__restrict__ n64) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *n_in_ptr) return;  // the level's size, written by the level above
    const int b = qin[i].x, slot = qin[i].y;
    int c[4] = {child_l[b], child_r[b], 0, 0};
    int nc = 2;
    while (nc < 4) {
        int pick = -1;
        float area = -1.f;
        for (int k = 0; k < nc; k++) {
            if (c[k] >= 0 && count[c[k]] > L) {
                const float a = box_area(nbox32 + 6 * c[k]);
                if (a > area) area = a, pick = k;
            }
        }
        if (pick < 0) break;
        const int x = c[pick];
        c[pick] = child_l[x];
        c[nc++] = child_r[x];
    }
    const float inf = __int_as_float(0x7f800000);
    const double dinf = __longlong_as_double(0x7ff0000000000000ll);
    float b32[6][4];
    double b64[6][4];
    int ref[4];
    for (int k = 0; k < 4; k++) {
        const float *f = nullptr;
        const double *d = nullptr;
        if (k >= nc) {
            ref[k] = kEmptyRef;
        } else if (c[k] < 0) {
            const int pos = -c[k] - 1;
            ref[k] = leaf_ref(pos, 1);
            f = pbox32 + 6 * sorted_ids[pos];
            d = pbox64 + 6 * sorted_ids[pos];
        } else {
            f = nbox32 + 6 * c[k];
            d = nbox64 + 6 * c[k];
            if (count[c[k]] <= L) {
                ref[k] = leaf_ref(first_of[c[k]], count[c[k]]);
            } else {
                ref[k] = atomicAdd(slots, 1);
                qout[atomicAdd(n_out, 1)] = make_int2(c[k], ref[k]);
            }
        }
        for (int r = 0; r < 6; r++) {
            b32[r][k] = f ? f[r] : ((r & 1) ? -inf : inf);
            b64[r][k] = d ? d[r] : ((r & 1) ? -dinf : dinf);
        }
    }
    // rows: lo x, hi x, lo y, hi y, lo z, hi z (box arrays are lo/hi interleaved per axis)
    for (int r = 0; r < 6; r++) {
        n32[8 * slot + r] = make_float4(b32[r][0], b32[r][1], b32[r][2], b32[r][3]);
        if (n64) {
            n64[14 * slot + 2 * r] = make_double2(b64[r][0], b64[r][1]);
            n64[14 * slot + 2 * r + 1] = make_double2(b64[r][2], b64[r][3]);
        }
    }
    n32[8 * slot + 6] =
        make_float4(__int_as_float(ref[0]), __int_as_float(ref[1]), __int_as_float(ref[2]), __int_as_float(ref[3]));
    n32[8 * slot + 7] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (n64) {
        n64[14 * slot + 12] =
            make_double2(__longlong_as_double((long long)(unsigned(ref[0])) | ((long long)(unsigned(ref[1])) << 32)),
                         __longlong_as_double((long long)(unsigned(ref[2])) | ((long long)(unsigned(ref[3])) << 32)));
        n64[14 * slot + 13] = make_double2(0.0, 0.0);
    }
}

// Start of the 4-wide collapse: level 0 is the root (binary node 0 into slot 0), one slot used.
__global__ void k_collapse4_init(int2 *__restrict__ q0, int *__restrict__ level_sizes, int *__restrict__ slots) {
    q0[0] = make_int2(0, 0);
    level_sizes[0] = 1;
    *slots = 1;
}

// The flag words of the build: [0] the first bad triangle (none: INT_MAX), [1..6] the scene's box as
// ordered ints (min seeded with +FLT_MAX, max with -FLT_MAX), the rest zero.
__global__ void k_init_flags(int *__restrict__ flags) {
    const int k = threadIdx.x;
    if (k >= 16) return;
    int v = 0;
    if (k == 0) v = 0x7fffffff;
    if (k >= 1 && k <= 3) v = 0x7f7fffff;
    if (k >= 4 && k <= 6) v = int(0xff7fffffu ^ 0x7fffffffu);
    flags[k] = v;
}

// The 4-wide root of a mesh of <= L triangles: one leaf, three empty slots.
__global__ void k_write_small_root4(int n, const float *__restrict__ box32, const double *__restrict__ box64,
                                    float4 *__restrict__ n32, double2 *__restrict__ n64) {
    float b[6] = {FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX};
    double e[6] = {DBL_MAX, -DBL_MAX, DBL_MAX, -DBL_MAX, DBL_MAX, -DBL_MAX};
    for (int t = 0; t < n; t++)
        for (int k = 0; k < 6; k += 2) {
            b[k] = fminf(b[k], box32[6 * t + k]), b[k + 1] = fmaxf(b[k + 1], box32[6 * t + k + 1]);
            e[k] = fmin(e[k], box64[6 * t + k]), e[k + 1] = fmax(e[k + 1], box64[6 * t + k + 1]);
        }
    const float inf = __int_as_float(0x7f800000);
    const double dinf = __longlong_as_double(0x7ff0000000000000ll);
    for (int r = 0; r < 6; r++) {
        const float pad = (r & 1) ? -inf : inf;
        const double dpad = (r & 1) ? -dinf : dinf;
        n32[r] = make_float4(b[r], pad, pad, pad);
        if (n64) n64[2 * r] = make_double2(e[r], dpad), n64[2 * r + 1] = make_double2(dpad, dpad);
    }
    const int e0 = kEmptyRef;
    n32[6] = make_float4(__int_as_float(leaf_ref(0, n)), __int_as_float(e0), __int_as_float(e0), __int_as_float(e0));
    n32[7] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (n64) {
        n64[12] = make_double2(
            __longlong_as_double((long long)(unsigned(leaf_ref(0, n))) | ((long long)(unsigned(e0)) << 32)),
            __longlong_as_double((long long)(unsigned(e0)) | ((long long)(unsigned(e0)) << 32)));
        n64[13] = make_double2(0.0, 0.0);
    }
}

// Depth and leaf count of the collapsed tree: a node is kept iff its subtree has > L triangles
// (its ancestors then have more), so walk parents from every kept node.
__global__ void k_depth(int n, int L, const int *__restrict__ count, const int *__restrict__ parent_int,
                        const int *__restrict__ child_l, const int *__restrict__ child_r, int *__restrict__ stats) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    if (i != 0 && count[i] <= L) return;
    int depth = 1;
    for (int p = parent_int[i]; p >= 0 && depth < 1 << 20; p = parent_int[p]) depth++;
    atomicMax(&stats[0], depth);
    int leaves = 0;
    const int c[2] = {child_l[i], child_r[i]};
    for (int h = 0; h < 2; h++) leaves += (c[h] < 0 || count[c[h]] <= L) ? 1 : 0;
    atomicAdd(&stats[1], leaves);
}

// The fix-up path's FP32 filter record of one triangle: the triangle itself, or, when it is
// ill-conditioned (height below 1/8 of its longest edge PQ, third corner R), a proxy triangle that
// contains it: PQ widened by L/4 at both ends (L = |PQ|) and an apex L/2 off its middle, towards R in
// the triangle's plane. R projects inside PQ (PQ is the longest edge) at height below L/8, and the
// proxy is at least L/6 high over all of PQ, so it contains P, Q and R; its distance is a lower
// bound of the triangle's, and its height (1/3 of its base) keeps the float test accurate. A proxy's
// record has the sign bit of its ab.ab set: its key may enter the window but never moves its centre.
__device__ bool filter_record(double ax, double ay, double az, double bx, double by, double bz, double cx,
                              double cy, double cz, int t, float4 *__restrict__ out) {
    const double abx = bx - ax, aby = by - ay, abz = bz - az, acx = cx - ax, acy = cy - ay, acz = cz - az;
    const double bcx = cx - bx, bcy = cy - by, bcz = cz - bz;
    const double lab = abx * abx + aby * aby + abz * abz, lac = acx * acx + acy * acy + acz * acz;
    const double lbc = bcx * bcx + bcy * bcy + bcz * bcz;
    const double l2 = fmax(fmax(lab, lac), lbc);
    const double nx = aby * acz - abz * acy, ny = abz * acx - abx * acz, nz = abx * acy - aby * acx;
    const bool ill = l2 > 0.0 && !(64.0 * (nx * nx + ny * ny + nz * nz) >= l2 * l2);
    double v[3][3] = {{ax, ay, az}, {bx, by, bz}, {cx, cy, cz}};
    if (ill) {
        // P, Q: the longest edge; R: the third corner
        int ip = 0, iq = 1, ir = 2;
        if (lac >= lab && lac >= lbc) ip = 0, iq = 2, ir = 1;
        else if (lbc >= lab && lbc >= lac) ip = 1, iq = 2, ir = 0;
        const double *P = v[ip], *Q = v[iq], *R = v[ir];
        const double L = sqrt(l2);
        double e[3] = {(Q[0] - P[0]) / L, (Q[1] - P[1]) / L, (Q[2] - P[2]) / L};
        const double rp[3] = {R[0] - P[0], R[1] - P[1], R[2] - P[2]};
        const double x = rp[0] * e[0] + rp[1] * e[1] + rp[2] * e[2];
        double u[3] = {rp[0] - x * e[0], rp[1] - x * e[1], rp[2] - x * e[2]};  // R's offset off PQ
        double lu = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        if (!(lu > 1e-9 * L)) {  // collinear to rounding: any direction across PQ
            const double w[3] = {fabs(e[0]) < 0.9 ? 1.0 : 0.0, fabs(e[0]) < 0.9 ? 0.0 : 1.0, 0.0};
            u[0] = e[1] * w[2] - e[2] * w[1], u[1] = e[2] * w[0] - e[0] * w[2], u[2] = e[0] * w[1] - e[1] * w[0];
        }
        const double ue = u[0] * e[0] + u[1] * e[1] + u[2] * e[2];  // re-orthogonalised against PQ
        for (int d = 0; d < 3; d++) u[d] -= ue * e[d];
        lu = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        for (int d = 0; d < 3; d++) u[d] /= lu;
        double pr[3][3];
        for (int d = 0; d < 3; d++) {
            pr[0][d] = P[d] - 0.25 * L * e[d];
            pr[1][d] = Q[d] + 0.25 * L * e[d];
            pr[2][d] = 0.5 * (P[d] + Q[d]) + 0.5 * L * u[d];
        }
        for (int a = 0; a < 3; a++)
            for (int d = 0; d < 3; d++) v[a][d] = pr[a][d];
    }
    // a, ab = b - a, ac = c - a and the products ab.ab, ac.ac, ab.ac, from the rounded corners (so the
    // record is the triangle the float corners describe), in double and then rounded once
    float f[3][3];
    for (int k = 0; k < 3; k++)
        for (int d = 0; d < 3; d++) f[k][d] = float(v[k][d]);
    double eb[3], ec[3];
    for (int d = 0; d < 3; d++) eb[d] = double(f[1][d]) - double(f[0][d]), ec[d] = double(f[2][d]) - double(f[0][d]);
    const double bb = eb[0] * eb[0] + eb[1] * eb[1] + eb[2] * eb[2];
    const double cc = ec[0] * ec[0] + ec[1] * ec[1] + ec[2] * ec[2];
    const double bc = eb[0] * ec[0] + eb[1] * ec[1] + eb[2] * ec[2];
    // a proxy is marked by the sign bit of ab.ab (never negative otherwise)
    const float fbb = float(bb);
    out[0] = make_float4(f[0][0], f[0][1], f[0][2], ill ? __int_as_float(__float_as_int(fbb) | 0x80000000) : fbb);
    out[1] = make_float4(float(eb[0]), float(eb[1]), float(eb[2]), float(cc));
    out[2] = make_float4(float(ec[0]), float(ec[1]), float(ec[2]), float(bc));
    (void)t;
    return ill;
}

// The fix-up window's bound term of one filter record (the triangle the float corners describe, or its
// proxy): the FP32 filter's error at a query p is at most u (8 R + 7.7 alpha L) + min(D, 2 D^2 / d) with D
// = 90 u alpha R (device_geom.cuh, tri_dist_sq_filter, states the terms it bounds: input rounding, each
// fmaf, the quotient and reciprocal, the region decisions), u = 2^-24, L the record's longest edge, alpha =
// L^2 / |ab x ac| and R the largest distance from p to a corner. That is at most u (17 d + (16 + 188 alpha)
// L) at any distance d (near the record R <= 2L; far from it the D^2 term is below u d); with the input
// rounding of p and of the corners it stays below u (18.1 d + 2 sqrt(3) M) + u (20 + 188 alpha) L, M the
// largest coordinate magnitude. This returns the record's term (20 + 188 alpha) L, and false when the
// record is not safe for the float filter: an edge shorter than 2^-23 (its products underflow), a record
// that rounding to float made degenerate or needle-like (alpha > 16), or a non-finite value.
__device__ bool filter_bound(const float4 *__restrict__ rec, float *term) {
    const double e1[3] = {rec[1].x, rec[1].y, rec[1].z}, e2[3] = {rec[2].x, rec[2].y, rec[2].z};
    const double e3[3] = {e2[0] - e1[0], e2[1] - e1[1], e2[2] - e1[2]};
    const double l1 = e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2];
    const double l2 = e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2];
    const double l3 = e3[0] * e3[0] + e3[1] * e3[1] + e3[2] * e3[2];
    const double ll = fmax(fmax(l1, l2), l3);
    *term = 0.f;
    if (ll == 0.0) return true;  // all corners equal: only the corner test runs, exactly
    const double nx = e1[1] * e2[2] - e1[2] * e2[1], ny = e1[2] * e2[0] - e1[0] * e2[2];
    const double nz = e1[0] * e2[1] - e1[1] * e2[0];
    const double n = sqrt(nx * nx + ny * ny + nz * nz);
    const double shortest = fmin(fmin(l1, l2), l3);
    const double alpha = ll / n;
    if (!(shortest >= 0x1p-46) || !(alpha <= 16.0) || !(ll < 0x1p120)) return false;
    *term = __double2float_ru((20.0 + 188.0 * alpha) * sqrt(ll));
    return true;
}

}  // namespace

// The window (sqrt(best) + tau)^2 (1 + 2^-16), tau = tau_rel (M + sqrt(best)), keeps the double
// winner whenever tau exceeds the sum of its key's error above its distance and the error below of
// the key that set best. With the bound above both are at most u (18.1 d + 2 sqrt(3) M + term), so
// tau_rel >= u (6.93 + 2 term / M) and tau_rel >= 36.2 u suffice (2^-9 added for best lying below
// the winner's distance; the (1 + 2^-16) factor covers the rounding of the window itself). The
// default 2^-16 = 256 u holds them whenever term / M <= 124: the torus-knot tube's largest term is 27.7 M (a triangle of aspect 7.2),
// a 320-triangle sphere's 94 M; a mesh of a few large triangles gets a wider window. A mesh whose
// window would pass 2^-8, or with a record the float filter cannot take, is answered by the FP64
// kernel.
void set_filter_window(DeviceMesh *m, float largest_term, bool records_safe) {
    const double u = 0x1p-24, M = double(m->coord_scale);
    double tau = 1.0 / 65536.0;
    if (largest_term > 0.f) {
        if (!(M > 0.0)) {
            m->tau_rel_min = 1.0f;
            m->filter_ok = 0;
            return;
        }
        tau = fmax(tau, u * (6.93 + 2.0 * double(largest_term) / M) * (1.0 + 0x1p-9));
    }
    m->tau_rel_min = float(tau) < tau ? nextafterf(float(tau), INFINITY) : float(tau);
    m->filter_ok = records_safe && M <= double(kFilterMaxCoord) && tau <= 0x1p-8 ? 1 : 0;
}

namespace {

__global__ void k_tri_records(int nt, const int *__restrict__ sorted_ids, const int *__restrict__ s0,
                              const int *__restrict__ s1, const int *__restrict__ s2, const double *__restrict__ vx,
                              const double *__restrict__ vy, const double *__restrict__ vz, float4 *__restrict__ t32,
                              double2 *__restrict__ t64, float4 *__restrict__ filt, int *__restrict__ nill) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nt) return;
    const int t = sorted_ids[p];
    const int a = s0[t], b = s1[t], c = s2[t];
    const double ax = vx[a], ay = vy[a], az = vz[a], bx = vx[b], by = vy[b], bz = vz[b];
    const double cx = vx[c], cy = vy[c], cz = vz[c];
    t32[3 * p + 0] = make_float4(float(ax), float(ay), float(az), float(bx));
    t32[3 * p + 1] = make_float4(float(by), float(bz), float(cx), float(cy));
    t32[3 * p + 2] = make_float4(float(cz), __int_as_float(t), 0.f, 0.f);
    if (filt) {
        if (filter_record(ax, ay, az, bx, by, bz, cx, cy, cz, t, filt + 3 * size_t(p))) atomicAdd(nill, 1);
        float term;
        if (filter_bound(filt + 3 * size_t(p), &term))
            atomicMax(nill + 1, __float_as_int(term));  // non-negative floats order like their bits
        else
            atomicAdd(nill + 2, 1);
    }
    if (t64) {
        t64[5 * p + 0] = make_double2(ax, ay);
        t64[5 * p + 1] = make_double2(az, bx);
        t64[5 * p + 2] = make_double2(by, bz);
        t64[5 * p + 3] = make_double2(cx, cy);
        t64[5 * p + 4] = make_double2(cz, double(t));
    }
}

// ---- pseudo-normals --------------------------------------------------------------------------------

// Face normals, the per-(face, corner) angle contributions in visit order 3t + v, the vertex and
// edge sort keys; edge normals initialised to the face's own (serial/bvh/bvh.cpp:1681-1710).
__global__ void k_face_normals(int nt, int nv, const int *__restrict__ s0, const int *__restrict__ s1,
                               const int *__restrict__ s2, const double *__restrict__ vx,
                               const double *__restrict__ vy, const double *__restrict__ vz,
                               double *__restrict__ face_n, double *__restrict__ edge_n, double *__restrict__ contrib,
                               uint32_t *__restrict__ vkey, int *__restrict__ vval, uint64_t *__restrict__ ekey,
                               int *__restrict__ eval) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const int id[3] = {s0[t], s1[t], s2[t]};
    double p[3][3];
    for (int v = 0; v < 3; v++) p[v][0] = vx[id[v]], p[v][1] = vy[id[v]], p[v][2] = vz[id[v]];
    const double u[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
    const double w[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
    double n[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
    const double len = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    if (len > 0) {
        for (int d = 0; d < 3; d++) n[d] /= len;
    }
    for (int d = 0; d < 3; d++) face_n[3 * t + d] = n[d];
    for (int v = 0; v < 3; v++) {
        const double *a = p[v], *b = p[(v + 1) % 3], *c = p[(v + 2) % 3];
        const double e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
        const double e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
        const double l1 = sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
        const double l2 = sqrt(e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2]);
        const double cosine = (l1 > 0 && l2 > 0) ? (e1[0] * e2[0] + e1[1] * e2[1] + e1[2] * e2[2]) / (l1 * l2) : 1.0;
        const double mn = (cosine < 1.0) ? cosine : 1.0;
        const double cl = (-1.0 < mn) ? mn : -1.0;
        const double angle = acos(cl);
        for (int d = 0; d < 3; d++) contrib[3 * (3 * t + v) + d] = angle * n[d];
        vkey[3 * t + v] = uint32_t(id[v]);
        vval[3 * t + v] = 3 * t + v;
    }
    for (int e = 0; e < 3; e++) {
        for (int d = 0; d < 3; d++) edge_n[9 * t + 3 * e + d] = n[d];
        const uint64_t a = uint64_t(id[e]), b = uint64_t(id[(e + 1) % 3]);
        ekey[3 * t + e] = (a < b ? a : b) * uint64_t(nv) + (a < b ? b : a);
        eval[3 * t + e] = 3 * t + e;
    }
}

// One thread per run of equal vertex keys: sums the contributions in visit order.
__global__ void k_vertex_sums(int nocc, const uint32_t *__restrict__ vkey, const int *__restrict__ vval,
                              const double *__restrict__ contrib, double *__restrict__ vertex_n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nocc) return;
    if (i > 0 && vkey[i - 1] == vkey[i]) return;
    double acc[3] = {0.0, 0.0, 0.0};
    int j = i;
    for (; j < nocc && vkey[j] == vkey[i]; j++) {
        const int o = vval[j];
        for (int d = 0; d < 3; d++) acc[d] += contrib[3 * o + d];
    }
    for (int d = 0; d < 3; d++) vertex_n[3 * size_t(vkey[i]) + d] = acc[d];
}

// One thread per run of equal edge keys: replays the reference's first-occurrence map.
__global__ void k_edge_sums(int nocc, const uint64_t *__restrict__ ekey, const int *__restrict__ eval,
                            const double *__restrict__ face_n, double *__restrict__ edge_n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nocc) return;
    if (i > 0 && ekey[i - 1] == ekey[i]) return;
    const int first = eval[i];
    int j = i + 1;
    for (; j < nocc && ekey[j] == ekey[i]; j++) {
        const int o = eval[j];
        for (int d = 0; d < 3; d++) {
            const double sum = face_n[3 * (first / 3) + d] + face_n[3 * (o / 3) + d];
            edge_n[9 * (o / 3) + 3 * (o % 3) + d] = sum;
            edge_n[9 * (first / 3) + 3 * (first % 3) + d] = sum;
        }
    }
}

int bits_for(uint64_t maxval) {
    int b = 1;
    while (b < 64 && (maxval >> b) != 0) b++;
    return b;
}

#define LAUNCH_CHECK(what)                                                  \
    do {                                                                    \
        cudaError_t e_ = cudaGetLastError();                                \
        if (e_ != cudaSuccess) return cuda_fail(e_, what, __FILE__, __LINE__); \
    } while (0)

int build_normals(MeshStorage *s, DeviceMesh *m, const int *s0, const int *s1, const int *s2, const double *vx,
                  const double *vy, const double *vz, cudaStream_t stream) {
    const int nt = m->nt, nv = m->nv, nocc = 3 * nt;
    double *face_n, *edge_n, *vertex_n;
    SSDF_CHECK(dalloc(s, &face_n, 3 * size_t(nt), stream));
    SSDF_CHECK(dalloc(s, &edge_n, 9 * size_t(nt), stream));
    SSDF_CHECK(dalloc(s, &vertex_n, 3 * size_t(nv), stream));
    MeshStorage tmp;
    double *contrib;
    uint32_t *vkey;
    uint64_t *ekey;
    int *vval, *eval;
    int st = SSDF_OK;
    if ((st = dalloc(&tmp, &contrib, 3 * size_t(nocc), stream)) == SSDF_OK &&
        (st = dalloc(&tmp, &vkey, nocc, stream)) == SSDF_OK && (st = dalloc(&tmp, &vval, nocc, stream)) == SSDF_OK &&
        (st = dalloc(&tmp, &ekey, nocc, stream)) == SSDF_OK && (st = dalloc(&tmp, &eval, nocc, stream)) == SSDF_OK) {
        cudaMemsetAsync(vertex_n, 0, sizeof(double) * 3 * size_t(nv), stream);
        k_face_normals<<<grid_blocks(nt, 128), 128, 0, stream>>>(nt, nv, s0, s1, s2, vx, vy, vz, face_n, edge_n,
                                                                 contrib, vkey, vval, ekey, eval);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) st = cuda_fail(e, "k_face_normals", __FILE__, __LINE__);
        if (st == SSDF_OK) st = radix_sort_pairs_u32(vkey, vval, nocc, bits_for(uint64_t(nv)), stream);
        if (st == SSDF_OK)
            st = radix_sort_pairs_u64(ekey, eval, nocc, bits_for(uint64_t(nv) * uint64_t(nv)), stream);
        if (st == SSDF_OK) {
            k_vertex_sums<<<grid_blocks(nocc, 256), 256, 0, stream>>>(nocc, vkey, vval, contrib, vertex_n);
            k_edge_sums<<<grid_blocks(nocc, 256), 256, 0, stream>>>(nocc, ekey, eval, face_n, edge_n);
            e = cudaGetLastError();
            if (e != cudaSuccess) st = cuda_fail(e, "normal sums", __FILE__, __LINE__);
        }
    }
    for (void *p : tmp.blocks) cudaFreeAsync(p, stream);
    m->face_n = face_n;
    m->edge_n = edge_n;
    m->vertex_n = vertex_n;
    return st;
}

}  // namespace

// The storage comes from the stream-ordered pool (cudaMallocAsync): cudaFree on it does not wait for
// work that still reads it, so the caller has ensured that none does (ssdf_mesh_destroy waits for the
// device) -- or frees it in stream order behind that work with mesh_free_async.
void mesh_free(MeshStorage *storage) {
    if (!storage) return;
    for (void *p : storage->blocks) cudaFree(p);
    delete storage;
}

void mesh_free_async(MeshStorage *storage, cudaStream_t stream) {
    if (!storage) return;
    for (void *p : storage->blocks) cudaFreeAsync(p, stream);
    delete storage;
}

size_t mesh_bytes(const MeshStorage *storage) { return storage ? storage->bytes : 0; }

// Deepest 4-wide level the collapse writes: a tree that reaches it is refused (3 x depth4 must stay
// below kStackSize), so one more level than an accepted tree can have.
constexpr int kMaxLevels4 = kStackSize / 3 + 1;

// Page-locked words for the build's read-backs (one set per calling thread, kept until exit), so the
// copies stay asynchronous and the build waits once, at its end.
constexpr int kReadbackWords = 64;
static int readback_words(int **out) {
    static thread_local int *w = nullptr;
    if (!w) SSDF_CUDA(cudaHostAlloc((void **)&w, sizeof(int) * kReadbackWords, cudaHostAllocPortable));
    *out = w;
    return SSDF_OK;
}

static int mesh_build_impl(MeshStorage *s, MeshStorage *tmp, DeviceMesh *m, int nt, const int *s0_in,
                           const int *s1_in, const int *s2_in, int nv, const void *sx, const void *sy, const void *sz,
                           int coord_f64, int device_ptrs, const ssdf_build_opts &opts, cudaStream_t stream) {
    const int L = opts.leaf_size > 0 ? opts.leaf_size : 4;
    m->nt = nt;
    m->nv = nv;
    m->leaf_size = L;
    // indices (kept: the sign step needs the caller's vertex ids)
    int *s0, *s1, *s2;
    SSDF_CHECK(dalloc(s, &s0, nt, stream));
    SSDF_CHECK(dalloc(s, &s1, nt, stream));
    SSDF_CHECK(dalloc(s, &s2, nt, stream));
    const cudaMemcpyKind kind = device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    SSDF_CUDA(cudaMemcpyAsync(s0, s0_in, sizeof(int) * size_t(nt), kind, stream));
    SSDF_CUDA(cudaMemcpyAsync(s1, s1_in, sizeof(int) * size_t(nt), kind, stream));
    SSDF_CUDA(cudaMemcpyAsync(s2, s2_in, sizeof(int) * size_t(nt), kind, stream));
    m->s0 = s0, m->s1 = s1, m->s2 = s2;
    // vertices, widened to double
    const size_t gsz = coord_f64 ? sizeof(double) : sizeof(float);
    void *gx, *gy, *gz;
    double *vx, *vy, *vz;
    SSDF_CHECK(dalloc(tmp, &vx, nv, stream));
    SSDF_CHECK(dalloc(tmp, &vy, nv, stream));
    SSDF_CHECK(dalloc(tmp, &vz, nv, stream));
    if (device_ptrs) {
        gx = const_cast<void *>(sx), gy = const_cast<void *>(sy), gz = const_cast<void *>(sz);
    } else {
        char *g;
        SSDF_CHECK(dalloc(tmp, &g, 3 * gsz * size_t(nv), stream));
        gx = g, gy = g + gsz * nv, gz = g + 2 * gsz * nv;
        SSDF_CUDA(cudaMemcpyAsync(gx, sx, gsz * nv, cudaMemcpyHostToDevice, stream));
        SSDF_CUDA(cudaMemcpyAsync(gy, sy, gsz * nv, cudaMemcpyHostToDevice, stream));
        SSDF_CUDA(cudaMemcpyAsync(gz, sz, gsz * nv, cudaMemcpyHostToDevice, stream));
    }
    if (coord_f64)
        k_widen<double><<<grid_blocks(nv, 256), 256, 0, stream>>>(nv, (const double *)gx, (const double *)gy,
                                                                  (const double *)gz, vx, vy, vz);
    else
        k_widen<float><<<grid_blocks(nv, 256), 256, 0, stream>>>(nv, (const float *)gx, (const float *)gy,
                                                                 (const float *)gz, vx, vy, vz);
    LAUNCH_CHECK("k_widen");
    // validation + per-triangle boxes
    // [0] first bad triangle, [1..6] scene, [7] scale, [8..9] depth / leaves, [10] ill, [11] largest
    // filter bound term (float bits), [12] records unsafe for the float filter
    int *flags;
    SSDF_CHECK(dalloc(tmp, &flags, 16, stream));
    k_init_flags<<<1, 32, 0, stream>>>(flags);
    LAUNCH_CHECK("k_init_flags");
    if (device_ptrs) {
        // host arrays were checked on the host (check_mesh_host); device arrays are checked here,
        // before any kernel indexes the vertices with them
        k_validate<<<grid_blocks(nt, 256), 256, 0, stream>>>(nt, nv, s0, s1, s2, flags);
        LAUNCH_CHECK("k_validate");
        int bad = 0;
        SSDF_CUDA(cudaMemcpyAsync(&bad, flags, sizeof(int), cudaMemcpyDeviceToHost, stream));
        SSDF_CUDA(cudaStreamSynchronize(stream));
        if (bad != 0x7fffffff)
            return fail(SSDF_ERR_INVALID_ARGUMENT, "triangle " + std::to_string(bad) +
                                                       " has a vertex index outside [0, " + std::to_string(nv) + ")");
    }
    float *box32, *cen;
    double *box64;
    SSDF_CHECK(dalloc(tmp, &box32, 6 * size_t(nt), stream));
    SSDF_CHECK(dalloc(tmp, &box64, 6 * size_t(nt), stream));
    SSDF_CHECK(dalloc(tmp, &cen, 3 * size_t(nt), stream));
    k_prep<<<grid_blocks(nt, 256), 256, 0, stream>>>(nt, s0, s1, s2, vx, vy, vz, box32, box64, cen, flags + 1,
                                                     flags + 7);
    LAUNCH_CHECK("k_prep");
    // Morton order
    uint32_t *keys;
    int *ids;
    SSDF_CHECK(dalloc(tmp, &keys, nt, stream));
    SSDF_CHECK(dalloc(tmp, &ids, nt, stream));
    k_morton<<<grid_blocks(nt, 256), 256, 0, stream>>>(nt, cen, flags + 1, keys, ids);
    LAUNCH_CHECK("k_morton");
    SSDF_CHECK(radix_sort_pairs_u32(keys, ids, nt, 30, stream));
    // topology
    const bool keep64 = opts.keep_fp64 != 0;
    const int nint = nt > 1 ? nt - 1 : 0;
    m->nnodes = nint > 0 ? nint : 1;
    float4 *nodes32;
    double2 *nodes64 = nullptr;
    SSDF_CHECK(dalloc(s, &nodes32, 4 * size_t(m->nnodes), stream));
    if (keep64) SSDF_CHECK(dalloc(s, &nodes64, 8 * size_t(m->nnodes), stream));
    float4 *nodes4_32;
    double2 *nodes4_64 = nullptr;
    SSDF_CHECK(dalloc(s, &nodes4_32, 8 * size_t(m->nnodes), stream));
    if (keep64) SSDF_CHECK(dalloc(s, &nodes4_64, 14 * size_t(m->nnodes), stream));
    // read-backs: [0..1] depth and leaves, [2..2 + kMaxLevels4] 4-wide level sizes, then the slots
    // used, then the coordinate scale and the three filter words
    static_assert(2 + kMaxLevels4 + 2 + 4 <= kReadbackWords, "read-back words");
    int *rb = nullptr;
    SSDF_CHECK(readback_words(&rb));
    int *const depth_leaves = rb, *const level_hist = rb + 2;
    int *const scale_word = rb + 2 + kMaxLevels4 + 2, *const filt_info = scale_word + 1;
    depth_leaves[0] = depth_leaves[1] = 1;
    int nnodes4 = 1, depth4 = 1;
    bool collapsed = false;
    if (nt <= L) {
        // one leaf over everything (its triangle order is the Morton order)
        k_write_small_root<<<1, 1, 0, stream>>>(nt, box32, box64, nodes32, nodes64);
        LAUNCH_CHECK("k_write_small_root");
        k_write_small_root4<<<1, 1, 0, stream>>>(nt, box32, box64, nodes4_32, nodes4_64);
        LAUNCH_CHECK("k_write_small_root4");
    } else {
        int *child_l, *child_r, *first_of, *last_of, *parent_int, *parent_leaf, *arrivals, *count;
        float *nbox32;
        double *nbox64;
        SSDF_CHECK(dalloc(tmp, &child_l, nint, stream));
        SSDF_CHECK(dalloc(tmp, &child_r, nint, stream));
        SSDF_CHECK(dalloc(tmp, &first_of, nint, stream));
        SSDF_CHECK(dalloc(tmp, &last_of, nint, stream));
        SSDF_CHECK(dalloc(tmp, &parent_int, nint, stream));
        SSDF_CHECK(dalloc(tmp, &parent_leaf, nt, stream));
        SSDF_CHECK(dalloc(tmp, &arrivals, nint, stream));
        SSDF_CHECK(dalloc(tmp, &count, nint, stream));
        SSDF_CHECK(dalloc(tmp, &nbox32, 6 * size_t(nint), stream));
        SSDF_CHECK(dalloc(tmp, &nbox64, 6 * size_t(nint), stream));
        k_karras<<<grid_blocks(nint, 256), 256, 0, stream>>>(nt, keys, child_l, child_r, first_of, last_of,
                                                             parent_int, parent_leaf);
        LAUNCH_CHECK("k_karras");
        SSDF_CUDA(cudaMemsetAsync(arrivals, 0, sizeof(int) * nint, stream));
        k_refit<<<grid_blocks(nt, 256), 256, 0, stream>>>(nt, ids, child_l, child_r, parent_int, parent_leaf, box32,
                                                          box64, nbox32, nbox64, arrivals);
        LAUNCH_CHECK("k_refit");
        for (int round = 0; round < opts.treelet_opt && round < 8; round++) {  // treelet_opt: rounds (0 = none)
            SSDF_CHECK(treelet_optimize(nt, child_l, child_r, parent_int, parent_leaf, first_of, nbox32, nbox64,
                                        box32, box64, ids, stream));
        }
        SSDF_CUDA(cudaMemsetAsync(arrivals, 0, sizeof(int) * nint, stream));
        k_counts<<<grid_blocks(nt, 256), 256, 0, stream>>>(nt, child_l, child_r, parent_int, parent_leaf, count,
                                                           arrivals);
        LAUNCH_CHECK("k_counts");
        k_write_nodes<<<grid_blocks(nint, 256), 256, 0, stream>>>(nt, L, child_l, child_r, first_of, count, ids,
                                                                  box32, box64, nbox32, nbox64, nodes32, nodes64);
        LAUNCH_CHECK("k_write_nodes");
        k_depth<<<grid_blocks(nint, 256), 256, 0, stream>>>(nt, L, count, parent_int, child_l, child_r, flags + 8);
        LAUNCH_CHECK("k_depth");
        SSDF_CUDA(cudaMemcpyAsync(depth_leaves, flags + 8, 2 * sizeof(int), cudaMemcpyDeviceToHost, stream));
        // 4-wide collapse, one level per launch. Each level's kernel reads its size from the level
        // above, so the host launches kMaxLevels4 levels without waiting between them (a grid of at
        // most min(4^k, nint) threads at level k); the sizes come back with the build's last sync.
        // A tree with a level at kMaxLevels4 is too deep for the traversal stack (3 x depth4 <
        // kStackSize) and is refused below.
        int2 *qa, *qb;
        int *level_sizes;  // [kMaxLevels4 + 1] queue sizes per level, then the slots used
        SSDF_CHECK(dalloc(tmp, &qa, nint, stream));
        SSDF_CHECK(dalloc(tmp, &qb, nint, stream));
        SSDF_CHECK(dalloc(tmp, &level_sizes, kMaxLevels4 + 2, stream));
        SSDF_CUDA(cudaMemsetAsync(level_sizes, 0, sizeof(int) * (kMaxLevels4 + 2), stream));
        k_collapse4_init<<<1, 1, 0, stream>>>(qa, level_sizes, level_sizes + kMaxLevels4 + 1);
        LAUNCH_CHECK("k_collapse4_init");
        long long bound = 1;
        for (int k = 0; k < kMaxLevels4; k++) {
            const int n_k = int(std::min<long long>(bound, nint));
            k_collapse4<<<grid_blocks(n_k, 128), 128, 0, stream>>>(
                level_sizes + k, qa, qb, level_sizes + k + 1, level_sizes + kMaxLevels4 + 1, L, child_l, child_r,
                first_of, count, ids, box32, box64, nbox32, nbox64, nodes4_32, nodes4_64);
            LAUNCH_CHECK("k_collapse4");
            bound *= 4;
            int2 *t = qa;
            qa = qb;
            qb = t;
        }
        SSDF_CUDA(cudaMemcpyAsync(level_hist, level_sizes, sizeof(int) * (kMaxLevels4 + 2), cudaMemcpyDeviceToHost,
                                  stream));  // page-locked: no wait here
        collapsed = true;
    }
    // triangle records in leaf order
    float4 *t32, *filt = nullptr;
    double2 *t64 = nullptr;
    SSDF_CHECK(dalloc(s, &t32, 3 * size_t(nt), stream));
    if (keep64) SSDF_CHECK(dalloc(s, &t64, 5 * size_t(nt), stream));
    if (keep64) SSDF_CHECK(dalloc(s, &filt, 3 * size_t(nt), stream));  // the fix-up path's filter records
    k_tri_records<<<grid_blocks(nt, 256), 256, 0, stream>>>(nt, ids, s0, s1, s2, vx, vy, vz, t32, t64, filt,
                                                            flags + 10);
    LAUNCH_CHECK("k_tri_records");
    SSDF_CUDA(cudaMemcpyAsync(scale_word, flags + 7, sizeof(int), cudaMemcpyDeviceToHost, stream));
    SSDF_CUDA(cudaMemcpyAsync(filt_info, flags + 10, 3 * sizeof(int), cudaMemcpyDeviceToHost, stream));
    if (opts.normals) SSDF_CHECK(build_normals(s, m, s0, s1, s2, vx, vy, vz, stream));
    SSDF_CUDA(cudaStreamSynchronize(stream));  // the build's one wait: every read-back has landed
    float scale;
    memcpy(&scale, scale_word, sizeof(float));
    m->coord_scale = scale;
    m->nill = filt_info[0];
    if (keep64) {
        float term;
        memcpy(&term, &filt_info[1], sizeof(float));
        set_filter_window(m, term, filt_info[2] == 0);
    }
    if (collapsed) {
        depth4 = 0;
        while (depth4 <= kMaxLevels4 && level_hist[depth4] > 0) depth4++;
        nnodes4 = level_hist[kMaxLevels4 + 1];
    }
    m->depth = depth_leaves[0];
    m->nleaves = depth_leaves[1];
    m->nodes32 = nodes32;
    m->nodes64 = nodes64;
    m->nodes4_32 = nodes4_32;
    m->nodes4_64 = nodes4_64;
    m->nnodes4 = nnodes4;
    m->depth4 = depth4;
    m->tris32 = t32;
    m->tris64 = t64;
    m->filt32 = filt;
    if (m->depth >= kStackSize || 3 * m->depth4 >= kStackSize)
        return fail(SSDF_ERR_NOT_SUPPORTED,
                    "BVH depth " + std::to_string(m->depth) + " exceeds the traversal stack (" +
                        std::to_string(kStackSize) + ")");
    return SSDF_OK;
}

int mesh_build(MeshStorage **storage, DeviceMesh *mesh, ptrdiff_t nt, const int *s0, const int *s1, const int *s2,
               ptrdiff_t nv, const void *sx, const void *sy, const void *sz, int coord_f64, int device_ptrs,
               const ssdf_build_opts &opts, cudaStream_t stream) {
    if (nt <= 0 || nv <= 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "empty mesh");
    if (nt >= kMaxTriangles) return fail(SSDF_ERR_NOT_SUPPORTED, "more than 2^26 triangles in one mesh");
    if (nv >= (1ll << 31)) return fail(SSDF_ERR_NOT_SUPPORTED, "more than 2^31 vertices");
    if (opts.leaf_size < 0 || opts.leaf_size > kMaxLeafSize)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "leaf_size must be 0 (default) or 1.." + std::to_string(kMaxLeafSize));
    if (!s0 || !s1 || !s2 || !sx || !sy || !sz) return fail(SSDF_ERR_INVALID_ARGUMENT, "null mesh array");
    retain_pool_memory();
    MeshStorage *s = new MeshStorage();
    MeshStorage tmp;
    *mesh = DeviceMesh();
    int st = mesh_build_impl(s, &tmp, mesh, int(nt), s0, s1, s2, int(nv), sx, sy, sz, coord_f64, device_ptrs, opts,
                             stream);
    for (void *p : tmp.blocks) cudaFreeAsync(p, stream);
    if (st == SSDF_OK) {
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) st = cuda_fail(e, "mesh build", __FILE__, __LINE__);
    }
    if (st != SSDF_OK) {
        cudaStreamSynchronize(stream);
        mesh_free(s);
        *mesh = DeviceMesh();
        return st;
    }
    *storage = s;
    return SSDF_OK;
}

}  // namespace ssdf_b200
