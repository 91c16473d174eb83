// treelet_opt.cu -- SAH treelet refinement of the LBVH (after Karras and Aila, "Fast parallel
// construction of high-quality bounding volume hierarchies", HPG 2013).
//
// One bottom-up pass with per-node arrival counters (the second thread to reach a node owns it, so
// its subtree is final; a warp then works on its lanes' treelets together): every node with at least
// kTreeletLeaves triangles below it roots a treelet,
// grown from its two children by opening the largest-area internal member until it has seven
// members. The binary tree over those members with the lowest surface-area cost,
//     cost(node) = area(node) + cost(left) + cost(right),   cost(triangle) = area(triangle),
// is found exactly by dynamic programming over the 127 member subsets (each subset's best split
// among its 2^k - 2 partitions), and replaces the old arrangement when it is cheaper, reusing the
// treelet's six internal nodes (the root keeps its identity, so the walk continues upward). Boxes
// and parent links inside the treelet are rewritten. The pass then re-derives the leaf order (a
// depth-first numbering of the triangles), so every subtree is again a contiguous range of leaf
// positions, as the leaf collapse and the node records require.
#include <cuda_runtime.h>

#include <cfloat>

#include "internal.h"

namespace ssdf_b200 {

namespace {

constexpr int kTreeletLeaves = 7;
constexpr int kSubsets = 1 << kTreeletLeaves;

struct TreeArrays {
    int *child_l, *child_r, *parent_int, *parent_leaf;
    float *nbox32;
    double *nbox64;
    const float *pbox32;
    const double *pbox64;
    const int *ids;  // leaf position -> triangle
    float *cost;     // per internal node: SAH cost of its subtree
    int *count;      // per internal node: triangles below
};

__device__ __forceinline__ float area6(const float *b) {
    const float dx = fmaxf(b[1] - b[0], 0.f), dy = fmaxf(b[3] - b[2], 0.f), dz = fmaxf(b[5] - b[4], 0.f);
    return 2.f * (dx * dy + dy * dz + dz * dx);
}

// Box / cost / count of a child reference (internal >= 0, leaf -(pos + 1)); reads bypass L1 since
// other threads wrote them.
__device__ __forceinline__ void ref_box32(const TreeArrays &t, int ref, float *b) {
    const float *s = ref >= 0 ? t.nbox32 + 6 * ref : t.pbox32 + 6 * t.ids[-ref - 1];
    for (int k = 0; k < 6; k++) b[k] = __ldcg(s + k);
}
__device__ __forceinline__ void ref_box64(const TreeArrays &t, int ref, double *b) {
    const double *s = ref >= 0 ? t.nbox64 + 6 * ref : t.pbox64 + 6 * t.ids[-ref - 1];
    for (int k = 0; k < 6; k++) b[k] = __ldcg(s + k);
}
__device__ __forceinline__ float ref_cost(const TreeArrays &t, int ref) {
    if (ref >= 0) return __ldcg(t.cost + ref);
    float b[6];
    ref_box32(t, ref, b);
    return area6(b);
}
__device__ __forceinline__ int ref_count(const TreeArrays &t, int ref) { return ref >= 0 ? __ldcg(t.count + ref) : 1; }

__device__ __forceinline__ void set_parent(const TreeArrays &t, int ref, int parent) {
    if (ref >= 0)
        __stcg(t.parent_int + ref, parent);
    else
        __stcg(t.parent_leaf + (-ref - 1), parent);
}

// A treelet in the making, in shared memory (one per warp): its members and their boxes and costs,
// the internal nodes it reuses, and the dynamic programme's cost and best split of every subset.
struct TreeletWork {
    double mb64[kTreeletLeaves][6];
    float mb[kTreeletLeaves][6];
    float mcost[kTreeletLeaves];
    int mcount[kTreeletLeaves];
    int member[kTreeletLeaves];
    int inner[kTreeletLeaves - 1];
    int m, ni;  // members, internal nodes (m < 3: nothing to optimise)
    float old_cost;
    float c[kSubsets];
    unsigned char split[kSubsets];
    unsigned char subs[40];  // a round's subsets, in increasing order (at most C(7, 3) = 35)
    // the rebuilt arrangement: internal node onode[k] now covers the members of subset oset[k]
    int onode[kTreeletLeaves - 1], oset[kTreeletLeaves - 1];
    int norder;
};

// One lane: grows the treelet rooted at internal node x (its subtree is final) from its two children
// by opening the largest-area internal member until it has seven members. A treelet of fewer than
// three members gets its cost stored here and w.m < 3.
__device__ void form_treelet(const TreeArrays &t, int x, TreeletWork &w) {
    int m = 2, ni = 1;
    w.member[0] = __ldcg(t.child_l + x);
    w.member[1] = __ldcg(t.child_r + x);
    w.inner[0] = x;
    ref_box32(t, w.member[0], w.mb[0]);
    ref_box32(t, w.member[1], w.mb[1]);
    while (m < kTreeletLeaves) {
        int pick = -1;
        float best = -1.f;
        for (int k = 0; k < m; k++) {
            if (w.member[k] >= 0) {
                const float a = area6(w.mb[k]);
                if (a > best) best = a, pick = k;
            }
        }
        if (pick < 0) break;
        const int y = w.member[pick];
        w.inner[ni++] = y;
        w.member[pick] = __ldcg(t.child_l + y);
        w.member[m] = __ldcg(t.child_r + y);
        ref_box32(t, w.member[pick], w.mb[pick]);
        ref_box32(t, w.member[m], w.mb[m]);
        m++;
    }
    w.m = m, w.ni = ni;
    if (m < 3) {
        float b[6];
        for (int q = 0; q < 6; q++) b[q] = __ldcg(t.nbox32 + 6 * x + q);
        __stcg(t.cost + x, area6(b) + ref_cost(t, w.member[0]) + ref_cost(t, w.member[1]));
        return;
    }
    for (int k = 0; k < m; k++) {
        w.mcost[k] = ref_cost(t, w.member[k]);
        w.mcount[k] = ref_count(t, w.member[k]);
        ref_box64(t, w.member[k], w.mb64[k]);
    }
    // current cost of the treelet: the old internal nodes' areas + members' costs
    float old_cost = 0.f;
    for (int k = 0; k < ni; k++) {
        float b[6];
        for (int q = 0; q < 6; q++) b[q] = __ldcg(t.nbox32 + 6 * w.inner[k] + q);
        old_cost += area6(b);
    }
    for (int k = 0; k < m; k++) old_cost += w.mcost[k];
    w.old_cost = old_cost;
}

// The whole warp: the best binary tree over the members, by dynamic programming over the member
// subsets in rounds of growing size (a round reads only smaller subsets). A round's subsets are listed
// in increasing order and dealt to groups of g lanes (g as large as the count allows: one lane per
// subset in the crowded rounds, 4 per subset for the 7 subsets of 6 members, all 32 for the full set);
// the lanes of a group search every g-th split of their subset in the sequential order, and the group
// keeps the cheapest split, the first in that order among equals -- the sequential search's choice.
__device__ void treelet_dp(TreeletWork &w, int lane) {
    constexpr unsigned kAll = 0xffffffffu;
    const int m = w.m, full = (1 << m) - 1;
    for (int s = 1 + lane; s <= full; s += 32)
        if ((s & (s - 1)) == 0) w.c[s] = w.mcost[__ffs(s) - 1], w.split[s] = 0;
    __syncwarp();
    for (int size = 2; size <= m; size++) {
        int nsub = 0;
        for (int base = 1; base <= full; base += 32) {
            const int s = base + lane;
            const bool in = s <= full && __popc(s) == size;
            const unsigned bal = __ballot_sync(kAll, in);
            if (in) w.subs[nsub + __popc(bal & ((1u << lane) - 1u))] = (unsigned char)s;
            nsub += __popc(bal);
        }
        __syncwarp();
        int g = 1;
        while (g * 2 * nsub <= 32) g *= 2;
        const int r = lane & (g - 1);
        for (int first = 0; first < nsub; first += 32 / g) {
            const int j = first + lane / g;
            const int s = j < nsub ? int(w.subs[j]) : 0;
            float best = FLT_MAX;
            int bp = 0, bk = 0x7fffffff;
            if (s) {
                // partitions (p, s \ p) with p holding the lowest member of s: each split once
                const int low = s & -s;
                int k = 0;
                for (int p = (s - 1) & s; p > 0; p = (p - 1) & s) {
                    if (!(p & low)) continue;
                    if ((k & (g - 1)) == r) {
                        const float v = w.c[p] + w.c[s ^ p];
                        if (v < best) best = v, bp = p, bk = k;
                    }
                    k++;
                }
            }
            for (int o = 1; o < g; o <<= 1) {
                const float ob = __shfl_xor_sync(kAll, best, o);
                const int obp = __shfl_xor_sync(kAll, bp, o), obk = __shfl_xor_sync(kAll, bk, o);
                if (ob < best || (ob == best && obk < bk)) best = ob, bp = obp, bk = obk;
            }
            if (s && r == 0) {
                float b[6] = {FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX};
                for (int k = 0; k < m; k++) {
                    if (!((s >> k) & 1)) continue;
                    for (int q = 0; q < 6; q += 2)
                        b[q] = fminf(b[q], w.mb[k][q]), b[q + 1] = fmaxf(b[q + 1], w.mb[k][q + 1]);
                }
                w.c[s] = area6(b) + best;
                w.split[s] = (unsigned char)bp;
            }
        }
        __syncwarp();
    }
}

// One lane: replaces the treelet's arrangement by the programme's when it is cheaper, reusing the
// treelet's internal nodes (the root keeps x): child and parent links top-down, and in w.onode /
// w.oset which members each reused node now covers (w.norder of them; 0 when the old arrangement
// stays, whose cost is stored here).
__device__ void rebuild_plan(const TreeArrays &t, int x, TreeletWork &w) {
    const int m = w.m, full = (1 << m) - 1;
    w.norder = 0;
    if (!(w.c[full] < w.old_cost * (1.f - 1e-6f))) {
        __stcg(t.cost + x, w.old_cost);
        return;
    }
    int stack_set[kTreeletLeaves], stack_node[kTreeletLeaves];
    int sp = 0, used = 1, norder = 0;
    stack_set[sp] = full, stack_node[sp] = x, sp++;
    while (sp > 0) {
        sp--;
        const int s = stack_set[sp], node = stack_node[sp];
        w.onode[norder] = node, w.oset[norder] = s, norder++;
        const int halves[2] = {w.split[s], s ^ w.split[s]};
        int refs[2];
        for (int h = 0; h < 2; h++) {
            const int hs = halves[h];
            if ((hs & (hs - 1)) == 0) {
                refs[h] = w.member[__ffs(hs) - 1];
            } else {
                refs[h] = w.inner[used++];
                stack_set[sp] = hs, stack_node[sp] = refs[h], sp++;
            }
        }
        __stcg(t.child_l + node, refs[0]);
        __stcg(t.child_r + node, refs[1]);
        set_parent(t, refs[0], node);
        set_parent(t, refs[1], node);
    }
    w.norder = norder;
}

// The whole warp, after rebuild_plan: lane k writes reused node w.onode[k]'s boxes (float and double),
// triangle count and cost. A node's box is the union of its members' boxes -- the same values the
// union of its two children's boxes gives, min and max being exact -- so no lane waits for another.
__device__ void rebuild_write(const TreeArrays &t, const TreeletWork &w, int lane) {
    if (lane >= w.norder) return;
    const int node = w.onode[lane], s = w.oset[lane];
    float b[6];
    double d[6];
    int cnt = 0;
    bool first = true;
    for (int j = 0; j < w.m; j++) {
        if (!((s >> j) & 1)) continue;
        for (int q = 0; q < 6; q += 2) {
            b[q] = first ? w.mb[j][q] : fminf(b[q], w.mb[j][q]);
            b[q + 1] = first ? w.mb[j][q + 1] : fmaxf(b[q + 1], w.mb[j][q + 1]);
            d[q] = first ? w.mb64[j][q] : fmin(d[q], w.mb64[j][q]);
            d[q + 1] = first ? w.mb64[j][q + 1] : fmax(d[q + 1], w.mb64[j][q + 1]);
        }
        cnt += w.mcount[j];
        first = false;
    }
    for (int q = 0; q < 6; q++) {
        __stcg(t.nbox32 + 6 * node + q, b[q]);
        __stcg(t.nbox64 + 6 * node + q, d[q]);
    }
    __stcg(t.count + node, cnt);
    __stcg(t.cost + node, w.c[s]);
    __threadfence();
}

constexpr int kTreeletThreads = 128;

// One thread per triangle climbs from its leaf; the second thread to reach a node owns it (its
// subtree is then final). Each round, the warp optimises its lanes' owned treelets one after the
// other, all 32 lanes sharing each one's dynamic programme. Lanes without work stay in the loop (the
// warp-wide votes need every lane) until the whole warp has climbed out.
__global__ void __launch_bounds__(kTreeletThreads) k_treelets(int n, TreeArrays t, int *arrivals) {
    __shared__ TreeletWork s_work[kTreeletThreads / 32];
    TreeletWork &w = s_work[threadIdx.x >> 5];
    constexpr unsigned kAll = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    int node = p < n ? __ldcg(t.parent_leaf + p) : -1;
    while (__any_sync(kAll, node >= 0)) {
        bool own = false;
        if (node >= 0) {
            __threadfence();
            if (atomicAdd(&arrivals[node], 1) == 0) {
                node = -1;  // the first arrival: the other child's thread continues
            } else {
                __threadfence();
                const int l = __ldcg(t.child_l + node), r = __ldcg(t.child_r + node);
                const int cnt = ref_count(t, l) + ref_count(t, r);
                __stcg(t.count + node, cnt);
                if (cnt >= kTreeletLeaves) {
                    own = true;
                } else {
                    float b[6];
                    for (int q = 0; q < 6; q++) b[q] = __ldcg(t.nbox32 + 6 * node + q);
                    __stcg(t.cost + node, area6(b) + ref_cost(t, l) + ref_cost(t, r));
                }
            }
        }
        unsigned todo = __ballot_sync(kAll, own);
        while (todo) {
            const int owner = __ffs(todo) - 1;
            todo &= todo - 1;
            const int x = __shfl_sync(kAll, node, owner);
            if (lane == owner) form_treelet(t, x, w);
            __syncwarp();
            if (w.m >= 3) {
                treelet_dp(w, lane);
                if (lane == owner) rebuild_plan(t, x, w);
                __syncwarp();
                rebuild_write(t, w, lane);
            }
            __syncwarp();
        }
        if (node >= 0) {
            __threadfence();
            node = __ldcg(t.parent_int + node);
        }
    }
}

// New leaf position of every triangle: its rank in a depth-first, left-first walk of the new tree,
// found by walking up and adding the sizes of left siblings.
__global__ void k_leaf_positions(int n, const int *__restrict__ child_l, const int *__restrict__ parent_int,
                                 const int *__restrict__ parent_leaf, const int *__restrict__ count,
                                 int *__restrict__ newpos) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int ref = -(p + 1);
    int node = parent_leaf[p];
    int off = 0;
    int guard = 0;
    while (node >= 0 && guard++ < (1 << 20)) {
        const int l = child_l[node];
        if (l != ref) off += l >= 0 ? count[l] : 1;
        ref = node;
        node = parent_int[node];
    }
    newpos[p] = off;
}

__global__ void k_relabel(int n, const int *__restrict__ newpos, const int *__restrict__ ids_old,
                          const int *__restrict__ parent_leaf_old, const int *__restrict__ child_l_old,
                          const int *__restrict__ child_r_old, int *__restrict__ ids_new,
                          int *__restrict__ parent_leaf_new, int *__restrict__ child_l_new,
                          int *__restrict__ child_r_new) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int q = newpos[p];
    ids_new[q] = ids_old[p];
    const int parent = parent_leaf_old[p];
    parent_leaf_new[q] = parent;
    if (child_l_old[parent] == -(p + 1)) child_l_new[parent] = -(q + 1);
    if (child_r_old[parent] == -(p + 1)) child_r_new[parent] = -(q + 1);
}

// first_of: leaf position of the leftmost triangle below each internal node.
__global__ void k_first_of(int nint, const int *__restrict__ child_l, int *__restrict__ first_of) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nint) return;
    int ref = i;
    int guard = 0;
    while (ref >= 0 && guard++ < (1 << 20)) ref = child_l[ref];
    first_of[i] = -ref - 1;
}

}  // namespace

int treelet_optimize(int n, int *child_l, int *child_r, int *parent_int, int *parent_leaf, int *first_of,
                     float *nbox32, double *nbox64, const float *pbox32, const double *pbox64, int *sorted_ids,
                     cudaStream_t stream) {
    const int nint = n - 1;
    if (nint < kTreeletLeaves) return SSDF_OK;
    float *cost = nullptr;
    int *count = nullptr, *arrivals = nullptr, *newpos = nullptr, *ids2 = nullptr, *pl2 = nullptr, *cl2 = nullptr,
        *cr2 = nullptr;
    int st = SSDF_OK;
    auto alloc = [&](void **p, size_t b) {
        if (st == SSDF_OK && cudaMallocAsync(p, b, stream) != cudaSuccess) st = fail(SSDF_ERR_OUT_OF_MEMORY, "treelet scratch");
    };
    alloc((void **)&cost, sizeof(float) * nint);
    alloc((void **)&count, sizeof(int) * nint);
    alloc((void **)&arrivals, sizeof(int) * nint);
    alloc((void **)&newpos, sizeof(int) * n);
    alloc((void **)&ids2, sizeof(int) * n);
    alloc((void **)&pl2, sizeof(int) * n);
    alloc((void **)&cl2, sizeof(int) * nint);
    alloc((void **)&cr2, sizeof(int) * nint);
    cudaError_t e = cudaSuccess;
    if (st == SSDF_OK) {
        TreeArrays t{child_l, child_r, parent_int, parent_leaf, nbox32, nbox64, pbox32, pbox64, sorted_ids, cost, count};
        e = cudaMemsetAsync(arrivals, 0, sizeof(int) * nint, stream);
        if (e == cudaSuccess) {
            k_treelets<<<grid_blocks(n, kTreeletThreads), kTreeletThreads, 0, stream>>>(n, t, arrivals);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) {
            k_leaf_positions<<<grid_blocks(n, 256), 256, 0, stream>>>(n, child_l, parent_int, parent_leaf, count,
                                                                       newpos);
            e = cudaMemcpyAsync(cl2, child_l, sizeof(int) * nint, cudaMemcpyDeviceToDevice, stream);
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(cr2, child_r, sizeof(int) * nint, cudaMemcpyDeviceToDevice, stream);
        if (e == cudaSuccess) {
            k_relabel<<<grid_blocks(n, 256), 256, 0, stream>>>(n, newpos, sorted_ids, parent_leaf, child_l, child_r, ids2,
                                                                pl2, cl2, cr2);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(sorted_ids, ids2, sizeof(int) * n, cudaMemcpyDeviceToDevice, stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(parent_leaf, pl2, sizeof(int) * n, cudaMemcpyDeviceToDevice, stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(child_l, cl2, sizeof(int) * nint, cudaMemcpyDeviceToDevice, stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(child_r, cr2, sizeof(int) * nint, cudaMemcpyDeviceToDevice, stream);
        if (e == cudaSuccess) {
            k_first_of<<<grid_blocks(nint, 256), 256, 0, stream>>>(nint, child_l, first_of);
            e = cudaGetLastError();
        }
        if (e != cudaSuccess) st = cuda_fail(e, "treelet refinement", __FILE__, __LINE__);
    }
    for (void *p : {(void *)cost, (void *)count, (void *)arrivals, (void *)newpos, (void *)ids2, (void *)pl2,
                    (void *)cl2, (void *)cr2})
        if (p) cudaFreeAsync(p, stream);
    return st;
}

}  // namespace ssdf_b200
