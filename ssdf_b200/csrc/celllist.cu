// celllist.cu -- ssdf::edf_celllist on the GPU.
//
// Same structure as the reference (serial/ssdf.hpp:642-963): a 2-D grid of cells over the two
// widest axes of the triangles' bounding box, cell size = the largest triangle extent, triangles
// binned by the centre of their box and, inside a cell, sorted by their minimum on the third axis
// with a running maximum of their maximum, so a sweep from the point's position can stop early.
// The reference then tests every cell for every point (serial/ssdf.hpp:938-956); here each point
// visits cells in square rings around its own cell and stops once a ring's lower bound,
// (r - 2) * cell_size, exceeds its current best -- a triangle binned in a cell lies within half a
// cell of it. All tests keep ties (relative and absolute margins), so the value is the
// brute-force minimum: bitwise the reference's in T's arithmetic, closest triangle the lowest
// index at the minimum.
// The device build: boxes + bounds (reduction), cell keys (cell << 32 | float min, rounded down),
// one stable radix sort, per-cell ranges, boxes and running maxima.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "device_geom.cuh"
#include "internal.h"

namespace ssdf_b200 {

namespace {

constexpr int kRec = 16;  // vertices (9), box (6), padding
constexpr long long kMaxCells = 1 << 22;

__device__ __forceinline__ unsigned long long d2o(double v) {
    const long long i = __double_as_longlong(v);
    return (unsigned long long)(i >= 0 ? (i ^ (1ll << 63)) : ~i);
}
inline double o2d_host(unsigned long long o) {
    const long long i = (o >> 63) ? (long long)(o ^ (1ull << 63)) : (long long)~o;
    double d;
    memcpy(&d, &i, sizeof(d));
    return d;
}
__device__ __forceinline__ uint32_t f2key(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u >> 31) ? ~u : (u | 0x80000000u);
}

// Boxes, validation, bounds: red[0..2] min, red[3..5] max (ordered u64 of the double value),
// red[6] max extent.
template <typename T>
__global__ void k_cl_boxes(int nt, int nv, const int *__restrict__ s0, const int *__restrict__ s1,
                           const int *__restrict__ s2, const T *__restrict__ sx, const T *__restrict__ sy,
                           const T *__restrict__ sz, T *__restrict__ box, unsigned long long *__restrict__ red,
                           int *__restrict__ err) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX}, ext = 0.0;
    if (t < nt) {
        const int id[3] = {s0[t], s1[t], s2[t]};
        if (id[0] < 0 || id[0] >= nv || id[1] < 0 || id[1] >= nv || id[2] < 0 || id[2] >= nv) {
            atomicMin(err, t);
        } else {
            const T *c[3] = {sx, sy, sz};
            for (int d = 0; d < 3; d++) {
                const T a = c[d][id[0]], b = c[d][id[1]], e = c[d][id[2]];
                const T l = fmin(fmin(a, b), e), h = fmax(fmax(a, b), e);
                box[6 * t + 2 * d] = l;
                box[6 * t + 2 * d + 1] = h;
                lo[d] = double(l), hi[d] = double(h);
                ext = fmax(ext, double(h - l));
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        for (int d = 0; d < 3; d++) {
            lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
            hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
        }
        ext = fmax(ext, __shfl_xor_sync(0xffffffffu, ext, o));
    }
    if ((threadIdx.x & 31) == 0) {
        for (int d = 0; d < 3; d++) {
            atomicMin(&red[d], d2o(lo[d]));
            atomicMax(&red[3 + d], d2o(hi[d]));
        }
        atomicMax(&red[6], d2o(ext));
    }
}

struct CellGrid {
    int axis0, axis1, sort_axis;
    int n0, n1;
    double min0, min1, cs;
};

template <typename T>
__global__ void k_cl_keys(int nt, const T *__restrict__ box, CellGrid g, uint64_t *__restrict__ keys,
                          int *__restrict__ vals) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const T *b = box + 6 * t;
    const double c0 = 0.5 * (double(b[2 * g.axis0]) + double(b[2 * g.axis0 + 1]));
    const double c1 = 0.5 * (double(b[2 * g.axis1]) + double(b[2 * g.axis1 + 1]));
    int i0 = int(floor((c0 - g.min0) / g.cs)), i1 = int(floor((c1 - g.min1) / g.cs));
    i0 = max(0, min(i0, g.n0 - 1));
    i1 = max(0, min(i1, g.n1 - 1));
    const unsigned long long cell = (unsigned long long)i1 * g.n0 + i0;
    const float mn = __double2float_rd(double(b[2 * g.sort_axis]));
    keys[t] = (cell << 32) | f2key(mn);
    vals[t] = t;
}

template <typename T>
__global__ void k_cl_records(int nt, const int *__restrict__ ids, const uint64_t *__restrict__ keys,
                             const int *__restrict__ s0, const int *__restrict__ s1, const int *__restrict__ s2,
                             const T *__restrict__ sx, const T *__restrict__ sy, const T *__restrict__ sz,
                             const T *__restrict__ box, int sort_axis, T *__restrict__ rec, int *__restrict__ rid,
                             float *__restrict__ smin, float *__restrict__ smax, int *__restrict__ cell_start,
                             int *__restrict__ cell_end) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nt) return;
    const int t = ids[p];
    T *r = rec + size_t(kRec) * p;
    const int id[3] = {s0[t], s1[t], s2[t]};
    for (int v = 0; v < 3; v++) {
        r[3 * v] = sx[id[v]];
        r[3 * v + 1] = sy[id[v]];
        r[3 * v + 2] = sz[id[v]];
    }
    for (int k = 0; k < 6; k++) r[9 + k] = box[6 * t + k];
    r[15] = T(0);
    rid[p] = t;
    smin[p] = __double2float_rd(double(box[6 * t + 2 * sort_axis]));
    smax[p] = __double2float_ru(double(box[6 * t + 2 * sort_axis + 1]));
    const unsigned cell = unsigned(keys[p] >> 32);
    if (p == 0 || unsigned(keys[p - 1] >> 32) != cell) cell_start[cell] = p;
    if (p == nt - 1 || unsigned(keys[p + 1] >> 32) != cell) cell_end[cell] = p + 1;
}

// Per cell: union box and the running maximum of the sort-axis maxima (overwrites smax).
template <typename T>
__global__ void k_cl_cells(int ncells, const int *__restrict__ cell_start, const int *__restrict__ cell_end,
                           const T *__restrict__ rec, float *__restrict__ smax, T *__restrict__ cbox) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    const int b = cell_start[c], e = cell_end[c];
    T bx[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
    if (e > b) {
        for (int k = 0; k < 6; k++) bx[k] = rec[size_t(kRec) * b + 9 + k];
        float run = smax[b];
        for (int p = b; p < e; p++) {
            const T *r = rec + size_t(kRec) * p + 9;
            for (int k = 0; k < 6; k += 2) bx[k] = fmin(bx[k], r[k]), bx[k + 1] = fmax(bx[k + 1], r[k + 1]);
            run = fmaxf(run, smax[p]);
            smax[p] = run;
        }
    }
    for (int k = 0; k < 6; k++) cbox[6 * c + k] = bx[k];
}

template <typename T>
__device__ __forceinline__ T cl_abs_margin(float scale);
template <>
__device__ __forceinline__ double cl_abs_margin<double>(float scale) {
    const double s = double(scale) * 0x1p-40;
    return s * s;
}
template <>
__device__ __forceinline__ float cl_abs_margin<float>(float scale) {
    const float s = scale * 0x1p-16f;
    return s * s;
}

// COUNT: the counting instantiation (Ericson tests, and box tests of cells and triangles, into
// counters[0..1]).
// Bounded to 5 resident blocks per SM (94 registers in double). The kernel is latency bound with its
// loads served by L1 (96 % hits, ncu), but trading registers for occupancy loses: on the 64^3
// icosphere grid 3.47 ms at 5 blocks, 3.48 unbounded (102 registers), 3.63 at 6 (80), 3.97 at 7
// (72, spills) and 3.80 at 8 (64, spills).
#ifndef SSDF_B200_CL_MIN_BLOCKS
#define SSDF_B200_CL_MIN_BLOCKS 5
#endif
template <typename T, bool COUNT>
__global__ void __launch_bounds__(128, SSDF_B200_CL_MIN_BLOCKS) k_cl_query(int npoints, const T *__restrict__ x, const T *__restrict__ y,
                                                  const T *__restrict__ z, CellGrid g, float scale,
                                                  const int *__restrict__ cell_start, const int *__restrict__ cell_end,
                                                  const T *__restrict__ cbox, const T *__restrict__ rec,
                                                  const int *__restrict__ rid, const float *__restrict__ smin, const float *__restrict__ smax,
                                                  T *__restrict__ out, int *__restrict__ outtri,
                                                  unsigned long long *__restrict__ counters) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npoints) return;
    unsigned long long n_tri = 0, n_box = 0;
    const T px = x[q], py = y[q], pz = z[q];
    const T o = out[q];
    T best = o * o;
    int bid = -1;
    const T rel = T(1) + T(1) / T(65536), margin = cl_abs_margin<T>(scale);
    T thr = best * rel + margin;
    const T p3[3] = {px, py, pz};
    const double u0 = double(p3[g.axis0]), u1 = double(p3[g.axis1]);
    const double pc = double(p3[g.sort_axis]);
    double f0 = floor((u0 - g.min0) / g.cs), f1 = floor((u1 - g.min1) / g.cs);
    f0 = fmin(fmax(f0, 0.0), double(g.n0 - 1));
    f1 = fmin(fmax(f1, 0.0), double(g.n1 - 1));
    const int c0 = (f0 == f0) ? int(f0) : 0, c1 = (f1 == f1) ? int(f1) : 0;
    const int rmax = max(g.n0, g.n1);
    for (int r = 0; r <= rmax; r++) {
        if (r >= 2) {
            const T lb = T(double(r - 2) * g.cs);
            if (lb * lb > thr) break;
        }
        const int i_lo = c0 - r, i_hi = c0 + r, j_lo = c1 - r, j_hi = c1 + r;
        // ring cells: rows j_lo / j_hi over [i_lo, i_hi], columns i_lo / i_hi over (j_lo, j_hi)
        const int nring = r == 0 ? 1 : 8 * r;
        for (int s = 0; s < nring; s++) {
            int i, j;
            if (r == 0) {
                i = c0, j = c1;
            } else if (s < 2 * r + 1) {
                i = i_lo + s, j = j_lo;
            } else if (s < 4 * r + 2) {
                i = i_lo + (s - 2 * r - 1), j = j_hi;
            } else if (s < 6 * r + 1) {
                i = i_lo, j = j_lo + 1 + (s - 4 * r - 2);
            } else {
                i = i_hi, j = j_lo + 1 + (s - 6 * r - 1);
            }
            if (i < 0 || i >= g.n0 || j < 0 || j >= g.n1) continue;
            const int c = j * g.n0 + i;
            const int b = __ldg(cell_start + c), e = __ldg(cell_end + c);
            if (e <= b) continue;
            const T *cb = cbox + 6 * c;
            if (COUNT) n_box++;
            if (!(box_dist_sq<T>(px, py, pz, __ldg(cb), __ldg(cb + 1), __ldg(cb + 2), __ldg(cb + 3), __ldg(cb + 4),
                                 __ldg(cb + 5)) < thr))
                continue;
            // lower_bound of pc in the cell's sorted minima
            int lo = b, hi = e;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (double(__ldg(smin + mid)) < pc) lo = mid + 1; else hi = mid;
            }
            auto eval = [&](int p) {
                const T *rr = rec + size_t(kRec) * p;
                if (COUNT) n_box++;
                if (!(box_dist_sq<T>(px, py, pz, __ldg(rr + 9), __ldg(rr + 10), __ldg(rr + 11), __ldg(rr + 12),
                                     __ldg(rr + 13), __ldg(rr + 14)) < thr))
                    return;
                if (COUNT) n_tri++;
                const T d2 = tri_dist_sq_exact<T>(px, py, pz, __ldg(rr), __ldg(rr + 1), __ldg(rr + 2), __ldg(rr + 3),
                                                  __ldg(rr + 4), __ldg(rr + 5), __ldg(rr + 6), __ldg(rr + 7),
                                                  __ldg(rr + 8));
                const int id = __ldg(rid + p);
                if (d2 < best || (d2 == best && bid >= 0 && id < bid)) {
                    best = d2;
                    bid = id;
                    thr = best * rel + margin;
                }
            };
            for (int p = lo - 1; p >= b; p--) {
                const double mg = pc - double(__ldg(smax + p));
                if (mg >= 0.0 && T(mg) * T(mg) > thr) break;
                eval(p);
            }
            for (int p = lo; p < e; p++) {
                const double mg = double(__ldg(smin + p)) - pc;
                if (mg >= 0.0 && T(mg) * T(mg) > thr) break;
                eval(p);
            }
        }
    }
    out[q] = sqrt(best);
    if (outtri && bid >= 0) outtri[q] = bid;
    if (COUNT) {  // untimed: one atomic per thread (the last warp may be partial)
        atomicAdd(counters, n_tri);
        atomicAdd(counters + 1, n_box);
    }
}

int bits_for(unsigned long long v) {
    int b = 1;
    while (b < 64 && (v >> b) != 0) b++;
    return b;
}

template <typename T>
int celllist_impl(ptrdiff_t npoints, const T *x, const T *y, const T *z, ptrdiff_t nt_, const int *s0, const int *s1,
                  const int *s2, ptrdiff_t nv, const T *sx, const T *sy, const T *sz, T *out, int *outtri,
                  cudaStream_t stream) {
    const int nt = int(nt_);
    std::vector<void *> tmp;
    auto alloc = [&](void **p, size_t bytes) -> int {
        cudaError_t e = cudaMallocAsync(p, bytes ? bytes : 16, stream);
        if (e != cudaSuccess) return fail(SSDF_ERR_OUT_OF_MEMORY, "cell list scratch");
        tmp.push_back(*p);
        return SSDF_OK;
    };
    auto release = [&]() {
        for (void *p : tmp) cudaFreeAsync(p, stream);
    };
    T *box;
    unsigned long long *red;
    int *err;
    int st = SSDF_OK;
    if ((st = alloc((void **)&box, sizeof(T) * 6 * size_t(nt))) != SSDF_OK ||
        (st = alloc((void **)&red, sizeof(unsigned long long) * 8)) != SSDF_OK ||
        (st = alloc((void **)&err, sizeof(int) * 4)) != SSDF_OK) {
        release();
        return st;
    }
    // seeds: +max for the minima, -max for the maxima and 0 for the extent (ordered encodings)
    unsigned long long hred[8];
    auto enc = [](double v) {
        long long i;
        memcpy(&i, &v, sizeof(i));
        return (unsigned long long)(i >= 0 ? (i ^ (1ll << 63)) : ~i);
    };
    for (int d = 0; d < 3; d++) hred[d] = enc(DBL_MAX), hred[3 + d] = enc(-DBL_MAX);
    hred[6] = enc(0.0);
    hred[7] = 0;
    const int herr[4] = {0x7fffffff, 0, 0, 0};
    unsigned long long *counters = nullptr;  // the counting instantiation's (SSDF_B200_COUNT)
    cudaError_t e = cudaMemcpyAsync(red, hred, sizeof(hred), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(err, herr, sizeof(herr), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) {
        k_cl_boxes<T><<<grid_blocks(nt, 256), 256, 0, stream>>>(nt, int(nv), s0, s1, s2, sx, sy, sz, box, red, err);
        e = cudaGetLastError();
    }
    int herr2[4];
    if (e == cudaSuccess) e = cudaMemcpyAsync(hred, red, sizeof(hred), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(herr2, err, sizeof(herr2), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        release();
        return cuda_fail(e, "cell list bounds", __FILE__, __LINE__);
    }
    if (herr2[0] != 0x7fffffff) {
        release();
        return fail(SSDF_ERR_INVALID_ARGUMENT, "triangle " + std::to_string(herr2[0]) + " has a vertex index out of range");
    }
    // grid axes and cell size, as serial/ssdf.hpp:725-767 chooses them
    double gmin[3], gmax[3];
    for (int d = 0; d < 3; d++) gmin[d] = o2d_host(hred[d]), gmax[d] = o2d_host(hred[3 + d]);
    const double max_extent = o2d_host(hred[6]);
    const T span_x = T(gmax[0]) - T(gmin[0]), span_y = T(gmax[1]) - T(gmin[1]), span_z = T(gmax[2]) - T(gmin[2]);
    CellGrid g;
    if (span_x >= span_y && span_x >= span_z) {
        g.axis0 = 0;
        if (span_y >= span_z) g.axis1 = 1, g.sort_axis = 2; else g.axis1 = 2, g.sort_axis = 1;
    } else if (span_y >= span_x && span_y >= span_z) {
        g.axis0 = 1;
        if (span_x >= span_z) g.axis1 = 0, g.sort_axis = 2; else g.axis1 = 2, g.sort_axis = 0;
    } else {
        g.axis0 = 2;
        if (span_x >= span_y) g.axis1 = 0, g.sort_axis = 1; else g.axis1 = 1, g.sort_axis = 0;
    }
    const double spans[3] = {double(span_x), double(span_y), double(span_z)};
    double cs = std::max(max_extent, 1e-8);
    // cap the number of cells (the result does not depend on the cell size)
    while (std::ceil(spans[g.axis0] / cs) * std::ceil(spans[g.axis1] / cs) > double(kMaxCells)) cs *= 2.0;
    g.cs = cs;
    g.min0 = gmin[g.axis0];
    g.min1 = gmin[g.axis1];
    g.n0 = std::max(1, int(std::ceil(spans[g.axis0] / cs)));
    g.n1 = std::max(1, int(std::ceil(spans[g.axis1] / cs)));
    const long long ncells = (long long)g.n0 * g.n1;
    uint64_t *keys;
    int *ids, *cstart, *cend, *rid;
    T *rec, *cbox;
    float *smin, *smax;
    if ((st = alloc((void **)&keys, sizeof(uint64_t) * nt)) != SSDF_OK ||
        (st = alloc((void **)&ids, sizeof(int) * nt)) != SSDF_OK ||
        (st = alloc((void **)&cstart, sizeof(int) * ncells)) != SSDF_OK ||
        (st = alloc((void **)&cend, sizeof(int) * ncells)) != SSDF_OK ||
        (st = alloc((void **)&rec, sizeof(T) * kRec * size_t(nt))) != SSDF_OK ||
        (st = alloc((void **)&rid, sizeof(int) * size_t(nt))) != SSDF_OK ||
        (st = alloc((void **)&cbox, sizeof(T) * 6 * size_t(ncells))) != SSDF_OK ||
        (st = alloc((void **)&smin, sizeof(float) * nt)) != SSDF_OK ||
        (st = alloc((void **)&smax, sizeof(float) * nt)) != SSDF_OK) {
        release();
        return st;
    }
    k_cl_keys<T><<<grid_blocks(nt, 256), 256, 0, stream>>>(nt, box, g, keys, ids);
    e = cudaGetLastError();
    if (e == cudaSuccess) {
        st = radix_sort_pairs_u64(keys, ids, nt, 32 + bits_for((unsigned long long)ncells), stream);
    }
    if (e == cudaSuccess && st == SSDF_OK) e = cudaMemsetAsync(cstart, 0, sizeof(int) * ncells, stream);
    if (e == cudaSuccess && st == SSDF_OK) e = cudaMemsetAsync(cend, 0, sizeof(int) * ncells, stream);
    if (e == cudaSuccess && st == SSDF_OK) {
        k_cl_records<T><<<grid_blocks(nt, 256), 256, 0, stream>>>(nt, ids, keys, s0, s1, s2, sx, sy, sz, box,
                                                                 g.sort_axis, rec, rid, smin, smax, cstart, cend);
        k_cl_cells<T><<<grid_blocks(ncells, 128), 128, 0, stream>>>(int(ncells), cstart, cend, rec, smax, cbox);
        const double scale = std::max({std::fabs(gmin[0]), std::fabs(gmin[1]), std::fabs(gmin[2]),
                                       std::fabs(gmax[0]), std::fabs(gmax[1]), std::fabs(gmax[2])});
        const bool count = env_int("SSDF_B200_COUNT", 0) != 0;
        if (count) {
            e = cudaMallocAsync(&counters, 2 * sizeof(unsigned long long), stream);
            if (e == cudaSuccess) e = cudaMemsetAsync(counters, 0, 2 * sizeof(unsigned long long), stream);
        }
        if (e == cudaSuccess) {
            if (count)
                k_cl_query<T, true><<<grid_blocks(npoints, 128), 128, 0, stream>>>(
                    int(npoints), x, y, z, g, float(scale), cstart, cend, cbox, rec, rid, smin, smax, out, outtri,
                    counters);
            else
                k_cl_query<T, false><<<grid_blocks(npoints, 128), 128, 0, stream>>>(
                    int(npoints), x, y, z, g, float(scale), cstart, cend, cbox, rec, rid, smin, smax, out, outtri,
                    counters);
            e = cudaGetLastError();
        }
    }
    unsigned long long hc[2] = {0, 0};
    if (e == cudaSuccess && st == SSDF_OK && counters)
        e = cudaMemcpyAsync(hc, counters, sizeof(hc), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && st == SSDF_OK) e = cudaStreamSynchronize(stream);
    if (counters) {
        cudaFreeAsync(counters, stream);
        if (e == cudaSuccess && st == SSDF_OK) set_last_counts(hc[0], hc[1], 0, 0);
    }
    if (e != cudaSuccess && st == SSDF_OK) st = cuda_fail(e, "cell list edf", __FILE__, __LINE__);
    release();
    return st;
}

}  // namespace

int celllist_edf(int f64, ptrdiff_t npoints, const void *x, const void *y, const void *z, ptrdiff_t nt,
                 const int *s0, const int *s1, const int *s2, ptrdiff_t nv, const void *sx, const void *sy,
                 const void *sz, void *out, int *outtri, cudaStream_t stream) {
    if (npoints <= 0 || nt <= 0 || nv <= 0) return SSDF_OK;
    if (npoints > 0x7fffffff || nt > kMaxTriangles)
        return fail(SSDF_ERR_NOT_SUPPORTED, "cell-list edf: too many points or triangles for one launch");
    if (f64)
        return celllist_impl<double>(npoints, (const double *)x, (const double *)y, (const double *)z, nt, s0, s1, s2,
                                     nv, (const double *)sx, (const double *)sy, (const double *)sz, (double *)out,
                                     outtri, stream);
    return celllist_impl<float>(npoints, (const float *)x, (const float *)y, (const float *)z, nt, s0, s1, s2, nv,
                                (const float *)sx, (const float *)sy, (const float *)sz, (float *)out, outtri, stream);
}

}  // namespace ssdf_b200
