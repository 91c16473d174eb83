// sdf_rebuild.cu -- signed distance to the level set of a sampled field, on the device: marching
// tetrahedra, the BVH of the triangles, a banded closest-point query (serial/bvh/sdf_rebuild.cpp,
// serial/bvh/sdf_rebuild.hpp:23-78), cubic refinement of a field, and the rounding of a region's
// edges by an opening and a closing made of such rebuilds.
//
// Marching tetrahedra (level_set_triangles, serial/bvh/sdf_rebuild.cpp:13-118,190-250): a cell is
// cut into the six tetrahedra about its corner-0-to-corner-7 diagonal, so neighbouring cells cut
// their shared face alike; an edge crossing is interpolated from its corner of lower grid index, so
// every cell on the edge finds the same point; triangles with two vertices equal after rounding to
// G are dropped. One thread per cell counts, a scan places each cell's triangles, and the same
// thread emits them: the triangles come out in the reference's order (cells x fastest, then y,
// then z; tetrahedra and triangles in order within a cell), each vertex bitwise its value (double
// arithmetic in the reference's expression order, the library being built without contraction).
//
// The rebuild's query is the library's fix-up query in double over those triangles, started from
// the band as an in/out bound, so a sample farther than the band gets the band. Samples whose
// |f - level| is at least the band are not searched (the field is 1-Lipschitz); the sign is that of
// f - level, zero on the level set (serial/bvh/sdf_rebuild.cpp:252-299). The reference searches
// with cuBQL in float from the float-rounded sample; this returns the distance in double from the
// sample itself.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "internal.h"

namespace ssdf_b200 {

namespace {

constexpr int kThreadsR = 128;

// The six tetrahedra of a cell about its diagonal from corner 0 to corner 7; corner c sits at
// (c & 1, (c >> 1) & 1, (c >> 2) & 1) in cell units.
__constant__ int c_tets[6][4] = {{0, 1, 3, 7}, {0, 1, 5, 7}, {0, 2, 3, 7}, {0, 2, 6, 7}, {0, 4, 5, 7}, {0, 4, 6, 7}};

struct CellValues {
    long long g[8];    // grid index of each corner
    double v[8];       // value less the level
    double p[8][3];    // position
};

template <typename T>
__device__ bool load_corners(const GridDesc &gd, const T *__restrict__ f, double level, long long i, long long j,
                             long long k, CellValues &c) {
    const long long sy = gd.n[0], sz = gd.n[0] * gd.n[1];
    int above = 0;
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const long long ci = i + (q & 1), cj = j + ((q >> 1) & 1), ck = k + ((q >> 2) & 1);
        c.g[q] = ci + cj * sy + ck * sz;
        c.v[q] = double(f[c.g[q]]) - level;
        above += c.v[q] > 0 ? 1 : 0;
    }
    if (above == 0 || above == 8) return false;
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const long long ijk[3] = {i + (q & 1), j + ((q >> 1) & 1), k + ((q >> 2) & 1)};
#pragma unroll
        for (int d = 0; d < 3; d++) c.p[q][d] = gd.o[d] + double(ijk[d]) * gd.h[d];
    }
    return true;
}

// The level crossing on the edge between corners a and b, interpolated from the corner of lower grid
// index.
__device__ void edge_crossing(const CellValues &c, int a, int b, double q[3]) {
    if (c.g[b] < c.g[a]) {
        const int s = a;
        a = b;
        b = s;
    }
    const double t = c.v[a] / (c.v[a] - c.v[b]);
#pragma unroll
    for (int d = 0; d < 3; d++) q[d] = c.p[a][d] + t * (c.p[b][d] - c.p[a][d]);
}

// The 0, 1 or 2 triangles of tetrahedron tet, degenerate ones (two vertices equal in G) dropped.
template <typename G>
__device__ int tet_triangles(const CellValues &c, int tet, double tri[2][3][3]) {
    int up[4], down[4], nu = 0, nd = 0;
    for (int a = 0; a < 4; a++) {
        const int q = c_tets[tet][a];
        if (c.v[q] > 0)
            up[nu++] = q;
        else
            down[nd++] = q;
    }
    if (nu == 0 || nd == 0) return 0;
    int m;
    if (nu == 1 || nd == 1) {
        // one corner apart: the triangle on its three edges
        const int lone = nu == 1 ? up[0] : down[0];
        const int *others = nu == 1 ? down : up;
        for (int a = 0; a < 3; a++) edge_crossing(c, lone, others[a], tri[0][a]);
        m = 1;
    } else {
        // two and two: the quadrilateral on the four edges between them, as triangles (0,1,2), (0,2,3)
        double q[4][3];
        edge_crossing(c, up[0], down[0], q[0]);
        edge_crossing(c, up[0], down[1], q[1]);
        edge_crossing(c, up[1], down[1], q[2]);
        edge_crossing(c, up[1], down[0], q[3]);
        const int quad[2][3] = {{0, 1, 2}, {0, 2, 3}};
        for (int s = 0; s < 2; s++)
            for (int a = 0; a < 3; a++)
                for (int d = 0; d < 3; d++) tri[s][a][d] = q[quad[s][a]][d];
        m = 2;
    }
    int kept = 0;
    for (int s = 0; s < m; s++) {
        bool degenerate = false;
        for (int a = 0; a < 3; a++) {
            const int b = (a + 1) % 3;
            degenerate |= G(tri[s][a][0]) == G(tri[s][b][0]) && G(tri[s][a][1]) == G(tri[s][b][1]) &&
                          G(tri[s][a][2]) == G(tri[s][b][2]);
        }
        if (degenerate) continue;
        if (kept != s)
            for (int a = 0; a < 3; a++)
                for (int d = 0; d < 3; d++) tri[kept][a][d] = tri[s][a][d];
        kept++;
    }
    return kept;
}

// One thread per cell: its triangle count (EMIT false) or its triangles at offset[cell] (EMIT true).
template <typename G, typename T, bool EMIT>
__global__ void __launch_bounds__(kThreadsR) k_marching(GridDesc gd, const T *__restrict__ f, double level,
                                                        long long ncells, int *__restrict__ count,
                                                        const int *__restrict__ offset, G *__restrict__ x,
                                                        G *__restrict__ y, G *__restrict__ z) {
    const long long cell = blockIdx.x * (long long)kThreadsR + threadIdx.x;
    if (cell >= ncells) return;
    const long long cx = gd.n[0] - 1, cy = gd.n[1] - 1;
    const long long i = cell % cx, r = cell / cx, j = r % cy, k = r / cy;
    CellValues c;
    if (!load_corners(gd, f, level, i, j, k, c)) {
        if (!EMIT) count[cell] = 0;
        return;
    }
    long long next = EMIT ? offset[cell] : 0;
    int total = 0;
    for (int t = 0; t < 6; t++) {
        double tri[2][3][3];
        const int m = tet_triangles<G>(c, t, tri);
        if (EMIT) {
            for (int s = 0; s < m; s++, next++)
                for (int a = 0; a < 3; a++) {
                    x[3 * next + a] = G(tri[s][a][0]);
                    y[3 * next + a] = G(tri[s][a][1]);
                    z[3 * next + a] = G(tri[s][a][2]);
                }
        }
        total += m;
    }
    if (!EMIT) count[cell] = total;
}

__global__ void k_soup_indices(long long n, int *__restrict__ s0, int *__restrict__ s1, int *__restrict__ s2) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    s0[t] = int(3 * t), s1[t] = int(3 * t + 1), s2[t] = int(3 * t + 2);
}

// Per strided sample: the query's in/out start (the band where searched, 0 elsewhere).
template <typename T>
__global__ void k_band_start(GridDesc gd, long long stride, GridDesc og, const T *__restrict__ f, T level, T band,
                             int searched, T *__restrict__ out) {
    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long n = og.n[0] * og.n[1] * og.n[2];
    if (p >= n) return;
    const long long i = p % og.n[0], r = p / og.n[0], j = r % og.n[1], k = r / og.n[1];
    const T v = f[stride * (i + j * gd.n[0] + k * gd.n[0] * gd.n[1])] - level;
    out[p] = (searched && fabs(double(v)) < double(band)) ? band : T(0);
}

// d = the searched distance (at most the band) or the band; out = sign(f - level) * d, 0 on the set.
template <typename T>
__global__ void k_band_sign(GridDesc gd, long long stride, GridDesc og, const T *__restrict__ f, T level, T band,
                            int searched, T *__restrict__ out) {
    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long n = og.n[0] * og.n[1] * og.n[2];
    if (p >= n) return;
    const long long i = p % og.n[0], r = p / og.n[0], j = r % og.n[1], k = r / og.n[1];
    const T v = f[stride * (i + j * gd.n[0] + k * gd.n[0] * gd.n[1])] - level;
    const T d = (searched && fabs(double(v)) < double(band)) ? out[p] : band;
    out[p] = v > T(0) ? d : (v < T(0) ? -d : T(0));
}

template <typename T>
__global__ void k_shift(long long n, T *__restrict__ v, T s) {
    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p < n) v[p] += s;
}

// refine_field: coarse samples to multiples of factor, then per axis the cubic through the four
// nearest samples (the end samples repeated), weights w[4 m + q] for t = m / factor.
template <typename T>
__global__ void k_refine_place(GridDesc gd, long long factor, long long fx, long long fxy, const T *__restrict__ f,
                               T *__restrict__ fine) {
    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long n = gd.n[0] * gd.n[1] * gd.n[2];
    if (p >= n) return;
    const long long i = p % gd.n[0], r = p / gd.n[0], j = r % gd.n[1], k = r / gd.n[1];
    fine[i * factor + fx * (j * factor) + fxy * (k * factor)] = f[p];
}

template <typename T>
__global__ void k_refine_axis(long long n1, long long n2, long long n, long long factor, long long stride,
                              long long step1, long long step2, const double *__restrict__ w, T *__restrict__ fine) {
    const long long item = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long per_line = (n - 1) * (factor - 1);
    if (item >= n1 * n2 * per_line) return;
    const long long line_id = item / per_line, rest = item % per_line;
    const long long q1 = line_id % n1, q2 = line_id / n1;
    const long long c = rest / (factor - 1), m = rest % (factor - 1) + 1;
    T *const line = fine + q1 * step1 + q2 * step2;
    const long long cm = c > 0 ? c - 1 : 0, cp = c + 2 < n - 1 ? c + 2 : n - 1;
    const T v0 = line[cm * factor * stride], v1 = line[c * factor * stride], v2 = line[(c + 1) * factor * stride],
            v3 = line[cp * factor * stride];
    const double *wm = w + 4 * m;
    line[(c * factor + m) * stride] = T(wm[0] * v0 + wm[1] * v1 + wm[2] * v2 + wm[3] * v3);
}

inline unsigned blocks_for(long long n, int t) { return unsigned((n + t - 1) / t); }

}  // namespace

GridDesc grid_strided(const GridDesc &g, long long stride, bool g64) {
    GridDesc s = g;
    for (int d = 0; d < 3; d++) {
        s.n[d] = (g.n[d] - 1) / stride + 1;
        // h * G(stride) in G (serial/bvh/sdf_rebuild.cpp:122-130)
        s.h[d] = g64 ? g.h[d] * double(stride) : double(float(g.h[d]) * float(stride));
    }
    return s;
}

GridDesc grid_refined(const GridDesc &g, long long factor, bool g64) {
    GridDesc r = g;
    for (int d = 0; d < 3; d++) {
        r.n[d] = (g.n[d] - 1) * factor + 1;
        const double h = g.h[d] / double(factor);  // G(double(h) / double(factor))
        r.h[d] = g64 ? h : double(float(h));
    }
    return r;
}

// Triangles of {f = level} on the device. With *d_offsets null it counts them (into *ntri) and keeps
// the per-cell offsets in *d_offsets (the caller frees them, stream-ordered); with x not null it
// writes the soup into device x, y, z [3 * ntri] (sized from the counting call).
template <typename G, typename T>
int level_set_device(const GridDesc &gd, const T *d_f, T level, long long *ntri, G *x, G *y, G *z, int **d_offsets,
                     cudaStream_t stream) {
    for (int d = 0; d < 3; d++)
        if (gd.n[d] < 2) {
            *ntri = 0;
            return SSDF_OK;
        }
    const long long ncells = (gd.n[0] - 1) * (gd.n[1] - 1) * (gd.n[2] - 1);
    if (ncells >= 0x7fffffffll) return fail(SSDF_ERR_NOT_SUPPORTED, "more than 2^31 - 1 cells");
    int *count = nullptr, *offset = *d_offsets;
    if (!offset) {
        SSDF_CUDA(cudaMallocAsync(&count, sizeof(int) * size_t(ncells), stream));
        SSDF_CUDA(cudaMallocAsync(&offset, sizeof(int) * size_t(ncells), stream));
        k_marching<G, T, false><<<blocks_for(ncells, kThreadsR), kThreadsR, 0, stream>>>(
            gd, d_f, double(level), ncells, count, nullptr, nullptr, nullptr, nullptr);
        SSDF_CUDA(cudaGetLastError());
        SSDF_CHECK(exclusive_scan_i32(count, offset, int(ncells), stream));
        int last[2] = {0, 0};
        SSDF_CUDA(cudaMemcpyAsync(&last[0], offset + ncells - 1, sizeof(int), cudaMemcpyDeviceToHost, stream));
        SSDF_CUDA(cudaMemcpyAsync(&last[1], count + ncells - 1, sizeof(int), cudaMemcpyDeviceToHost, stream));
        SSDF_CUDA(cudaStreamSynchronize(stream));
        cudaFreeAsync(count, stream);
        *d_offsets = offset;
        *ntri = (long long)last[0] + last[1];
    }
    if (x) {
        k_marching<G, T, true><<<blocks_for(ncells, kThreadsR), kThreadsR, 0, stream>>>(
            gd, d_f, double(level), ncells, nullptr, offset, x, y, z);
        SSDF_CUDA(cudaGetLastError());
    }
    return SSDF_OK;
}

// rebuild_sdf on device arrays: d_out has strided(stride).size() entries.
template <typename G, typename T>
int rebuild_device(const GridDesc &gd, const T *d_f, T level, T band, long long stride, T *d_out, cudaStream_t stream) {
    if (stride < 1) return fail(SSDF_ERR_INVALID_ARGUMENT, "rebuild_sdf: stride must be >= 1");
    const bool g64 = sizeof(G) == 8;
    const GridDesc og = grid_strided(gd, stride, g64);
    const long long nout = og.n[0] * og.n[1] * og.n[2];
    long long ntri = 0;
    int *offsets = nullptr;
    SSDF_CHECK((level_set_device<G, T>(gd, d_f, level, &ntri, (G *)nullptr, (G *)nullptr, (G *)nullptr, &offsets,
                                       stream)));
    if (ntri >= kMaxTriangles) {
        cudaFreeAsync(offsets, stream);
        return fail(SSDF_ERR_NOT_SUPPORTED, "level set of more than 2^26 triangles");
    }
    const int searched = ntri > 0 ? 1 : 0;
    if (nout > 0) {
        k_band_start<T><<<blocks_for(nout, 256), 256, 0, stream>>>(gd, stride, og, d_f, level, band, searched, d_out);
        SSDF_CUDA(cudaGetLastError());
    }
    int st = SSDF_OK;
    if (searched && nout > 0) {
        G *soup = nullptr;
        int *idx = nullptr;
        SSDF_CUDA(cudaMallocAsync(&soup, sizeof(G) * 9 * size_t(ntri), stream));
        SSDF_CUDA(cudaMallocAsync(&idx, sizeof(int) * 3 * size_t(ntri), stream));
        G *x = soup, *y = soup + 3 * ntri, *z = soup + 6 * ntri;
        st = level_set_device<G, T>(gd, d_f, level, &ntri, x, y, z, &offsets, stream);
        if (st == SSDF_OK) {
            k_soup_indices<<<blocks_for(ntri, 256), 256, 0, stream>>>(ntri, idx, idx + ntri, idx + 2 * ntri);
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) st = cuda_fail(e, "rebuild_sdf indices", __FILE__, __LINE__);
        }
        ssdf_mesh *mesh = nullptr;
        if (st == SSDF_OK) {
            ssdf_build_opts bo;
            bo.leaf_size = 0, bo.keep_fp64 = 1, bo.normals = 0, bo.treelet_opt = 1;
            st = ssdf_mesh_create(&mesh, ptrdiff_t(ntri), idx, idx + ntri, idx + 2 * ntri, ptrdiff_t(3 * ntri), x, y, z,
                                  g64 ? SSDF_F64 : SSDF_F32, 1, &bo, stream);
        }
        if (st == SSDF_OK) {
            // the strided samples o + i h (in double from G's o and h), in/out from the band
            ssdf_query_opts qo;
            memset(&qo, 0, sizeof(qo));
            const char *pe = env_str("SSDF_B200_PRECISION");
            const int prec = pe && !strcmp(pe, "f64") ? SSDF_PREC_F64 : SSDF_PREC_F32_FIXUP;
            qo.precision = prec;
            qo.output = SSDF_OUT_EDF;
            qo.coord_type = SSDF_F64;
            qo.out_type = sizeof(T) == 8 ? SSDF_F64 : SSDF_F32;
            QueryArgs a;
            const double lo[3] = {og.o[0], og.o[1], og.o[2]};
            st = fill_grid_args(mesh, og.n[0], og.n[1], og.n[2], lo, lo, d_out, nullptr, &qo, &a);
            if (st == SSDF_OK) {
                for (int d = 0; d < 3; d++) a.lo64[d] = og.o[d], a.h64[d] = og.h[d];
                st = launch_query(a, prec, stream);
            }
        }
        if (mesh) ssdf_mesh_destroy_async(mesh, stream);  // in stream order, behind the query
        cudaFreeAsync(soup, stream);
        cudaFreeAsync(idx, stream);
    }
    cudaFreeAsync(offsets, stream);
    SSDF_CHECK(st);
    if (nout > 0) {
        k_band_sign<T><<<blocks_for(nout, 256), 256, 0, stream>>>(gd, stride, og, d_f, level, band, searched, d_out);
        SSDF_CUDA(cudaGetLastError());
    }
    return SSDF_OK;
}

template <typename G, typename T>
int refine_device(const GridDesc &gd, const T *d_f, long long factor, T *d_fine, cudaStream_t stream) {
    if (factor < 1) return fail(SSDF_ERR_INVALID_ARGUMENT, "refine_field: factor must be >= 1");
    const GridDesc rg = grid_refined(gd, factor, sizeof(G) == 8);
    const long long n = gd.n[0] * gd.n[1] * gd.n[2];
    if (n <= 0) return SSDF_OK;
    const long long fx = rg.n[0], fxy = rg.n[0] * rg.n[1];
    k_refine_place<T><<<blocks_for(n, 256), 256, 0, stream>>>(gd, factor, fx, fxy, d_f, d_fine);
    SSDF_CUDA(cudaGetLastError());
    if (factor == 1) return SSDF_OK;
    // weights of the cubic through samples -1, 0, 1, 2 at t = m / factor
    std::vector<double> w(4 * size_t(factor));
    for (long long m = 0; m < factor; m++) {
        const double t = double(m) / double(factor);
        w[4 * m + 0] = -t * (t - 1) * (t - 2) / 6;
        w[4 * m + 1] = (t + 1) * (t - 1) * (t - 2) / 2;
        w[4 * m + 2] = -(t + 1) * t * (t - 2) / 2;
        w[4 * m + 3] = (t + 1) * t * (t - 1) / 6;
    }
    double *dw = nullptr;
    SSDF_CUDA(cudaMallocAsync(&dw, sizeof(double) * w.size(), stream));
    SSDF_CUDA(cudaMemcpyAsync(dw, w.data(), sizeof(double) * w.size(), cudaMemcpyHostToDevice, stream));
    for (int axis = 0; axis < 3; axis++) {
        const long long stride = axis == 0 ? 1 : (axis == 1 ? fx : fxy);
        const long long na = gd.n[axis];
        const int a1 = (axis + 1) % 3, a2 = (axis + 2) % 3;
        const long long s1 = a1 == 0 ? 1 : (a1 == 1 ? fx : fxy), s2 = a2 == 0 ? 1 : (a2 == 1 ? fx : fxy);
        const long long c1 = a1 < axis ? 1 : factor, c2 = a2 < axis ? 1 : factor;
        const long long n1 = a1 < axis ? rg.n[a1] : gd.n[a1], n2 = a2 < axis ? rg.n[a2] : gd.n[a2];
        const long long items = n1 * n2 * (na - 1) * (factor - 1);
        if (items <= 0) continue;
        k_refine_axis<T><<<blocks_for(items, 256), 256, 0, stream>>>(n1, n2, na, factor, stride, c1 * s1, c2 * s2, dw,
                                                                     d_fine);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            cudaFreeAsync(dw, stream);
            return cuda_fail(e, "refine_field", __FILE__, __LINE__);
        }
    }
    cudaFreeAsync(dw, stream);
    return SSDF_OK;
}

// round_sdf on device arrays (serial/bvh/sdf_rebuild.hpp:57-78): R(f, 0), then the opening
// R(., r) + r and the closing R(., -r) - r as asked, then R(., 0) on the strided samples.
template <typename G, typename T>
int round_device(const GridDesc &gd, const T *d_f, T radius, T band, bool open, bool close, long long stride, T *d_out,
                 T *d_f0, cudaStream_t stream) {
    const long long n = gd.n[0] * gd.n[1] * gd.n[2];
    T *buf = nullptr;
    const int nbuf = 1 + (open ? 1 : 0) + (close ? 1 : 0);
    SSDF_CUDA(cudaMallocAsync(&buf, sizeof(T) * size_t(n > 0 ? n : 1) * nbuf, stream));
    T *r0 = buf, *a = buf + n, *b = buf + 2 * n;
    int st = rebuild_device<G, T>(gd, d_f, T(0), band, 1, r0, stream);
    const T *current = r0;
    if (st == SSDF_OK && open) {
        st = rebuild_device<G, T>(gd, current, radius, band, 1, a, stream);
        if (st == SSDF_OK && n > 0) k_shift<T><<<blocks_for(n, 256), 256, 0, stream>>>(n, a, radius);
        current = a;
    }
    if (st == SSDF_OK && close) {
        T *next = open ? b : a;
        st = rebuild_device<G, T>(gd, current, T(-radius), band, 1, next, stream);
        if (st == SSDF_OK && n > 0) k_shift<T><<<blocks_for(n, 256), 256, 0, stream>>>(n, next, T(-radius));
        current = next;
    }
    if (st == SSDF_OK) st = rebuild_device<G, T>(gd, current, T(0), band, stride, d_out, stream);
    if (st == SSDF_OK && d_f0) {
        const cudaError_t e = cudaMemcpyAsync(d_f0, r0, sizeof(T) * size_t(n), cudaMemcpyDeviceToDevice, stream);
        if (e != cudaSuccess) st = cuda_fail(e, "round_sdf f0", __FILE__, __LINE__);
    }
    cudaFreeAsync(buf, stream);
    return st;
}

template int level_set_device<float, float>(const GridDesc &, const float *, float, long long *, float *, float *,
                                            float *, int **, cudaStream_t);
template int level_set_device<double, double>(const GridDesc &, const double *, double, long long *, double *,
                                              double *, double *, int **, cudaStream_t);
template int rebuild_device<float, float>(const GridDesc &, const float *, float, float, long long, float *,
                                          cudaStream_t);
template int rebuild_device<double, double>(const GridDesc &, const double *, double, double, long long, double *,
                                            cudaStream_t);
template int refine_device<float, float>(const GridDesc &, const float *, long long, float *, cudaStream_t);
template int refine_device<double, double>(const GridDesc &, const double *, long long, double *, cudaStream_t);
template int round_device<float, float>(const GridDesc &, const float *, float, float, bool, bool, long long, float *,
                                        float *, cudaStream_t);
template int round_device<double, double>(const GridDesc &, const double *, double, double, bool, bool, long long,
                                          double *, double *, cudaStream_t);

}  // namespace ssdf_b200

// ---- C ABI over host arrays (serial/bvh/sdf_rebuild.hpp:23-78) ---------------------------------------

namespace {

using namespace ssdf_b200;

// Device buffers freed (stream-ordered) and the stream drained when the call returns.
struct Buffers {
    cudaStream_t stream;
    std::vector<void *> ptrs;
    explicit Buffers(cudaStream_t s) : stream(s) {}
    ~Buffers() {
        for (void *p : ptrs) cudaFreeAsync(p, stream);
        cudaStreamSynchronize(stream);
    }
    template <typename V>
    int alloc(V **p, size_t count) {
        void *q = nullptr;
        if (cudaMallocAsync(&q, sizeof(V) * (count ? count : 1), stream) != cudaSuccess)
            return fail(SSDF_ERR_OUT_OF_MEMORY, "device allocation of " + std::to_string(sizeof(V) * count) + " bytes");
        ptrs.push_back(q);
        *p = static_cast<V *>(q);
        return SSDF_OK;
    }
    template <typename V>
    int upload(V **p, const V *src, size_t count) {
        SSDF_CHECK(alloc(p, count));
        SSDF_CUDA(cudaMemcpyAsync(*p, src, sizeof(V) * count, cudaMemcpyHostToDevice, stream));
        return SSDF_OK;
    }
};

template <typename G>
int make_grid(const ptrdiff_t n[3], const G o[3], const G h[3], GridDesc *g) {
    if (!n || !o || !h) return fail(SSDF_ERR_INVALID_ARGUMENT, "null grid");
    for (int d = 0; d < 3; d++) {
        if (n[d] < 0) return fail(SSDF_ERR_INVALID_ARGUMENT, "negative grid size");
        g->n[d] = n[d];
        g->o[d] = double(o[d]);
        g->h[d] = double(h[d]);
    }
    return SSDF_OK;
}

int grid_stream(cudaStream_t *s) {
    *s = library_stream();
    if (!*s) return fail(SSDF_ERR_CUDA, "no usable CUDA device");
    return SSDF_OK;
}

long long grid_size(const GridDesc &g) { return g.n[0] * g.n[1] * g.n[2]; }

template <typename G>
int level_set_host(const ptrdiff_t n[3], const G o[3], const G h[3], const G *f, G level, ptrdiff_t capacity, G *x,
                   G *y, G *z, ptrdiff_t *ntriangles) {
    GridDesc g;
    SSDF_CHECK(make_grid(n, o, h, &g));
    if (!ntriangles) return fail(SSDF_ERR_INVALID_ARGUMENT, "null triangle count");
    *ntriangles = 0;
    const long long size = grid_size(g);
    if (size == 0) return SSDF_OK;
    if (!f) return fail(SSDF_ERR_INVALID_ARGUMENT, "null field");
    cudaStream_t s;
    SSDF_CHECK(grid_stream(&s));
    Buffers b(s);
    G *df = nullptr;
    SSDF_CHECK(b.upload(&df, f, size_t(size)));
    long long nt = 0;
    int *offsets = nullptr;
    const int st = level_set_device<G, G>(g, df, level, &nt, (G *)nullptr, (G *)nullptr, (G *)nullptr, &offsets, s);
    if (offsets) b.ptrs.push_back(offsets);
    SSDF_CHECK(st);
    *ntriangles = ptrdiff_t(nt);
    if (!x || nt == 0) return SSDF_OK;
    if (!y || !z) return fail(SSDF_ERR_INVALID_ARGUMENT, "null vertex array");
    if (capacity < nt)
        return fail(SSDF_ERR_INVALID_ARGUMENT, "level set has " + std::to_string(nt) + " triangles, capacity " +
                                                   std::to_string(capacity));
    G *soup = nullptr;
    SSDF_CHECK(b.alloc(&soup, 9 * size_t(nt)));
    SSDF_CHECK((level_set_device<G, G>(g, df, level, &nt, soup, soup + 3 * nt, soup + 6 * nt, &offsets, s)));
    SSDF_CUDA(cudaMemcpyAsync(x, soup, sizeof(G) * 3 * size_t(nt), cudaMemcpyDeviceToHost, s));
    SSDF_CUDA(cudaMemcpyAsync(y, soup + 3 * nt, sizeof(G) * 3 * size_t(nt), cudaMemcpyDeviceToHost, s));
    SSDF_CUDA(cudaMemcpyAsync(z, soup + 6 * nt, sizeof(G) * 3 * size_t(nt), cudaMemcpyDeviceToHost, s));
    SSDF_CUDA(cudaStreamSynchronize(s));
    return SSDF_OK;
}

template <typename G>
int rebuild_host(const ptrdiff_t n[3], const G o[3], const G h[3], const G *f, G level, G band, ptrdiff_t stride,
                 G *out) {
    GridDesc g;
    SSDF_CHECK(make_grid(n, o, h, &g));
    if (stride < 1) return fail(SSDF_ERR_INVALID_ARGUMENT, "rebuild_sdf: stride must be >= 1");
    const long long size = grid_size(g), nout = grid_size(grid_strided(g, stride, sizeof(G) == 8));
    if (size == 0) return SSDF_OK;
    if (!f || !out) return fail(SSDF_ERR_INVALID_ARGUMENT, "null field or output");
    cudaStream_t s;
    SSDF_CHECK(grid_stream(&s));
    Buffers b(s);
    G *df = nullptr, *dout = nullptr;
    SSDF_CHECK(b.upload(&df, f, size_t(size)));
    SSDF_CHECK(b.alloc(&dout, size_t(nout)));
    SSDF_CHECK((rebuild_device<G, G>(g, df, level, band, stride, dout, s)));
    SSDF_CUDA(cudaMemcpyAsync(out, dout, sizeof(G) * size_t(nout), cudaMemcpyDeviceToHost, s));
    SSDF_CUDA(cudaStreamSynchronize(s));
    return SSDF_OK;
}

template <typename G>
int refine_host(const ptrdiff_t n[3], const G o[3], const G h[3], const G *f, ptrdiff_t factor, G *fine) {
    GridDesc g;
    SSDF_CHECK(make_grid(n, o, h, &g));
    if (factor < 1) return fail(SSDF_ERR_INVALID_ARGUMENT, "refine_field: factor must be >= 1");
    const long long size = grid_size(g), nfine = grid_size(grid_refined(g, factor, sizeof(G) == 8));
    if (size == 0) return SSDF_OK;
    if (!f || !fine) return fail(SSDF_ERR_INVALID_ARGUMENT, "null field");
    cudaStream_t s;
    SSDF_CHECK(grid_stream(&s));
    Buffers b(s);
    G *df = nullptr, *dfine = nullptr;
    SSDF_CHECK(b.upload(&df, f, size_t(size)));
    SSDF_CHECK(b.alloc(&dfine, size_t(nfine)));
    SSDF_CHECK((refine_device<G, G>(g, df, factor, dfine, s)));
    SSDF_CUDA(cudaMemcpyAsync(fine, dfine, sizeof(G) * size_t(nfine), cudaMemcpyDeviceToHost, s));
    SSDF_CUDA(cudaStreamSynchronize(s));
    return SSDF_OK;
}

template <typename G>
int round_host(const ptrdiff_t n[3], const G o[3], const G h[3], const G *f, G radius, G band, int open, int close,
               ptrdiff_t stride, G *out, G *f0) {
    GridDesc g;
    SSDF_CHECK(make_grid(n, o, h, &g));
    if (stride < 1) return fail(SSDF_ERR_INVALID_ARGUMENT, "round_sdf: stride must be >= 1");
    const long long size = grid_size(g), nout = grid_size(grid_strided(g, stride, sizeof(G) == 8));
    if (size == 0) return SSDF_OK;
    if (!f || !out) return fail(SSDF_ERR_INVALID_ARGUMENT, "null field or output");
    cudaStream_t s;
    SSDF_CHECK(grid_stream(&s));
    Buffers b(s);
    G *df = nullptr, *dout = nullptr, *df0 = nullptr;
    SSDF_CHECK(b.upload(&df, f, size_t(size)));
    SSDF_CHECK(b.alloc(&dout, size_t(nout)));
    if (f0) SSDF_CHECK(b.alloc(&df0, size_t(size)));
    SSDF_CHECK((round_device<G, G>(g, df, radius, band, open != 0, close != 0, stride, dout, df0, s)));
    SSDF_CUDA(cudaMemcpyAsync(out, dout, sizeof(G) * size_t(nout), cudaMemcpyDeviceToHost, s));
    if (f0) SSDF_CUDA(cudaMemcpyAsync(f0, df0, sizeof(G) * size_t(size), cudaMemcpyDeviceToHost, s));
    SSDF_CUDA(cudaStreamSynchronize(s));
    return SSDF_OK;
}

}  // namespace

extern "C" {

int ssdf_b200_level_set_triangles_ff(const ptrdiff_t n[3], const float o[3], const float h[3], const float *f,
                                     float level, ptrdiff_t capacity, float *x, float *y, float *z,
                                     ptrdiff_t *ntriangles) {
    return level_set_host<float>(n, o, h, f, level, capacity, x, y, z, ntriangles);
}
int ssdf_b200_level_set_triangles_dd(const ptrdiff_t n[3], const double o[3], const double h[3], const double *f,
                                     double level, ptrdiff_t capacity, double *x, double *y, double *z,
                                     ptrdiff_t *ntriangles) {
    return level_set_host<double>(n, o, h, f, level, capacity, x, y, z, ntriangles);
}
int ssdf_b200_rebuild_sdf_ff(const ptrdiff_t n[3], const float o[3], const float h[3], const float *f, float level,
                             float band, ptrdiff_t stride, float *out) {
    return rebuild_host<float>(n, o, h, f, level, band, stride, out);
}
int ssdf_b200_rebuild_sdf_dd(const ptrdiff_t n[3], const double o[3], const double h[3], const double *f,
                             double level, double band, ptrdiff_t stride, double *out) {
    return rebuild_host<double>(n, o, h, f, level, band, stride, out);
}
int ssdf_b200_refine_field_ff(const ptrdiff_t n[3], const float o[3], const float h[3], const float *f,
                              ptrdiff_t factor, float *fine) {
    return refine_host<float>(n, o, h, f, factor, fine);
}
int ssdf_b200_refine_field_dd(const ptrdiff_t n[3], const double o[3], const double h[3], const double *f,
                              ptrdiff_t factor, double *fine) {
    return refine_host<double>(n, o, h, f, factor, fine);
}
int ssdf_b200_round_sdf_ff(const ptrdiff_t n[3], const float o[3], const float h[3], const float *f, float radius,
                           float band, int open, int close, ptrdiff_t stride, float *out, float *f0) {
    return round_host<float>(n, o, h, f, radius, band, open, close, stride, out, f0);
}
int ssdf_b200_round_sdf_dd(const ptrdiff_t n[3], const double o[3], const double h[3], const double *f, double radius,
                           double band, int open, int close, ptrdiff_t stride, double *out, double *f0) {
    return round_host<double>(n, o, h, f, radius, band, open, close, stride, out, f0);
}

}  // extern "C"
