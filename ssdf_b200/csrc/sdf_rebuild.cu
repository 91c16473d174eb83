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

// ---- marching tetrahedra ------------------------------------------------------------------------
//
// A cell's corners are numbered c = x + 2 y + 4 z for its offsets x, y, z in {0, 1}. Within a cell a
// corner's grid index grows with its number (the grid's strides are 1 < nx < nx ny whenever the grid
// has cells), so the corner of lower grid index on an edge is its lower-numbered corner: an edge is
// named by its code (lo << 3) | hi, and its crossing is interpolated from lo.
//
// The cell is cut into the six tetrahedra about its 0-7 diagonal (the order of this list is the order
// of the output). For each tetrahedron and each 4-bit pattern p of its corners above the level (bit s
// for its corner s), the table below lists the crossing edges of the triangles to emit, in emission
// order:
//   - a corner alone on its side of the level: one triangle on that corner's three edges, the other
//     corners taken in the tetrahedron's order;
//   - two corners on each side (u0, u1 above, d0, d1 not, each pair in the tetrahedron's order): the
//     quadrilateral u0d0, u0d1, u1d1, u1d0, emitted as its triangles (0, 1, 2) and (0, 2, 3).
// An entry packs the triangle count in bits 0-1 and six 6-bit edge codes from bit 2 on.
constexpr int kTetCorner[6][4] = {{0, 1, 3, 7}, {0, 1, 5, 7}, {0, 2, 3, 7}, {0, 2, 6, 7}, {0, 4, 5, 7}, {0, 4, 6, 7}};

struct TetTable {
    unsigned long long entry[6][16];
    int corner[6][4];
};

constexpr unsigned edge_code(int a, int b) { return a < b ? unsigned((a << 3) | b) : unsigned((b << 3) | a); }

constexpr TetTable make_tet_table() {
    TetTable tab{};
    for (int tet = 0; tet < 6; tet++) {
        for (int pat = 0; pat < 16; pat++) {
            int hi[4] = {0, 0, 0, 0}, lo[4] = {0, 0, 0, 0}, nh = 0, nl = 0;
            for (int s = 0; s < 4; s++) {
                if ((pat >> s) & 1)
                    hi[nh++] = kTetCorner[tet][s];
                else
                    lo[nl++] = kTetCorner[tet][s];
            }
            unsigned edges[6] = {0, 0, 0, 0, 0, 0};
            int ntri = 0;
            if (nh == 1 || nl == 1) {
                const int alone = nh == 1 ? hi[0] : lo[0];
                const int *rest = nh == 1 ? lo : hi;
                for (int v = 0; v < 3; v++) edges[v] = edge_code(alone, rest[v]);
                ntri = 1;
            } else if (nh == 2) {
                const unsigned quad[4] = {edge_code(hi[0], lo[0]), edge_code(hi[0], lo[1]), edge_code(hi[1], lo[1]),
                                          edge_code(hi[1], lo[0])};
                const int split[6] = {0, 1, 2, 0, 2, 3};
                for (int v = 0; v < 6; v++) edges[v] = quad[split[v]];
                ntri = 2;
            }
            unsigned long long e = (unsigned long long)ntri;
            for (int v = 0; v < 3 * ntri; v++) e |= (unsigned long long)edges[v] << (2 + 6 * v);
            tab.entry[tet][pat] = e;
        }
        for (int s = 0; s < 4; s++) tab.corner[tet][s] = kTetCorner[tet][s];
    }
    return tab;
}

__constant__ TetTable c_tet = make_tet_table();

// One cell (its lowest corner at grid (i, j, k)): corner values less the level and the pattern of the
// corners above it.
struct MtCell {
    double val[8];
    unsigned above;
    long long base[3];
};

// The crossing of edge `code` (corner positions o + index * h, then the interpolation from the lower
// corner, in the reference's expression order; the library is built without contraction).
__device__ __forceinline__ void mt_crossing(const GridDesc &gd, const MtCell &c, unsigned code, double q[3]) {
    const int a = int(code >> 3), b = int(code & 7);
    const double t = c.val[a] / (c.val[a] - c.val[b]);
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double pa = gd.o[d] + double(c.base[d] + ((a >> d) & 1)) * gd.h[d];
        const double pb = gd.o[d] + double(c.base[d] + ((b >> d) & 1)) * gd.h[d];
        q[d] = pa + t * (pb - pa);
    }
}

// Visits the cell's triangles in output order, each as its three vertices rounded to G, skipping those
// with two vertices equal in G (a corner on the level makes crossings coincide); returns how many.
template <typename G, class Emit>
__device__ int mt_cell_triangles(const GridDesc &gd, const MtCell &c, Emit emit) {
    int kept = 0;
    for (int tet = 0; tet < 6; tet++) {
        unsigned pat = 0;
#pragma unroll
        for (int s = 0; s < 4; s++) pat |= ((c.above >> c_tet.corner[tet][s]) & 1u) << s;
        const unsigned long long e = c_tet.entry[tet][pat];
        const int ntri = int(e & 3ull);
        for (int t = 0; t < ntri; t++) {
            G v[3][3];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                double q[3];
                mt_crossing(gd, c, unsigned((e >> (2 + 6 * (3 * t + k))) & 63ull), q);
                v[k][0] = G(q[0]), v[k][1] = G(q[1]), v[k][2] = G(q[2]);
            }
            auto same = [&](int a, int b) { return v[a][0] == v[b][0] && v[a][1] == v[b][1] && v[a][2] == v[b][2]; };
            if (same(0, 1) || same(1, 2) || same(2, 0)) continue;
            emit(kept, v);
            kept++;
        }
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
    MtCell c;
    c.base[0] = cell % cx;
    c.base[1] = (cell / cx) % cy;
    c.base[2] = cell / (cx * cy);
    const long long sy = gd.n[0], sz = gd.n[0] * gd.n[1];
    const long long g0 = c.base[0] + c.base[1] * sy + c.base[2] * sz;
    c.above = 0;
#pragma unroll
    for (int q = 0; q < 8; q++) {
        c.val[q] = double(f[g0 + (q & 1) + ((q >> 1) & 1) * sy + ((q >> 2) & 1) * sz]) - level;
        c.above |= (c.val[q] > 0 ? 1u : 0u) << q;
    }
    if (c.above == 0u || c.above == 0xffu) {  // the level does not cross this cell
        if (!EMIT) count[cell] = 0;
        return;
    }
    if (EMIT) {
        const long long first = offset[cell];
        mt_cell_triangles<G>(gd, c, [&](int t, const G (&v)[3][3]) {
            const long long o = 3 * (first + t);
#pragma unroll
            for (int k = 0; k < 3; k++) x[o + k] = v[k][0], y[o + k] = v[k][1], z[o + k] = v[k][2];
        });
    } else {
        count[cell] = mt_cell_triangles<G>(gd, c, [](int, const G (&)[3][3]) {});
    }
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

// refine_field (serial/bvh/sdf_rebuild.hpp:40-55). The fine grid's samples at multiples of factor
// along all three axes are the coarse ones; every other sample is the cubic through the four nearest
// samples along one axis (the end samples repeated), axis by axis -- x, then y, then z -- each value
// rounded to T before a later axis reads it. Pass `axis` here computes every fine sample whose index is
// a multiple of factor along the axes after `axis` and not along `axis` (for x: along any x), one
// thread per sample, gathering its four inputs from the previous pass's samples on its line (for x:
// straight from the coarse field, which also places the coarse samples).
__device__ __forceinline__ void cubic_weights(long long m, long long factor, double w[4]) {
    const double t = double(m) / double(factor);
    w[0] = -t * (t - 1) * (t - 2) / 6;
    w[1] = (t + 1) * (t - 1) * (t - 2) / 2;
    w[2] = -(t + 1) * t * (t - 2) / 2;
    w[3] = (t + 1) * t * (t - 1) / 6;
}

struct RefineDims {
    long long coarse[3], fine[3];  // samples per axis
    long long factor;
};

template <typename T, int AXIS>
__global__ void k_refine_pass(RefineDims d, const T *__restrict__ f, T *__restrict__ fine) {
    // outputs of this pass: fine indices along the axes up to AXIS, coarse ones after it
    long long ext[3];
#pragma unroll
    for (int a = 0; a < 3; a++) ext[a] = a <= AXIS ? d.fine[a] : d.coarse[a];
    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p >= ext[0] * ext[1] * ext[2]) return;
    long long idx[3] = {p % ext[0], (p / ext[0]) % ext[1], p / (ext[0] * ext[1])};
    const long long m = idx[AXIS] % d.factor, c = idx[AXIS] / d.factor;
    if (AXIS > 0 && m == 0) return;  // a multiple of factor along AXIS: an earlier pass wrote it
    // fine position of the output (indices after AXIS are coarse, so scaled)
    long long fpos[3];
#pragma unroll
    for (int a = 0; a < 3; a++) fpos[a] = a <= AXIS ? idx[a] : idx[a] * d.factor;
    const long long sy = d.fine[0], sz = d.fine[0] * d.fine[1];
    const long long out = fpos[0] + fpos[1] * sy + fpos[2] * sz;
    // the line's samples along AXIS at coarse position q: the coarse field (x) or the earlier passes
    auto line = [&](long long q) -> T {
        if (AXIS == 0) return f[q + d.coarse[0] * (idx[1] + d.coarse[1] * idx[2])];
        long long at[3] = {fpos[0], fpos[1], fpos[2]};
        at[AXIS] = q * d.factor;
        return fine[at[0] + at[1] * sy + at[2] * sz];
    };
    if (m == 0) {  // x pass only: the coarse sample itself
        fine[out] = line(c);
        return;
    }
    const long long n = d.coarse[AXIS];
    const T v0 = line(c > 0 ? c - 1 : 0), v1 = line(c), v2 = line(c + 1), v3 = line(c + 2 < n - 1 ? c + 2 : n - 1);
    double w[4];
    cubic_weights(m, d.factor, w);
    fine[out] = T(w[0] * v0 + w[1] * v1 + w[2] * v2 + w[3] * v3);
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
    if (gd.n[0] * gd.n[1] * gd.n[2] <= 0) return SSDF_OK;
    RefineDims d;
    for (int a = 0; a < 3; a++) d.coarse[a] = gd.n[a], d.fine[a] = rg.n[a];
    d.factor = factor;
    // pass a covers fine extents up to a and coarse ones after it
    const long long n0 = d.fine[0] * d.coarse[1] * d.coarse[2], n1 = d.fine[0] * d.fine[1] * d.coarse[2],
                    n2 = d.fine[0] * d.fine[1] * d.fine[2];
    k_refine_pass<T, 0><<<blocks_for(n0, 256), 256, 0, stream>>>(d, d_f, d_fine);
    SSDF_CUDA(cudaGetLastError());
    if (factor == 1) return SSDF_OK;
    k_refine_pass<T, 1><<<blocks_for(n1, 256), 256, 0, stream>>>(d, d_f, d_fine);
    SSDF_CUDA(cudaGetLastError());
    k_refine_pass<T, 2><<<blocks_for(n2, 256), 256, 0, stream>>>(d, d_f, d_fine);
    SSDF_CUDA(cudaGetLastError());
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
