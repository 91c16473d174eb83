// ssdf_distributed.hpp -- ssdf::pedf and ssdf::pedf_update (distributed/psdf.hpp:149-302, 304-482)
// over an NCCL communicator, for C++ callers of the reference's distributed distance functions.
//
// The reference's signature with the communicator replaced: an ncclComm_t (one process per GPU) in
// place of the MPI_Comm, DEVICE arrays in place of host arrays, and an optional CUDA stream on which
// the exchanges and the query run; the call returns when `out` holds the result. SSDF_USE_ALLGATHER
// keeps its meaning for pedf. Instantiations: <double, double, int>, <float, double, int>,
// <float, float, int>.
#pragma once

#include <cuda_runtime.h>
#include <nccl.h>

#include <cstddef>
#include <type_traits>

#include "ssdf_b200.h"

namespace ssdf {
namespace detail {
template <typename G, typename T>
constexpr bool pedf_types() {
    return (std::is_same<G, double>::value && std::is_same<T, double>::value) ||
           (std::is_same<G, float>::value && std::is_same<T, double>::value) ||
           (std::is_same<G, float>::value && std::is_same<T, float>::value);
}
template <typename X>
constexpr int code() {
    return std::is_same<X, double>::value ? SSDF_F64 : SSDF_F32;
}
}  // namespace detail

// distributed/psdf.hpp:149-163
template <typename G, typename T, typename I>
int pedf(ncclComm_t comm, const ptrdiff_t lnpoints, const G *x, const G *y, const G *z, const ptrdiff_t lnselements,
         const I *s0, const I *s1, const I *s2, const ptrdiff_t lnspoints, const G *sx, const G *sy, const G *sz,
         T *out, cudaStream_t stream = nullptr) {
    static_assert(std::is_same<I, int>::value, "ssdf_b200 indices are int");
    static_assert(detail::pedf_types<G, T>(), "pedf: <double,double>, <float,double>, <float,float>");
    return ssdf_pedf_nccl(comm, lnpoints, x, y, z, lnselements, s0, s1, s2, lnspoints, sx, sy, sz, detail::code<G>(),
                          detail::code<T>(), out, stream);
}

// distributed/psdf.hpp:304-318
template <typename G, typename T, typename I>
int pedf_update(ncclComm_t comm, const ptrdiff_t lnpoints, const G *x, const G *y, const G *z,
                const ptrdiff_t lnselements, const I *s0, const I *s1, const I *s2, const ptrdiff_t lnspoints,
                const G *sx, const G *sy, const G *sz, T *out, cudaStream_t stream = nullptr) {
    static_assert(std::is_same<I, int>::value, "ssdf_b200 indices are int");
    static_assert(detail::pedf_types<G, T>(), "pedf_update: <double,double>, <float,double>, <float,float>");
    return ssdf_pedf_update_nccl(comm, lnpoints, x, y, z, lnselements, s0, s1, s2, lnspoints, sx, sy, sz,
                                 detail::code<G>(), detail::code<T>(), out, stream);
}

}  // namespace ssdf
