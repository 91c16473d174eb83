// treelet_opt.cu -- SAH treelet refinement of the LBVH (placeholder until implemented).
#include "internal.h"

namespace ssdf_b200 {

int treelet_optimize(int, int *, int *, int *, int *, int *, float *, double *, const float *, const double *, int *,
                     cudaStream_t) {
    return fail(SSDF_ERR_NOT_SUPPORTED, "treelet refinement is not available in this build");
}

}  // namespace ssdf_b200
