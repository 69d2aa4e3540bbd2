// tq_tc.cu -- split-BF16 tcgen05 contraction (placeholder until the kernel lands).
#include "tq_mton.h"

namespace tq {

cudaError_t launch_tc_dist(const void *, const void *, const void *, const void *, int, size_t,
                           size_t, size_t, size_t, const float *, const float *, const float *,
                           const float *, float *, size_t, int *, cudaStream_t) {
    return cudaErrorNotSupported;
}

}  // namespace tq
