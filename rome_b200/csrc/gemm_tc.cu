// tcgen05 BF16 GEMM for the diff2 cross term (work in progress).
#include "common.cuh"
#include "gemm_tc.cuh"

namespace rome {
void tc_diff2_gemm(cudaStream_t, int, int, int, const void*, const void*, int precision, const Diff2Epi&) {
    fail(ROME_ERR_UNSUPPORTED, "tensor-core precision %d not available in this build", precision);
}
}  // namespace rome
