// Tensor-core (tcgen05) cross-term GEMM: declared here, implemented in
// gemm_tc.cu.  The epilogue type is fixed to the diff2 epilogue.
#pragma once
#include <cuda_runtime.h>

#include "epilogues.cuh"

namespace rome {
void tc_diff2_gemm(cudaStream_t st, int M, int N, int Kp, const void* A, const void* B, int precision,
                   const Diff2Epi& epi);
}
