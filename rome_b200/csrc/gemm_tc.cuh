// Tensor-core (tcgen05) cross-term contraction, implemented in gemm_tc.cu.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "epilogues.cuh"

namespace rome {
// diff2 = epilogue(A[M][Kp] . B[N][Kp]^T); A, B bf16 (hi plane, then lo plane
// for ROME_PREC_BF16X3), K-major, Kp a multiple of 64.
// derr: the context's device error flag (set when a bounded wait expires)
void tc_diff2_gemm(cudaStream_t st, int M, int N, int Kp, const void* A, const void* B, int precision,
                   const Diff2Epi& epi, int* derr);
// out[m][n] = A . B^T in split precision (hi*hi + hi*lo + lo*hi)
void tc_store_gemm(cudaStream_t st, int M, int N, int Kp, const void* A, const void* B, float* out, int ld,
                   int* derr);
// out[m][n] = A . B^T + bias[n / group]: split precision (hi and lo planes of
// A and B), or with split false the hi planes alone (one BF16 product)
void tc_bias_gemm(cudaStream_t st, int M, int N, int Kp, const void* A, const void* B, float* out, int ld,
                  const float* bias, int group, int* derr, bool split = true);
// bf16 hi plane then (with_lo) lo plane of a [rows][ldin] fp32 matrix, K columns used, padded to Kpad
void split_bf16(cudaStream_t st, const float* in, long rows, int K, int ldin, int Kpad, void* out,
                bool with_lo = true);
// the same planes of the transpose: [cols][rows_pad] from a [rows][ldin] matrix (rows beyond `rows` zero)
void split_bf16_t(cudaStream_t st, const float* in, int rows, int cols, int ldin, int rows_pad, void* out);
// the autotuner's choices: one line per key with every candidate's time
std::string tc_tuning_report();
// raises ROME_ERR_TIMEOUT if a tensor-core kernel's bounded wait expired
void tc_check_error(cudaStream_t st, int* derr);
}  // namespace rome
