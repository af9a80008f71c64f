// Tensor-core restricted (proposal) search of the MAP2D E-step, implemented
// in restricted_tc.cu.
#pragma once
#include <cuda_runtime.h>

namespace rome {

// Per-particle operands of the restricted contraction: xw[i][a] = Minvsigma2
// * ctf * X (complex, FP32) on the active pixels, w2[i][a] = Minvsigma2 *
// ctf^2, both zero padded to Kh = Kp / 2 columns, and S[i] = sum_n
// Minvsigma2 |X|^2 over all pixels.
void restricted_prep(cudaStream_t st, int P, int F, int Kact, int Kh, const double2* Fimg, const double* lctf,
                     const double* Minv, int apply_ctf, const int* act, float2* xw, float* w2, float* S);

// Width of the translation tile (UMMA N) for T translations: 32, 64, 128 or
// 256 (T <= 256).
inline int restricted_tile_tn(int T) { return T <= 32 ? 32 : T <= 64 ? 64 : T <= 128 ? 128 : 256; }

// The translation operand: row t < T holds (cos, -sin) of translation t's
// phase at every active pixel, interleaved like the cross-term operands
// (bf16 hi plane [TN][Kp], then the lo plane when split), rows T..TN-1 zero.
void restricted_shift_operand(cudaStream_t st, int T, int Kact, int Kp, const unsigned short* pidx,
                              const double2* tab, int precision, void* sh);

// diff2[i][q * T + t] for every particle i, proposal q < nprop and
// translation t < T (T <= 256): the per-(particle, proposal) product
// w = xw_i * conj(P_j) is formed on the CUDA cores straight into shared
// memory and contracted with the translation operand on the tensor cores.
// B: the dense contraction's orientation operand (bf16 [Jrows][Kp], lo plane
// after it for ROME_PREC_BF16X3).  derr: the context's device error flag.
void restricted_tc_diff2(cudaStream_t st, int precision, int P, int nprop, int T, int Kp, const int* prop,
                         const int* jvalid, const float2* xw, const float* w2, const void* B, long Jrows,
                         const void* sh, const float* S, const double* xi2, long Xr, float* diff2, unsigned* rowmin,
                         int* derr);

}  // namespace rome
