// GEMM epilogues shared by the CUDA-core and tensor-core contractions.
#pragma once
#include <cuda_runtime.h>

#include <cmath>

namespace rome {

struct StoreEpi {
    float* out;
    int ld;
    __device__ __forceinline__ void operator()(int m, int n, float v) const { out[(long)m * ld + n] = v; }
};

// diff2 epilogue of the cross-term GEMM (rows m = particle*T + translation,
// columns j = orientation), written in the reference's exp_Mweight layout
// [particle][((class*npsi+psi)*nor+over_rot)*T + trans*notr + over_trans].
// Hypotheses the reference skips (class/orientation not significant, or
// coarse translation not significant in the fine pass) become +inf.
struct Diff2Epi {
    float* diff2;
    const float* norm;
    const float* S;
    const double* xi2;
    const int* jvalid;
    int T, J;
    long X;
    int notr, nor, ntr;
    long ncoarse;
    const char* mcoarse;
    __device__ __forceinline__ void operator()(int m, int n, float c) const {
        int i = m / T, t = m - i * T;
        bool ok = jvalid[n] != 0;
        if (ok && mcoarse) ok = mcoarse[(long)i * ncoarse + (long)(n / nor) * ntr + t / notr] != 0;
        float v = INFINITY;
        if (ok) v = (float)(0.5 * ((double)norm[(long)i * J + n] - 2.0 * (double)c + (double)S[m] + xi2[i]));
        diff2[(long)i * X + (long)n * T + t] = v;
    }
};

}  // namespace rome
