// GEMM epilogues shared by the CUDA-core and tensor-core contractions.
// operator() stores one element and returns the stored value; finish_row()
// receives the minimum of the values a thread stored for one row.
#pragma once
#include <cuda_runtime.h>

#include <cmath>

namespace rome {

// order-preserving map of a float onto an unsigned key (for atomicMin)
__device__ __forceinline__ unsigned float_key(float f) {
    unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_float(unsigned k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

struct StoreEpi {
    float* out;
    int ld;
    __device__ __forceinline__ float operator()(int m, int n, float v) const {
        out[(long)m * ld + n] = v;
        return v;
    }
    __device__ __forceinline__ void finish_row(int, float) const {}
};

// out[m][n] = v + bias[n / group] (a per-class bias over `group` columns)
struct BiasStoreEpi {
    float* out;
    int ld;
    const float* bias;
    int group;
    __device__ __forceinline__ float operator()(int m, int n, float v) const {
        v += bias[n / group];
        out[(long)m * ld + n] = v;
        return v;
    }
    __device__ __forceinline__ void finish_row(int, float) const {}
};

// diff2 epilogue of the cross-term GEMM (rows m = particle*T + translation,
// columns j = orientation), written in the reference's exp_Mweight layout
// [particle][((class*npsi+psi)*nor+over_rot)*T + trans*notr + over_trans].
// Hypotheses the reference skips (class/orientation not significant, or
// coarse translation not significant in the fine pass) become +inf.  The
// per-particle minimum (exp_min_diff2, src/map2d_optimizer.cpp:1043-1062)
// is folded in with one atomicMin per row and tile.
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
    unsigned* rowmin;  // per particle, float_key order; may be null
    __device__ __forceinline__ float operator()(int m, int n, float c) const {
        int i = m / T, t = m - i * T;
        bool ok = jvalid[n] != 0;
        if (ok && mcoarse) ok = mcoarse[(long)i * ncoarse + (long)(n / nor) * ntr + t / notr] != 0;
        float v = INFINITY;
        if (ok) v = (float)(0.5 * ((double)norm[(long)i * J + n] - 2.0 * (double)c + (double)S[m] + xi2[i]));
        diff2[(long)i * X + (long)n * T + t] = v;
        return v;
    }
    __device__ __forceinline__ void finish_row(int m, float v) const {
        if (rowmin && v < INFINITY) atomicMin(&rowmin[m / T], float_key(v));
    }
};

}  // namespace rome
