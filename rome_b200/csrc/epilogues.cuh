// GEMM epilogues shared by the CUDA-core and tensor-core contractions.
// operator() stores one element and returns the stored value; finish_row()
// receives the minimum of the values a thread stored for one row.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

namespace rome {

// order-preserving map of a float onto an unsigned key (for atomicMin)
__device__ __forceinline__ unsigned float_key(float f) {
    unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_float(unsigned k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

// Epilogues are called per element (operator()) by the CUDA-core contraction
// and per 16 consecutive columns of one row (row() once per row and tile,
// then chunk16()) by the tensor-core one, which reads 16 columns at a time
// out of TMEM; chunk16 returns the minimum of the values it stored.
struct StoreEpi {
    float* out;
    int ld;
    __device__ __forceinline__ float operator()(int m, int n, float v) const {
        out[(long)m * ld + n] = v;
        return v;
    }
    __device__ __forceinline__ void finish_row(int, float) const {}
    struct Row {
        int m;
    };
    __device__ __forceinline__ Row row(int m) const { return Row{m}; }
    __device__ __forceinline__ float chunk16(const Row& r, int n, const float (&v)[16], int nvalid) const {
        float mn = INFINITY;
#pragma unroll
        for (int q = 0; q < 16; q++)
            if (q < nvalid) mn = fminf(mn, (*this)(r.m, n + q, v[q]));
        return mn;
    }
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
    struct Row {
        int m;
    };
    __device__ __forceinline__ Row row(int m) const { return Row{m}; }
    __device__ __forceinline__ float chunk16(const Row& r, int n, const float (&v)[16], int nvalid) const {
        float mn = INFINITY;
#pragma unroll
        for (int q = 0; q < 16; q++)
            if (q < nvalid) mn = fminf(mn, (*this)(r.m, n + q, v[q]));
        return mn;
    }
};

// diff2 epilogue of the cross-term GEMM (rows m = particle*T + translation,
// columns j = orientation), written in the reference's exp_Mweight layout
// [particle][((class*npsi+psi)*nor+over_rot)*T + trans*notr + over_trans].
// Hypotheses the reference skips (class/orientation not significant, or
// coarse translation not significant in the fine pass) become +inf.  The
// per-particle minimum (exp_min_diff2, src/map2d_optimizer.cpp:1043-1062)
// is folded in with one atomicMin per row and tile.  With ccx (per particle
// image norm |X|, exp_local_sqrtXi2) the epilogue writes the cross-correlation
// mode's value -C / (sqrt(N) |X|) instead (get_diff,
// src/map3d_optimizer.cpp:1086-1102; the operands then carry no
// Minvsigma2, so C is the signal product and N the reference power).
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
    const double* ccx = nullptr;
    __device__ __forceinline__ float operator()(int m, int n, float c) const {
        int i = m / T, t = m - i * T;
        bool ok = jvalid[n] != 0;
        if (ok && mcoarse) ok = mcoarse[(long)i * ncoarse + (long)(n / nor) * ntr + t / notr] != 0;
        float v = INFINITY;
        if (ok && ccx) v = (float)(-(double)c / (sqrt((double)norm[(long)i * J + n]) * ccx[i]));
        else if (ok) v = (float)(0.5 * ((double)norm[(long)i * J + n] - 2.0 * (double)c + (double)S[m] + xi2[i]));
        diff2[(long)i * X + (long)n * T + t] = v;
        return v;
    }
    __device__ __forceinline__ void finish_row(int m, float v) const {
        if (rowmin && v < INFINITY) atomicMin(&rowmin[m / T], float_key(v));
    }
    // per-row constants of a tile row: output base, S[m] + Xi2[i] (cross-correlation
    // mode: the image norm), the particle's norm row and Mcoarse row
    struct Row {
        long out;
        double rc;
        const float* nrm;
        const char* mc;
    };
    __device__ __forceinline__ Row row(int m) const {
        const int i = m / T, t = m - i * T;
        return Row{(long)i * X + t, ccx ? ccx[i] : (double)S[m] + xi2[i], norm + (long)i * J,
                   mcoarse ? mcoarse + (long)i * ncoarse + t / notr : nullptr};
    }
    __device__ __forceinline__ float chunk16(const Row& r, int n, const float (&v)[16], int nvalid) const {
        float nv[16];
        int jv[16];
        if (nvalid == 16 && (((uintptr_t)(r.nrm + n) | (uintptr_t)(jvalid + n)) & 15) == 0) {
            // 16-byte loads (when both addresses are 16-byte aligned): the row's norm terms and the
            // column validity
#pragma unroll
            for (int q = 0; q < 16; q += 4) {
                const float4 a = *(const float4*)(r.nrm + n + q);
                const int4 b = *(const int4*)(jvalid + n + q);
                nv[q] = a.x, nv[q + 1] = a.y, nv[q + 2] = a.z, nv[q + 3] = a.w;
                jv[q] = b.x, jv[q + 1] = b.y, jv[q + 2] = b.z, jv[q + 3] = b.w;
            }
        } else {
#pragma unroll
            for (int q = 0; q < 16; q++) {
                nv[q] = q < nvalid ? r.nrm[n + q] : 0.f;
                jv[q] = q < nvalid ? jvalid[n + q] : 0;
            }
        }
        float mn = INFINITY;
#pragma unroll
        for (int q = 0; q < 16; q++) {
            if (q >= nvalid) break;
            bool ok = jv[q] != 0;
            if (ok && r.mc) ok = r.mc[(long)((n + q) / nor) * ntr] != 0;
            const float val = !ok  ? INFINITY
                              : ccx ? (float)(-(double)v[q] / (sqrt((double)nv[q]) * r.rc))
                                    : (float)(0.5 * ((double)nv[q] - 2.0 * (double)v[q] + r.rc));
            diff2[r.out + (long)(n + q) * T] = val;
            mn = fminf(mn, val);
        }
        return mn;
    }
};

}  // namespace rome
