// Restricted (proposal) search of the MAP2D E-step: every particle is
// compared with its own list of orientations only (a learned proposal or any
// caller-chosen subset), with every translation.  The rows are ragged in the
// same sense as the 3D fine pass: row i holds nprop * T hypotheses in the
// order (proposal q ascending in orientation, translation), which is the
// reference's loop order (class -> psi -> trans) restricted to the subset.
#pragma once

#include <cuda_bf16.h>

#include "estep_kernels.cuh"

namespace rome {
// internal linkage: every translation unit that launches these kernels gets its own copy
namespace {

constexpr int RS_THREADS = 256, RS_TQ = 32, RS_QQ = 128, RS_KC = 32;

template <int PREC>
__device__ __forceinline__ float op_load(const void* base, long plane, long idx) {
    if (PREC == ROME_PREC_FP32) return ((const float*)base)[idx];
    const __nv_bfloat16* h = (const __nv_bfloat16*)base;
    float v = __bfloat162float(h[idx]);
    if (PREC == ROME_PREC_BF16X3) v += __bfloat162float(h[plane + idx]);
    return v;
}

// One CTA per (32 translations, 128 proposals, particle): the cross term as a
// register-tiled FP32 product (4 x 4 outputs per thread) of the particle's
// translation rows A[i*T + t] with the gathered orientation rows B[j], plus
// the norm term N_j = <W2_i, Q_j>; diff2 = (N - 2 C + S + Xi2) / 2 at
// [i][q * T + t] (+inf for orientations the reference would skip), and the
// per-particle minimum folded in.  Operands: FP32 or BF16 (hi, + lo for
// the split mode) as the dense contraction stores them.
template <int PREC>
__global__ void __launch_bounds__(RS_THREADS)
    restricted_diff2_kernel(int T, int Kp, int Kq, int nprop, long Mrows, long Jrows, const int* __restrict__ prop,
                            const int* __restrict__ jvalid, const void* __restrict__ A, const void* __restrict__ B,
                            const float* __restrict__ W2, const float* __restrict__ Q, const float* __restrict__ S,
                            const double* __restrict__ xi2, long Xr, float* __restrict__ diff2,
                            unsigned* __restrict__ rowmin) {
    __shared__ float As[RS_TQ][RS_KC + 1];
    __shared__ float Bs[RS_QQ][RS_KC + 1];
    __shared__ float Nq[RS_QQ];
    __shared__ int jq[RS_QQ];
    const int q0 = blockIdx.x * RS_QQ, t0 = blockIdx.y * RS_TQ, i = blockIdx.z;
    const int tid = threadIdx.x, tx = tid % 8, ty = tid / 8;
    for (int q = tid; q < RS_QQ; q += RS_THREADS) jq[q] = q0 + q < nprop ? prop[(long)i * nprop + q0 + q] : -1;
    __syncthreads();
    // norm term of each proposal: one warp per proposal at a time
    {
        const int warp = tid >> 5, lane = tid & 31;
        const float* w2 = W2 + (long)i * Kq;
        for (int q = warp; q < RS_QQ; q += RS_THREADS / 32) {
            float s = 0.f;
            if (jq[q] >= 0) {
                const float* qr = Q + (long)jq[q] * Kq;
                for (int a = lane; a < Kq; a += 32) s = fmaf(w2[a], qr[a], s);
            }
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
            if (lane == 0) Nq[q] = s;
        }
    }
    float acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = 0.f;
    const long arow0 = (long)i * T;
    for (int k0 = 0; k0 < Kp; k0 += RS_KC) {
        __syncthreads();
        for (int e = tid; e < RS_TQ * RS_KC; e += RS_THREADS) {
            const int r = e / RS_KC, c = e - r * RS_KC;
            const int t = t0 + r;
            As[r][c] = t < T ? op_load<PREC>(A, Mrows * Kp, (arow0 + t) * Kp + k0 + c) : 0.f;
        }
        for (int e = tid; e < RS_QQ * RS_KC; e += RS_THREADS) {
            const int r = e / RS_KC, c = e - r * RS_KC;
            const int j = jq[r];
            Bs[r][c] = j >= 0 ? op_load<PREC>(B, Jrows * Kp, (long)j * Kp + k0 + c) : 0.f;
        }
        __syncthreads();
#pragma unroll 8
        for (int k = 0; k < RS_KC; k++) {
            float a[4], b[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                a[u] = As[tx * 4 + u][k];
                b[u] = Bs[ty * 4 + u][k];
            }
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int v = 0; v < 4; v++) acc[u][v] = fmaf(a[u], b[v], acc[u][v]);
        }
    }
    float m = INFINITY;
    const double x2 = xi2[i];
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const int t = t0 + tx * 4 + u;
        if (t >= T) continue;
        const double s = (double)S[arow0 + t];
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const int ql = ty * 4 + v, q = q0 + ql;
            if (q >= nprop) continue;
            const int j = jq[ql];
            float d = INFINITY;
            if (jvalid[j]) d = (float)(0.5 * ((double)Nq[ql] - 2.0 * (double)acc[u][v] + s + x2));
            diff2[(long)i * Xr + (long)q * T + t] = d;
            m = fminf(m, d);
        }
    }
    for (int o = 16; o > 0; o >>= 1) m = fminf(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((tid & 31) == 0 && m < INFINITY) atomicMin(&rowmin[i], float_key(m));
}

// prior index of every proposal for the posterior: (pdf_direction index =
// class, translation taken from the hypothesis' position in the row)
__global__ void restricted_entries_kernel(long n, int nrot, const int* __restrict__ prop, int2* __restrict__ ent) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) ent[q] = make_int2(prop[q] / nrot, -1);
}

// significant hypotheses re-indexed from the row position q * T + t to the
// dense position j * T + t used by the wsum and back-projection kernels
__global__ void restricted_list_dense_kernel(int n, int T, int nprop, const int* __restrict__ prop,
                                             SigEntry* __restrict__ list) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    SigEntry s = list[q];
    const int r = s.e / T, t = s.e - r * T;
    s.e = prop[(long)s.i * nprop + r] * T + t;
    list[q] = s;
}

// the last pass's significant normalised weights summed per (class, psi):
// marg[i][j / nor] += w for dense hypothesis e = j * T + t
__global__ void post_marginal_kernel(int n, int T, int nor, int npk, const SigEntry* __restrict__ list,
                                     double* __restrict__ marg) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const SigEntry s = list[q];
    atomicAdd(&marg[(long)s.i * npk + (s.e / T) / nor], s.w);
}

}  // namespace
}  // namespace rome
