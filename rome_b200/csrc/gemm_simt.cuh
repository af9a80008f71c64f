// CUDA-core FP32 GEMM with a fused epilogue: C[m][n] = sum_k A[m][k] * B[n][k].
// Both operands are K-contiguous ("TN").  This is the plain-FP32 path of the
// diff2 cross term and of the small norm-term contraction.
//
// Tile 128 x 128 x 16, 256 threads, 8 x 8 outputs per thread, two shared
// memory stages with register prefetch of the next K slice.  K must be a
// multiple of 16 (operands are zero-padded); M and N are bounds-checked.
#pragma once

#include <cuda_runtime.h>

namespace rome {
// internal linkage: every translation unit that launches these kernels gets its own copy
namespace {

constexpr int SG_BM = 128, SG_BN = 128, SG_BK = 16, SG_THREADS = 256;

template <typename Epi>
__global__ void __launch_bounds__(SG_THREADS, 2)
    sgemm_tn_kernel(int M, int N, int K, const float* __restrict__ A, long lda, const float* __restrict__ B, long ldb,
                    Epi epi) {
    __shared__ __align__(16) float As[2][SG_BK][SG_BM + 4];
    __shared__ __align__(16) float Bs[2][SG_BK][SG_BN + 4];
    const int tid = threadIdx.x;
    const int tx = tid % 16, ty = tid / 16;
    const int m0 = blockIdx.y * SG_BM, n0 = blockIdx.x * SG_BN;

    // global -> register staging: each thread moves 2 float4 of A and of B
    const int lr = tid / 4, lk = (tid % 4) * 4;
    float4 ra[2], rb[2];
    auto load_regs = [&](int k0) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            int r = lr + h * 64;
            int gm = m0 + r, gn = n0 + r;
            ra[h] = (gm < M) ? *reinterpret_cast<const float4*>(A + (long)gm * lda + k0 + lk) : make_float4(0, 0, 0, 0);
            rb[h] = (gn < N) ? *reinterpret_cast<const float4*>(B + (long)gn * ldb + k0 + lk) : make_float4(0, 0, 0, 0);
        }
    };
    auto store_smem = [&](int s) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            int r = lr + h * 64;
            As[s][lk + 0][r] = ra[h].x;
            As[s][lk + 1][r] = ra[h].y;
            As[s][lk + 2][r] = ra[h].z;
            As[s][lk + 3][r] = ra[h].w;
            Bs[s][lk + 0][r] = rb[h].x;
            Bs[s][lk + 1][r] = rb[h].y;
            Bs[s][lk + 2][r] = rb[h].z;
            Bs[s][lk + 3][r] = rb[h].w;
        }
    };

    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = 0.f;

    const int nk = K / SG_BK;
    load_regs(0);
    store_smem(0);
    __syncthreads();
    for (int kt = 0; kt < nk; kt++) {
        const int s = kt & 1;
        if (kt + 1 < nk) load_regs((kt + 1) * SG_BK);
#pragma unroll
        for (int k = 0; k < SG_BK; k++) {
            float a[8], b[8];
            float4 t;
            t = *reinterpret_cast<const float4*>(&As[s][k][ty * 4]);
            a[0] = t.x; a[1] = t.y; a[2] = t.z; a[3] = t.w;
            t = *reinterpret_cast<const float4*>(&As[s][k][64 + ty * 4]);
            a[4] = t.x; a[5] = t.y; a[6] = t.z; a[7] = t.w;
            t = *reinterpret_cast<const float4*>(&Bs[s][k][tx * 4]);
            b[0] = t.x; b[1] = t.y; b[2] = t.z; b[3] = t.w;
            t = *reinterpret_cast<const float4*>(&Bs[s][k][64 + tx * 4]);
            b[4] = t.x; b[5] = t.y; b[6] = t.z; b[7] = t.w;
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 8; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        if (kt + 1 < nk) {
            store_smem(s ^ 1);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
        int m = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4);
        if (m >= M) continue;
        float rmin = INFINITY;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            int n = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + j - 4);
            if (n < N) rmin = fminf(rmin, epi(m, n, acc[i][j]));
        }
        epi.finish_row(m, rmin);
    }
}

template <typename Epi>
inline void sgemm_tn(cudaStream_t st, int M, int N, int K, const float* A, long lda, const float* B, long ldb, Epi epi) {
    if (M <= 0 || N <= 0) return;
    dim3 grid((N + SG_BN - 1) / SG_BN, (M + SG_BM - 1) / SG_BM);
    sgemm_tn_kernel<Epi><<<grid, SG_THREADS, 0, st>>>(M, N, K, A, lda, B, ldb, epi);
}

}  // namespace
}  // namespace rome
