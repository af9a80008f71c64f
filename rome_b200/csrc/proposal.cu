// Learned pose proposals for the MAP E-step (no counterpart in the
// reference): a small network over a particle's Fourier magnitude in polar
// coordinates predicts a distribution over (class, psi mod 180 deg); it is
// trained on the GPU on (image, posterior) pairs produced by the exhaustive
// E-step itself, with hand-written FP32 forward, backward and Adam kernels.
// Its top-k (class, psi) pairs (each psi with psi + 180, which the magnitude
// cannot tell apart) restrict the E-step's search; the exhaustive E-step
// stays the fallback and the judge.
//
// In polar coordinates an in-plane rotation is a circular shift along the
// angle axis, and every layer is equivariant to that shift, so one set of
// weights serves all psi (a first design, a plain CNN with a dense head,
// generalised poorly: it had to learn every rotation of every class
// separately):
//   x[N][2][R][A]  log(1+|X|), |CTF| at R radii x A = nr_psi/2 angles in [0, 180)
//   conv3x3 (2 -> c0) + ReLU, conv3x3 (c0 -> c1) + ReLU   (r: zero pad, theta: circular)
//   z[n][k][p] = bf[k] + sum_{c,r,d} wf[k][c][r][d] h[n][c][r][(d - p) mod A]
//   loss = mean_n sum -t log softmax(z[n])  (soft targets: the E-step posterior)
// Parameters: one flat FP32 array w0 b0 w1 b1 wf bf, each block at a multiple
// of 4 floats.  The CPU restatement is oracle/proposal_oracle.py.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <random>
#include <vector>

#include <cuda_bf16.h>

#include "common.cuh"
#include "gemm_tc.cuh"

using namespace rome;

struct RomeProposalNet {
    RomeGpuCtx* ctx = nullptr;
    RomeProposalSpec spec{};
    int R = 0, A = 0, K = 0, c0 = 0, c1 = 0;
    long off[6] = {0};  // w0 b0 w1 b1 wf bf
    long nparam = 0;
    float* params = nullptr;
    float* grads = nullptr;
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    long adam_t = 0;
    int cap_n = 0;        // batch capacity
    float* x = nullptr;   // [N][2][R][A]
    float* h0 = nullptr;  // [N][c0][R][A]
    float* h1 = nullptr;  // [N][c1][R][A]
    float* dh0 = nullptr;
    float* dh1 = nullptr;
    float* z = nullptr;   // [N][K*A]
    float* dz = nullptr;
    float* tgt = nullptr;
    double* loss_acc = nullptr;
    int* idx = nullptr;
    // the head as tensor-core GEMMs (split-bf16 operands):
    //   z = h . WT^T,  WT[(k,p)][(c,r,d)] = wf[k][c][r][(d + p) mod A]
    int CRA = 0, CRAp = 0, KA = 0, KAp = 0;  // C*R*A and K*A, padded to multiples of 64
    void* wt = nullptr;                      // WT  [KA][CRAp] hi, lo
    void* wtt = nullptr;                     // WT^T [CRA][KAp] hi, lo
    float* dwt = nullptr;                    // dL/dWT [KA][CRA]
    bool wt_dirty = true;                    // parameters changed since WT was expanded
    void* hs = nullptr;                      // h1 [n][CRAp] hi, lo
    void* dzs = nullptr;                     // dz [n][KAp] hi, lo
    void* dzt = nullptr;                     // dz^T [KA][npad] hi, lo
    void* ht = nullptr;                      // h1^T [CRA][npad] hi, lo
    float* wflip = nullptr;                  // conv 2 weights flipped for its input gradient
    float* wpart = nullptr;                  // per-sample conv weight/bias gradients [n][Co*Ci*9 + Co]
};

namespace rome {
namespace {

constexpr int PT = 256;

// ---- 3x3 convolution on the polar grid: zero padding along r, circular along theta ----
__global__ void __launch_bounds__(PT) pconv_fwd_kernel(int Ci, int R, int A, int Co, const float* __restrict__ x,
                                                        const float* __restrict__ w, const float* __restrict__ b,
                                                        float* __restrict__ y) {
    extern __shared__ float sw[];  // Ci * 9 weights of this output channel
    const int co = blockIdx.y, n = blockIdx.z;
    for (int q = threadIdx.x; q < Ci * 9; q += PT) sw[q] = w[(long)co * Ci * 9 + q];
    __syncthreads();
    const int p = blockIdx.x * PT + threadIdx.x;
    if (p >= R * A) return;
    const int r = p / A, a = p - r * A;
    const float* xn = x + (long)n * Ci * R * A;
    float acc = b[co];
    for (int ci = 0; ci < Ci; ci++) {
        const float* xc = xn + (long)ci * R * A;
        const float* wc = sw + ci * 9;
#pragma unroll
        for (int kh = 0; kh < 3; kh++) {
            const int rr = r + kh - 1;
            if (rr < 0 || rr >= R) continue;
#pragma unroll
            for (int kw = 0; kw < 3; kw++) {
                int aa = a + kw - 1;
                aa = aa < 0 ? aa + A : (aa >= A ? aa - A : aa);
                acc = fmaf(wc[kh * 3 + kw], xc[rr * A + aa], acc);
            }
        }
    }
    y[(((long)n * Co + co) * R + r) * A + a] = fmaxf(acc, 0.f);
}

// The same convolution with one CTA per sample: the sample's input planes
// and the layer's weights ([ci][tap][co], 16-byte groups of 4 output
// channels) in shared memory; each thread item is 4 output channels at one
// (r, theta) position, consecutive threads at consecutive positions.  The
// taps are accumulated in the order of pconv_fwd_kernel (bias, then ci, kh,
// kw), so both give identical results.  Used when Co % 4 == 0 and the
// sample fits in shared memory (pconv_smem_bytes).
size_t pconv_smem_bytes(int Ci, int R, int A, int Co) {
    const size_t xin = ((size_t)Ci * R * A + 3) / 4 * 4;
    return sizeof(float) * (xin + (size_t)Ci * 9 * Co);
}

template <bool RELU>
__global__ void __launch_bounds__(PT) pconv_fwd_smem_kernel(int Ci, int R, int A, int Co,
                                                             const float* __restrict__ x,
                                                             const float* __restrict__ w,
                                                             const float* __restrict__ b, float* __restrict__ y) {
    // one sample per block, its input and the weights in shared memory; a
    // thread computes 4 output channels at 4 consecutive angles of one
    // radius, so each input value it loads feeds 12 multiply-adds
    extern __shared__ float4 sm4[];
    float* xs = (float*)sm4;
    const int RA = R * A, G = Co / 4, AB = (A + 3) / 4;
    float* ws = xs + ((long)Ci * RA + 3) / 4 * 4;
    const int n = blockIdx.x;
    const float* xn = x + (long)n * Ci * RA;
    for (int q = threadIdx.x; q < Ci * RA; q += PT) xs[q] = xn[q];
    for (int q = threadIdx.x; q < Co * Ci * 9; q += PT) {
        const int co = q / (Ci * 9), rest = q - co * (Ci * 9);
        ws[rest * Co + co] = w[q];
    }
    __syncthreads();
    for (int item = threadIdx.x; item < G * R * AB; item += PT) {
        const int g = item / (R * AB), rem = item - g * (R * AB);
        const int r = rem / AB, a0 = (rem - r * AB) * 4;
        // the 6 angles a0-1 .. a0+4, circular
        int ai[6];
#pragma unroll
        for (int u = 0; u < 6; u++) {
            int aa = a0 + u - 1;
            aa = aa < 0 ? aa + A : (aa >= A ? aa - A : aa);
            ai[u] = aa;
        }
        float acc[4][4];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const float bias = b ? b[4 * g + c] : 0.f;
#pragma unroll
            for (int p = 0; p < 4; p++) acc[c][p] = bias;
        }
        for (int ci = 0; ci < Ci; ci++) {
            const float* xc = xs + ci * RA;
            const float4* wc = (const float4*)(ws + (long)ci * 9 * Co) + g;
#pragma unroll
            for (int kh = 0; kh < 3; kh++) {
                const int rr = r + kh - 1;
                if (rr < 0 || rr >= R) continue;
                const float* row = xc + rr * A;
                float v[6];
#pragma unroll
                for (int u = 0; u < 6; u++) v[u] = row[ai[u]];
#pragma unroll
                for (int kw = 0; kw < 3; kw++) {
                    const float4 wv = wc[(kh * 3 + kw) * G];
#pragma unroll
                    for (int p = 0; p < 4; p++) {
                        acc[0][p] = fmaf(wv.x, v[p + kw], acc[0][p]);
                        acc[1][p] = fmaf(wv.y, v[p + kw], acc[1][p]);
                        acc[2][p] = fmaf(wv.z, v[p + kw], acc[2][p]);
                        acc[3][p] = fmaf(wv.w, v[p + kw], acc[3][p]);
                    }
                }
            }
        }
#pragma unroll
        for (int c = 0; c < 4; c++)
#pragma unroll
            for (int p = 0; p < 4; p++)
                if (a0 + p < A)
                    y[(((long)n * Co + 4 * g + c) * R + r) * A + a0 + p] = RELU ? fmaxf(acc[c][p], 0.f) : acc[c][p];
    }
}

// w'[ci][co][t] = w[co][ci][8 - t]: the input gradient of a 3x3 polar convolution
// is the same convolution of dy with these weights (channels swapped, taps flipped)
__global__ void flip_weights_kernel(int Co, int Ci, const float* __restrict__ w, float* __restrict__ wt) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= Co * Ci * 9) return;
    const int co = q / (Ci * 9), rest = q - co * (Ci * 9), ci = rest / 9, t = rest - ci * 9;
    wt[((long)ci * Co + co) * 9 + (8 - t)] = w[q];
}

// Weight and bias gradients of a 3x3 polar convolution, one CTA per sample:
// the sample's input planes (row stride R*A + 1 against bank conflicts) and
// output gradients in shared memory; thread -> (co, ci) pair, its 9 taps in
// registers.  part[n][(co*Ci + ci)*9 + t] and part[n][Co*Ci*9 + co] are the
// sample's contributions, summed over samples by conv_grad_reduce_kernel in a
// fixed order (deterministic).
size_t wgrad_smem_bytes(int Ci, int R, int A, int Co) {
    return sizeof(float) * ((size_t)Ci * (R * A + 1) + (size_t)Co * R * A);
}

__global__ void __launch_bounds__(PT) conv_wgrad_sample_kernel(int Ci, int R, int A, int Co,
                                                                const float* __restrict__ x,
                                                                const float* __restrict__ dy,
                                                                float* __restrict__ part) {
    extern __shared__ float smw[];
    const int RA = R * A, XS = RA + 1;
    float* xs = smw;
    float* gs = smw + (long)Ci * XS;
    const int n = blockIdx.x;
    for (int q = threadIdx.x; q < Ci * RA; q += PT) {
        const int c = q / RA;
        xs[c * XS + (q - c * RA)] = x[(long)n * Ci * RA + q];
    }
    for (int q = threadIdx.x; q < Co * RA; q += PT) gs[q] = dy[(long)n * Co * RA + q];
    __syncthreads();
    const long stride = (long)Co * Ci * 9 + Co;
    for (int pr = threadIdx.x; pr < Co * Ci; pr += PT) {
        const int co = pr / Ci, ci = pr - co * Ci;
        const float* xc = xs + ci * XS;
        const float* gc = gs + co * RA;
        float acc[9];
#pragma unroll
        for (int t = 0; t < 9; t++) acc[t] = 0.f;
        for (int r = 0; r < R; r++) {
            for (int a = 0; a < A; a++) {
                const float g = gc[r * A + a];
                const int am = a == 0 ? A - 1 : a - 1, ap = a == A - 1 ? 0 : a + 1;
#pragma unroll
                for (int kh = 0; kh < 3; kh++) {
                    const int rr = r + kh - 1;
                    if (rr < 0 || rr >= R) continue;
                    const float* row = xc + rr * A;
                    acc[kh * 3 + 0] = fmaf(g, row[am], acc[kh * 3 + 0]);
                    acc[kh * 3 + 1] = fmaf(g, row[a], acc[kh * 3 + 1]);
                    acc[kh * 3 + 2] = fmaf(g, row[ap], acc[kh * 3 + 2]);
                }
            }
        }
#pragma unroll
        for (int t = 0; t < 9; t++) part[n * stride + (long)pr * 9 + t] = acc[t];
    }
    for (int co = threadIdx.x; co < Co; co += PT) {
        float sacc = 0.f;
        for (int q = 0; q < RA; q++) sacc += gs[co * RA + q];
        part[n * stride + (long)Co * Ci * 9 + co] = sacc;
    }
}

// out[j] = sum_n part[n][j] (n ascending), j < Co*Ci*9 -> dw, then Co biases -> db
__global__ void conv_grad_reduce_kernel(int N, int nw, int nb, const float* __restrict__ part, float* __restrict__ dw,
                                        float* __restrict__ db) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nw + nb) return;
    float s = 0.f;
    for (int n = 0; n < N; n++) s += part[(long)n * (nw + nb) + j];
    if (j < nw) dw[j] = s;
    else db[j - nw] = s;
}

// dy <- dy * (y > 0): the ReLU's gradient, in place
__global__ void relu_mask_kernel(long n, const float* __restrict__ y, float* __restrict__ dy) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n && !(y[q] > 0.f)) dy[q] = 0.f;
}

// dx[n][ci][r][a] = sum_co sum_taps w[co][ci][kh][kw] dy[n][co][r + 1 - kh][(a + 1 - kw) mod A]
__global__ void __launch_bounds__(PT) pconv_bwd_data_kernel(int Ci, int R, int A, int Co, const float* __restrict__ dy,
                                                             const float* __restrict__ w, float* __restrict__ dx) {
    const int ci = blockIdx.y, n = blockIdx.z;
    const int p = blockIdx.x * PT + threadIdx.x;
    if (p >= R * A) return;
    const int r = p / A, a = p - r * A;
    float acc = 0.f;
    for (int kh = 0; kh < 3; kh++) {
        const int ro = r + 1 - kh;
        if (ro < 0 || ro >= R) continue;
        for (int kw = 0; kw < 3; kw++) {
            int ao = a + 1 - kw;
            ao = ao < 0 ? ao + A : (ao >= A ? ao - A : ao);
            const float* dyp = dy + (long)n * Co * R * A + (long)ro * A + ao;
            const float* wp = w + (long)ci * 9 + kh * 3 + kw;
            for (int co = 0; co < Co; co++) acc = fmaf(wp[(long)co * Ci * 9], dyp[(long)co * R * A], acc);
        }
    }
    dx[(((long)n * Ci + ci) * R + r) * A + a] = acc;
}

template <typename T>
__device__ T block_sum(T v, T* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    T r = 0;
    if (threadIdx.x < 32) {
        r = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : (T)0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    return r;  // valid in thread 0
}

// dw[co][ci][kh][kw] = sum_{n,r,a} dy[n][co][r][a] x[n][ci][r + kh - 1][(a + kw - 1) mod A]
__global__ void __launch_bounds__(PT) pconv_bwd_weight_kernel(int N, int Ci, int R, int A, int Co,
                                                               const float* __restrict__ x, const float* __restrict__ dy,
                                                               float* __restrict__ dw) {
    __shared__ float sh[32];
    const int co = blockIdx.x, ci = blockIdx.y;
    float acc[9];
#pragma unroll
    for (int k = 0; k < 9; k++) acc[k] = 0.f;
    const long tot = (long)N * R * A;
    for (long q = threadIdx.x; q < tot; q += PT) {
        const int n = (int)(q / (R * A));
        const int p = (int)(q - (long)n * R * A);
        const int r = p / A, a = p - r * A;
        const float g = dy[((long)n * Co + co) * R * A + p];
        if (g == 0.f) continue;
        const float* xc = x + ((long)n * Ci + ci) * R * A;
#pragma unroll
        for (int kh = 0; kh < 3; kh++) {
            const int rr = r + kh - 1;
            if (rr < 0 || rr >= R) continue;
#pragma unroll
            for (int kw = 0; kw < 3; kw++) {
                int aa = a + kw - 1;
                aa = aa < 0 ? aa + A : (aa >= A ? aa - A : aa);
                acc[kh * 3 + kw] = fmaf(g, xc[rr * A + aa], acc[kh * 3 + kw]);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const float v = block_sum(acc[k], sh);
        if (threadIdx.x == 0) dw[((long)co * Ci + ci) * 9 + k] = v;
    }
}

// db[c] = sum_{n, pixels} dy[n][c][.]
__global__ void __launch_bounds__(PT) bias_grad_kernel(int N, int C, int HW, const float* __restrict__ dy,
                                                        float* __restrict__ db) {
    __shared__ float sh[32];
    const int c = blockIdx.x;
    float acc = 0.f;
    for (long q = threadIdx.x; q < (long)N * HW; q += PT) {
        const int n = (int)(q / HW);
        acc += dy[((long)n * C + c) * HW + (q - (long)n * HW)];
    }
    const float v = block_sum(acc, sh);
    if (threadIdx.x == 0) db[c] = v;
}

// ---- equivariant head: circular correlation along theta, full over (c, r) ----
// z[n][k][p] = bf[k] + sum_{c,r,d} wf[k][c][r][d] h[n][c][r][(d - p) mod A]
//            = bf[k] + sum_{c,r,d'} h[n][c][r][d'] wf[k][c][r][(d' + p) mod A]
// i.e. z = h . WT^T with the rolled weight matrix WT[(k,p)][(c,r,d')]; the
// three products of forward and backward run as split-bf16 tcgen05 GEMMs.

// WT (transposed = 0: [KA][CRAp]) or WT^T (transposed = 1: [CRA][KAp]), split
// into bf16 hi and lo planes, zero padded
__global__ void head_expand_kernel(int K, int CR, int A, int ld, int rows, int transposed, const float* __restrict__ wf,
                                   __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long)rows * ld) return;
    const int row = (int)(q / ld), col = (int)(q - (long)row * ld);
    const int kp = transposed ? col : row, crd = transposed ? row : col;
    float v = 0.f;
    if (kp < K * A && crd < CR * A) {
        const int k = kp / A, p = kp - k * A, cr = crd / A, d = crd - cr * A;
        int dd = d + p;
        if (dd >= A) dd -= A;
        v = wf[((long)k * CR + cr) * A + dd];
    }
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    hi[q] = h;
    lo[q] = __float2bfloat16_rn(v - __bfloat162float(h));
}

// dwf[k][c][r][d] = sum_p dWT[(k,p)][(c,r,(d - p) mod A)]
__global__ void head_fold_kernel(int K, int CR, int A, const float* __restrict__ dwt, float* __restrict__ dwf) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long)K * CR * A) return;
    const int k = (int)(q / ((long)CR * A));
    const int crd = (int)(q - (long)k * CR * A), cr = crd / A, d = crd - cr * A;
    const long CRA = (long)CR * A;
    float acc = 0.f;
    int idx = d;  // (d - p) mod A at p = 0
    for (int p = 0; p < A; p++) {
        acc += dwt[((long)k * A + p) * CRA + (long)cr * A + idx];
        if (--idx < 0) idx = A - 1;
    }
    dwf[q] = acc;
}

// per sample: p = softmax(z), loss += -sum t log p, dz = (p - t) / N
__global__ void __launch_bounds__(PT) softmax_xent_kernel(int N, int O, const float* __restrict__ z,
                                                           const float* __restrict__ t, float* __restrict__ dz,
                                                           double* __restrict__ loss) {
    __shared__ float shf[32];
    __shared__ double shd[32];
    __shared__ float s_max, s_sum;
    const int n = blockIdx.x;
    const float* zn = z + (long)n * O;
    float m = -INFINITY;
    for (int o = threadIdx.x; o < O; o += PT) m = fmaxf(m, zn[o]);
    for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31) == 0) shf[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        float mm = shf[0];
        for (int q = 1; q < PT / 32; q++) mm = fmaxf(mm, shf[q]);
        s_max = mm;
    }
    __syncthreads();
    float se = 0.f;
    for (int o = threadIdx.x; o < O; o += PT) se += __expf(zn[o] - s_max);
    se = block_sum(se, shf);
    if (threadIdx.x == 0) s_sum = se;
    __syncthreads();
    const float lse = s_max + logf(s_sum);
    double l = 0.0;
    for (int o = threadIdx.x; o < O; o += PT) {
        const float tv = t[(long)n * O + o];
        const float lp = zn[o] - lse;
        l -= (double)tv * (double)lp;
        if (dz) dz[(long)n * O + o] = (__expf(lp) - tv) / (float)N;
    }
    l = block_sum(l, shd);
    if (threadIdx.x == 0 && loss) atomicAdd(loss, l / N);
}

__global__ void adam_kernel(long n, float lr, float b1, float b2, float eps, float c1, float c2,
                            const float* __restrict__ g, float* __restrict__ p, float* __restrict__ m,
                            float* __restrict__ v) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const float gq = g[q];
    const float mq = b1 * m[q] + (1.f - b1) * gq;
    const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    p[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
}

__global__ void gather_rows_kernel(int n, long row, const int* __restrict__ idx, const float* __restrict__ src,
                                   float* __restrict__ dst) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long)n * row) return;
    const int r = (int)(q / row);
    dst[q] = src[(long)idx[r] * row + (q - (long)r * row)];
}

// Network input of one particle (oracle/proposal_oracle.py features()):
// bilinear samples of log(1 + |X|) and |CTF| on the polar grid r_i = r_lo +
// i (r_hi - r_lo) / (R - 1), theta_a = a pi / A (negative kx by Friedel
// symmetry), each channel normalised to zero mean and unit variance.
__device__ __forceinline__ double half_plane_at(const double* v, int cur, int cf, int x, int y, bool logmag,
                                                const double* vi) {
    if (x < 0) {
        x = -x;
        y = -y;
    }
    const int row = y >= 0 ? y : y + cur;
    const long e = (long)row * cf + x;
    if (logmag) return log1p(sqrt(v[e] * v[e] + vi[e] * vi[e]));
    return fabs(v[e]);
}

__global__ void __launch_bounds__(PT) polar_features_kernel(int cur, int R, int A, double r_lo, double r_hi,
                                                             const double* __restrict__ Fr,
                                                             const double* __restrict__ Fi,
                                                             const double* __restrict__ ctf, float* __restrict__ x) {
    extern __shared__ float sx[];  // 2 * R * A
    __shared__ double shd[32];
    __shared__ double s_mean[2], s_std[2];
    const int i = blockIdx.x, cf = cur / 2 + 1, n2 = R * A;
    const long base = (long)i * cur * cf;
    const double kPiD = 3.14159265358979323846;
    for (int q = threadIdx.x; q < n2; q += PT) {
        const int ri = q / A, a = q - ri * A;
        const double r = r_lo + ri * (r_hi - r_lo) / (R - 1);
        const double th = a * kPiD / A;
        const double kx = r * cos(th), ky = r * sin(th);
        const int x0 = (int)floor(kx), y0 = (int)floor(ky);
        const double fx = kx - x0, fy = ky - y0;
        for (int c = 0; c < 2; c++) {
            const double* v = c == 0 ? Fr + base : ctf + base;
            const double* vi = Fi + base;
            const bool lm = c == 0;
            const double v00 = half_plane_at(v, cur, cf, x0, y0, lm, vi);
            const double v01 = half_plane_at(v, cur, cf, x0 + 1, y0, lm, vi);
            const double v10 = half_plane_at(v, cur, cf, x0, y0 + 1, lm, vi);
            const double v11 = half_plane_at(v, cur, cf, x0 + 1, y0 + 1, lm, vi);
            sx[c * n2 + q] = (float)((1 - fy) * ((1 - fx) * v00 + fx * v01) + fy * ((1 - fx) * v10 + fx * v11));
        }
    }
    __syncthreads();
    for (int c = 0; c < 2; c++) {
        double s = 0.0, ss = 0.0;
        for (int q = threadIdx.x; q < n2; q += PT) s += sx[c * n2 + q];
        s = block_sum(s, shd);
        if (threadIdx.x == 0) s_mean[c] = s / n2;
        __syncthreads();
        for (int q = threadIdx.x; q < n2; q += PT) {
            const double d = sx[c * n2 + q] - s_mean[c];
            ss += d * d;
        }
        ss = block_sum(ss, shd);
        if (threadIdx.x == 0) s_std[c] = fmax(sqrt(ss / n2), 1e-12);
        __syncthreads();
    }
    for (int q = threadIdx.x; q < 2 * n2; q += PT) {
        const int c = q / n2;
        x[(long)i * 2 * n2 + q] = (float)((sx[q] - s_mean[c]) / s_std[c]);
    }
}

// top-k of each row of logits (descending; ties by lower index), with the
// softmax probability of each.  One warp per row and no sort: k rounds of a warp
// argmax over the row, each round restricted to the elements after the
// previous pick in the order (value descending, index ascending), which
// excludes every earlier pick.  The row is read from L1/L2 each round.
__global__ void __launch_bounds__(PT) topk_warp_kernel(int n, int O, int k, const float* __restrict__ z,
                                                        int* __restrict__ idx, float* __restrict__ prob) {
    const int row = (int)(((long)blockIdx.x * PT + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (row >= n) return;  // whole warps leave together
    const float* zr = z + (long)row * O;
    float pv = INFINITY, mx = 0.f, sum = 0.f;
    int pi = -1;
    for (int q = 0; q < k; q++) {
        float bv = -INFINITY;
        int bi = INT_MAX;
        for (int o = lane; o < O; o += 32) {
            const float v = __ldg(zr + o);
            const bool below = v < pv || (v == pv && o > pi);
            const bool better = v > bv || (v == bv && o < bi);
            if (below && better) {
                bv = v;
                bi = o;
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const float ov = __shfl_xor_sync(0xffffffffu, bv, off);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
            if (ov > bv || (ov == bv && oi < bi)) {
                bv = ov;
                bi = oi;
            }
        }
        if (q == 0) {
            mx = bv;
            float se = 0.f;
            for (int o = lane; o < O; o += 32) se += __expf(__ldg(zr + o) - mx);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) se += __shfl_xor_sync(0xffffffffu, se, off);
            sum = se;
        }
        if (lane == 0) {
            idx[(long)row * k + q] = bi;
            if (prob) prob[(long)row * k + q] = __expf(bv - mx) / sum;
        }
        pv = bv;
        pi = bi;
    }
}

// network outputs o = class * A + p (top-k per particle) -> the 2k
// orientations class * 2A + p and class * 2A + p + A, sorted ascending
// (the restricted E-step wants ascending, distinct lists); one thread per
// particle, insertion sort of at most 2 * 64 entries
__global__ void expand_proposals_kernel(int P, int k, int A, const int* __restrict__ idx,
                                        const float* __restrict__ prob, int* __restrict__ prop,
                                        float* __restrict__ mass) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    int* out = prop + (long)i * 2 * k;
    float m = 0.f;
    int n = 0;
    for (int q = 0; q < k; q++) {
        const int o = idx[(long)i * k + q];
        m += prob[(long)i * k + q];
        const int c = o / A, p = o - c * A;
        for (int h = 0; h < 2; h++) {
            const int j = c * 2 * A + p + h * A;
            int pos = n++;
            while (pos > 0 && out[pos - 1] > j) {
                out[pos] = out[pos - 1];
                pos--;
            }
            out[pos] = j;
        }
    }
    if (mass) mass[i] = m;
}

void net_alloc_batch(RomeProposalNet* net, int n) {
    if (n <= net->cap_n) return;
    const size_t ra = (size_t)net->R * net->A, O = (size_t)net->K * net->A;
    for (float** p : {&net->x, &net->h0, &net->h1, &net->dh0, &net->dh1, &net->z, &net->dz, &net->tgt})
        if (*p) cudaFree(*p);
    for (void** p : {&net->hs, &net->dzs, &net->dzt, &net->ht})
        if (*p) cudaFree(*p);
    ROME_CUDA(cudaMalloc(&net->x, sizeof(float) * n * 2 * ra));
    ROME_CUDA(cudaMalloc(&net->h0, sizeof(float) * n * net->c0 * ra));
    ROME_CUDA(cudaMalloc(&net->dh0, sizeof(float) * n * net->c0 * ra));
    ROME_CUDA(cudaMalloc(&net->h1, sizeof(float) * n * net->c1 * ra));
    ROME_CUDA(cudaMalloc(&net->dh1, sizeof(float) * n * net->c1 * ra));
    for (float** p : {&net->z, &net->dz, &net->tgt}) ROME_CUDA(cudaMalloc(p, sizeof(float) * n * O));
    const size_t npad = (size_t)(n + 63) / 64 * 64;
    ROME_CUDA(cudaMalloc(&net->hs, 4 * (size_t)n * net->CRAp));
    ROME_CUDA(cudaMalloc(&net->dzs, 4 * (size_t)n * net->KAp));
    ROME_CUDA(cudaMalloc(&net->dzt, 4 * (size_t)net->KA * npad));
    ROME_CUDA(cudaMalloc(&net->ht, 4 * (size_t)net->CRA * npad));
    if (net->idx) cudaFree(net->idx);
    ROME_CUDA(cudaMalloc(&net->idx, sizeof(int) * n));
    if (net->wpart) cudaFree(net->wpart);
    const size_t per = std::max((size_t)net->c1 * net->c0 * 9 + net->c1, (size_t)net->c0 * 2 * 9 + net->c0);
    ROME_CUDA(cudaMalloc(&net->wpart, sizeof(float) * per * n));
    net->cap_n = n;
}

// WT and WT^T from the current head weights (after every parameter change)
void net_expand_head(RomeProposalNet* net, cudaStream_t st) {
    if (!net->wt_dirty) return;
    const int CR = net->c1 * net->R;
    const float* wf = net->params + net->off[4];
    const long n1 = (long)net->KA * net->CRAp, n2 = (long)net->CRA * net->KAp;
    __nv_bfloat16* w1 = (__nv_bfloat16*)net->wt;
    __nv_bfloat16* w2 = (__nv_bfloat16*)net->wtt;
    head_expand_kernel<<<(unsigned)((n1 + PT - 1) / PT), PT, 0, st>>>(net->K, CR, net->A, net->CRAp, net->KA, 0, wf,
                                                                     w1, w1 + n1);
    head_expand_kernel<<<(unsigned)((n2 + PT - 1) / PT), PT, 0, st>>>(net->K, CR, net->A, net->KAp, net->CRA, 1, wf,
                                                                     w2, w2 + n2);
    ROME_CHECK_LAUNCH();
    net->ctx->total_launches += 2;
    net->wt_dirty = false;
}

// Raise a kernel's dynamic shared memory limit to its cap, once.  The limit
// is a property of the function shared by every host thread; setting it to
// each launch's own size would let one thread lower it between another
// thread's set and launch, so it is only ever raised, to the cap the launch
// sites check against.
void raise_smem_limit(const void* fn, int bytes) {
    static std::mutex mu;
    static std::map<const void*, int> limit;
    std::lock_guard<std::mutex> g(mu);
    int& cur = limit[fn];
    if (cur >= bytes) return;
    ROME_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    cur = bytes;
}

// one 3x3 polar convolution + ReLU over n samples
void conv_forward(int Ci, int R, int A, int Co, int n, const float* x, const float* w, const float* b, float* y,
                  cudaStream_t st) {
    const size_t sm = pconv_smem_bytes(Ci, R, A, Co);
    if (Co % 4 == 0 && sm <= 96 * 1024) {
        raise_smem_limit((const void*)pconv_fwd_smem_kernel<true>, 96 * 1024);
        pconv_fwd_smem_kernel<true><<<n, PT, sm, st>>>(Ci, R, A, Co, x, w, b, y);
    } else {
        dim3 g((R * A + PT - 1) / PT, Co, n);
        pconv_fwd_kernel<<<g, PT, sizeof(float) * Ci * 9, st>>>(Ci, R, A, Co, x, w, b, y);
    }
    ROME_CHECK_LAUNCH();
}

// split: the head contraction in split BF16 (training: gradients checked
// against the FP64 oracle); otherwise one BF16 product (the proposals rank
// the outputs, the training loss does not see them)
void net_forward(RomeProposalNet* net, int n, cudaStream_t st, bool split = true) {
    const int R = net->R, A = net->A;
    const float* P = net->params;
    conv_forward(2, R, A, net->c0, n, net->x, P + net->off[0], P + net->off[1], net->h0, st);
    conv_forward(net->c0, R, A, net->c1, n, net->h0, P + net->off[2], P + net->off[3], net->h1, st);
    net_expand_head(net, st);
    split_bf16(st, net->h1, n, net->CRA, net->CRA, net->CRAp, net->hs, split);
    tc_bias_gemm(st, n, net->KA, net->CRAp, net->hs, net->wt, net->z, net->KA, net->params + net->off[5], A,
                 net->ctx->d_err, split);
    net->ctx->total_launches += 4;
}

// weight and bias gradients of one convolution (Ci -> Co) over n samples
void conv_weight_grads(RomeProposalNet* net, int n, int Ci, int Co, const float* x, const float* dy, float* dw,
                       float* db, cudaStream_t st) {
    const int R = net->R, A = net->A;
    const size_t sm = wgrad_smem_bytes(Ci, R, A, Co);
    if (sm <= 200 * 1024) {
        const int nw = Co * Ci * 9, nb = Co;
        raise_smem_limit((const void*)conv_wgrad_sample_kernel, 200 * 1024);
        conv_wgrad_sample_kernel<<<n, PT, sm, st>>>(Ci, R, A, Co, x, dy, net->wpart);
        conv_grad_reduce_kernel<<<(nw + nb + PT - 1) / PT, PT, 0, st>>>(n, nw, nb, net->wpart, dw, db);
    } else {
        pconv_bwd_weight_kernel<<<dim3(Co, Ci), PT, 0, st>>>(n, Ci, R, A, Co, x, dy, dw);
        bias_grad_kernel<<<Co, PT, 0, st>>>(n, Co, R * A, dy, db);
    }
    ROME_CHECK_LAUNCH();
}

// gradients of the mean loss into net->grads (dz holds dL/dz)
void net_backward(RomeProposalNet* net, int n, cudaStream_t st) {
    const int R = net->R, A = net->A, CR = net->c1 * R;
    const int npad = (n + 63) / 64 * 64;
    // head: dWT = dz^T . h (folded into dwf), dbf = sum dz, dh = dz . WT
    split_bf16_t(st, net->dz, n, net->KA, net->KA, npad, net->dzt);
    split_bf16_t(st, net->h1, n, net->CRA, net->CRA, npad, net->ht);
    tc_store_gemm(st, net->KA, net->CRA, npad, net->dzt, net->ht, net->dwt, net->CRA, net->ctx->d_err);
    const long nw = (long)net->K * CR * A;
    head_fold_kernel<<<(unsigned)((nw + PT - 1) / PT), PT, 0, st>>>(net->K, CR, A, net->dwt, net->grads + net->off[4]);
    bias_grad_kernel<<<net->K, PT, 0, st>>>(n, net->K, A, net->dz, net->grads + net->off[5]);
    ROME_CHECK_LAUNCH();
    split_bf16(st, net->dz, n, net->KA, net->KA, net->KAp, net->dzs);
    tc_store_gemm(st, n, net->CRA, net->KAp, net->dzs, net->wtt, net->dh1, net->CRA, net->ctx->d_err);
    net->ctx->total_launches += 7;
    const long n1 = (long)n * net->c1 * R * A, n0 = (long)n * net->c0 * R * A;
    relu_mask_kernel<<<(unsigned)((n1 + PT - 1) / PT), PT, 0, st>>>(n1, net->h1, net->dh1);
    conv_weight_grads(net, n, net->c0, net->c1, net->h0, net->dh1, net->grads + net->off[2], net->grads + net->off[3],
                      st);
    // input gradient of conv 2 = conv of dh1 with the flipped, transposed weights
    const size_t smd = pconv_smem_bytes(net->c1, R, A, net->c0);
    if (net->c0 % 4 == 0 && smd <= 96 * 1024) {
        flip_weights_kernel<<<(net->c1 * net->c0 * 9 + PT - 1) / PT, PT, 0, st>>>(net->c1, net->c0,
                                                                              net->params + net->off[2], net->wflip);
        raise_smem_limit((const void*)pconv_fwd_smem_kernel<false>, 96 * 1024);
        pconv_fwd_smem_kernel<false><<<n, PT, smd, st>>>(net->c1, R, A, net->c0, net->dh1, net->wflip, nullptr,
                                                         net->dh0);
    } else {
        dim3 g0((R * A + PT - 1) / PT, net->c0, n);
        pconv_bwd_data_kernel<<<g0, PT, 0, st>>>(net->c0, R, A, net->c1, net->dh1, net->params + net->off[2],
                                                 net->dh0);
    }
    relu_mask_kernel<<<(unsigned)((n0 + PT - 1) / PT), PT, 0, st>>>(n0, net->h0, net->dh0);
    conv_weight_grads(net, n, 2, net->c0, net->x, net->dh0, net->grads + net->off[0], net->grads + net->off[1], st);
    ROME_CHECK_LAUNCH();
}

void net_loss_grad(RomeProposalNet* net, int n, cudaStream_t st) {
    ROME_CUDA(cudaMemsetAsync(net->loss_acc, 0, sizeof(double), st));
    net_forward(net, n, st);
    softmax_xent_kernel<<<n, PT, 0, st>>>(n, net->K * net->A, net->z, net->tgt, net->dz, net->loss_acc);
    ROME_CHECK_LAUNCH();
    net_backward(net, n, st);
}

}  // namespace
}  // namespace rome

extern "C" int rome_gpu_proposal_create(RomeGpuCtx* ctx, const RomeProposalSpec* spec, unsigned long long seed,
                                        RomeProposalNet** out) {
    if (!ctx || !spec || !out) return ROME_ERR_ARG;
    *out = nullptr;
    return guarded(ctx, [&] {
        ROME_REQUIRE(spec->n_r >= 2 && spec->n_r <= 64, "n_r %d (2..64)", spec->n_r);
        ROME_REQUIRE(spec->n_theta >= 4 && spec->n_theta <= 256, "n_theta %d (4..256)", spec->n_theta);
        ROME_REQUIRE(spec->n_classes > 0 && spec->n_classes * spec->n_theta <= 8192, "n_classes %d", spec->n_classes);
        ROME_REQUIRE(spec->channels[0] > 0 && spec->channels[0] <= 64 && spec->channels[1] > 0 &&
                         spec->channels[1] <= 64,
                     "channels");
        ROME_REQUIRE(spec->r_lo >= 0 && spec->r_hi > spec->r_lo, "radius range");
        ROME_CUDA(cudaSetDevice(ctx->device));
        auto* net = new RomeProposalNet();
        net->ctx = ctx;
        net->spec = *spec;
        net->R = spec->n_r;
        net->A = spec->n_theta;
        net->K = spec->n_classes;
        net->c0 = spec->channels[0];
        net->c1 = spec->channels[1];
        auto a4 = [](long v) { return (v + 3) / 4 * 4; };
        const long sizes[6] = {(long)net->c0 * 2 * 9, net->c0, (long)net->c1 * net->c0 * 9, net->c1,
                               (long)net->K * net->c1 * net->R * net->A, net->K};
        long o = 0;
        for (int b = 0; b < 6; b++) {
            net->off[b] = o;
            o = a4(o + sizes[b]);
        }
        net->nparam = o;
        // He-normal weights, zero biases (host RNG, seeded)
        std::vector<float> h(o, 0.f);
        std::mt19937_64 rng(seed);
        const double fan[3] = {2 * 9.0, net->c0 * 9.0, (double)net->c1 * net->R * net->A};
        for (int l = 0; l < 3; l++) {
            std::normal_distribution<double> nd(0.0, std::sqrt(2.0 / fan[l]) * (l < 2 ? 1.0 : 0.5));
            for (long q = 0; q < sizes[2 * l]; q++) h[net->off[2 * l] + q] = (float)nd(rng);
        }
        for (float** p : {&net->params, &net->grads, &net->adam_m, &net->adam_v})
            ROME_CUDA(cudaMalloc(p, sizeof(float) * o));
        ROME_CUDA(cudaMemcpy(net->params, h.data(), sizeof(float) * o, cudaMemcpyHostToDevice));
        ROME_CUDA(cudaMemset(net->grads, 0, sizeof(float) * o));
        ROME_CUDA(cudaMemset(net->adam_m, 0, sizeof(float) * o));
        ROME_CUDA(cudaMemset(net->adam_v, 0, sizeof(float) * o));
        ROME_CUDA(cudaMalloc(&net->loss_acc, sizeof(double)));
        net->CRA = net->c1 * net->R * net->A;
        net->CRAp = (net->CRA + 63) / 64 * 64;
        net->KA = net->K * net->A;
        net->KAp = (net->KA + 63) / 64 * 64;
        ROME_CUDA(cudaMalloc(&net->wt, 4 * (size_t)net->KA * net->CRAp));
        ROME_CUDA(cudaMalloc(&net->wtt, 4 * (size_t)net->CRA * net->KAp));
        ROME_CUDA(cudaMalloc(&net->dwt, sizeof(float) * (size_t)net->KA * net->CRA));
        ROME_CUDA(cudaMalloc(&net->wflip, sizeof(float) * (size_t)net->c1 * net->c0 * 9));
        *out = net;
    });
}

extern "C" void rome_gpu_proposal_destroy(RomeProposalNet* net) {
    if (!net) return;
    cudaSetDevice(net->ctx->device);
    for (float* p : {net->params, net->grads, net->adam_m, net->adam_v, net->x, net->h0, net->h1, net->dh0, net->dh1,
                     net->z, net->dz, net->tgt})
        if (p) cudaFree(p);
    if (net->loss_acc) cudaFree(net->loss_acc);
    if (net->idx) cudaFree(net->idx);
    for (void* p : {net->wt, net->wtt, (void*)net->dwt, net->hs, net->dzs, net->dzt, net->ht, (void*)net->wflip,
                    (void*)net->wpart})
        if (p) cudaFree(p);
    delete net;
}

extern "C" long rome_gpu_proposal_num_params(const RomeProposalNet* net) { return net ? net->nparam : -1; }

extern "C" int rome_gpu_proposal_get_params(RomeProposalNet* net, float* host) {
    if (!net || !host) return ROME_ERR_ARG;
    return guarded(net->ctx, [&] {
        ROME_CUDA(cudaSetDevice(net->ctx->device));
        ROME_CUDA(cudaMemcpy(host, net->params, sizeof(float) * net->nparam, cudaMemcpyDeviceToHost));
    });
}

extern "C" int rome_gpu_proposal_set_params(RomeProposalNet* net, const float* host) {
    if (!net || !host) return ROME_ERR_ARG;
    return guarded(net->ctx, [&] {
        ROME_CUDA(cudaSetDevice(net->ctx->device));
        ROME_CUDA(cudaMemcpy(net->params, host, sizeof(float) * net->nparam, cudaMemcpyHostToDevice));
        net->wt_dirty = true;
        net->adam_t = 0;
        ROME_CUDA(cudaMemset(net->adam_m, 0, sizeof(float) * net->nparam));
        ROME_CUDA(cudaMemset(net->adam_v, 0, sizeof(float) * net->nparam));
    });
}

extern "C" int rome_gpu_proposal_loss_grad(RomeProposalNet* net, int n, const float* x, const float* t, double* loss,
                                           float* grad, float* logits) {
    if (!net || n <= 0 || !x || !t) return ROME_ERR_ARG;
    return guarded(net->ctx, [&] {
        ROME_CUDA(cudaSetDevice(net->ctx->device));
        cudaStream_t st = net->ctx->stream;
        net_alloc_batch(net, n);
        const long row_x = 2L * net->R * net->A, O = (long)net->K * net->A;
        ROME_CUDA(cudaMemcpyAsync(net->x, x, sizeof(float) * row_x * n, cudaMemcpyHostToDevice, st));
        ROME_CUDA(cudaMemcpyAsync(net->tgt, t, sizeof(float) * O * n, cudaMemcpyHostToDevice, st));
        net_loss_grad(net, n, st);
        if (loss) ROME_CUDA(cudaMemcpyAsync(loss, net->loss_acc, sizeof(double), cudaMemcpyDeviceToHost, st));
        if (grad) ROME_CUDA(cudaMemcpyAsync(grad, net->grads, sizeof(float) * net->nparam, cudaMemcpyDeviceToHost, st));
        if (logits) ROME_CUDA(cudaMemcpyAsync(logits, net->z, sizeof(float) * O * n, cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaStreamSynchronize(st));
        tc_check_error(st, net->ctx->d_err);
    });
}

extern "C" int rome_gpu_proposal_train(RomeProposalNet* net, int n, const float* x, const float* t, int epochs,
                                       int batch, float lr, unsigned long long seed, double* epoch_loss) {
    if (!net || n <= 0 || !x || !t || epochs <= 0 || batch <= 0) return ROME_ERR_ARG;
    return guarded(net->ctx, [&] {
        ROME_CUDA(cudaSetDevice(net->ctx->device));
        cudaStream_t st = net->ctx->stream;
        const int B = std::min(batch, n);
        net_alloc_batch(net, B);
        const long row_x = 2L * net->R * net->A, row_t = (long)net->K * net->A;
        float *dx = nullptr, *dt = nullptr;
        int* dperm = nullptr;
        ROME_CUDA(cudaMalloc(&dx, sizeof(float) * row_x * n));
        ROME_CUDA(cudaMalloc(&dt, sizeof(float) * row_t * n));
        ROME_CUDA(cudaMalloc(&dperm, sizeof(int) * n));
        ROME_CUDA(cudaMemcpyAsync(dx, x, sizeof(float) * row_x * n, cudaMemcpyHostToDevice, st));
        ROME_CUDA(cudaMemcpyAsync(dt, t, sizeof(float) * row_t * n, cudaMemcpyHostToDevice, st));
        std::vector<int> perm(n);
        std::iota(perm.begin(), perm.end(), 0);
        std::mt19937_64 rng(seed);
        const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
        for (int ep = 0; ep < epochs; ep++) {
            std::shuffle(perm.begin(), perm.end(), rng);
            ROME_CUDA(cudaMemcpyAsync(dperm, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
            ROME_CUDA(cudaMemsetAsync(net->loss_acc, 0, sizeof(double), st));
            int nb = 0;
            for (int b0 = 0; b0 + B <= n; b0 += B, nb++) {
                gather_rows_kernel<<<(unsigned)((B * row_x + PT - 1) / PT), PT, 0, st>>>(B, row_x, dperm + b0, dx,
                                                                                        net->x);
                gather_rows_kernel<<<(unsigned)((B * row_t + PT - 1) / PT), PT, 0, st>>>(B, row_t, dperm + b0, dt,
                                                                                        net->tgt);
                ROME_CHECK_LAUNCH();
                net_forward(net, B, st);
                softmax_xent_kernel<<<B, PT, 0, st>>>(B, (int)row_t, net->z, net->tgt, net->dz, net->loss_acc);
                ROME_CHECK_LAUNCH();
                net_backward(net, B, st);
                net->adam_t++;
                const float c1 = 1.f - std::pow(b1, (float)net->adam_t), c2 = 1.f - std::pow(b2, (float)net->adam_t);
                adam_kernel<<<(unsigned)((net->nparam + PT - 1) / PT), PT, 0, st>>>(
                    net->nparam, lr, b1, b2, eps, c1, c2, net->grads, net->params, net->adam_m, net->adam_v);
                ROME_CHECK_LAUNCH();
                net->wt_dirty = true;
            }
            double l = 0;
            ROME_CUDA(cudaMemcpyAsync(&l, net->loss_acc, sizeof(double), cudaMemcpyDeviceToHost, st));
            // the host reshuffles `perm` next epoch: its copy must be done
            ROME_CUDA(cudaStreamSynchronize(st));
            tc_check_error(st, net->ctx->d_err);
            if (epoch_loss) epoch_loss[ep] = nb ? l / nb : 0.0;
        }
        cudaFree(dx);
        cudaFree(dt);
        cudaFree(dperm);
    });
}

namespace rome {
// top-k outputs of n feature rows already on the device
void proposal_predict_device(RomeProposalNet* net, int n, const float* dfeat, int k, int* didx, float* dprob,
                             cudaStream_t st) {
    const long row_x = 2L * net->R * net->A;
    const int O = net->K * net->A;
    const int chunk = 4096;
    net_alloc_batch(net, std::min(n, chunk));
    for (int done = 0; done < n;) {
        const int m = std::min(chunk, n - done);
        ROME_CUDA(cudaMemcpyAsync(net->x, dfeat + (long)done * row_x, sizeof(float) * row_x * m,
                                  cudaMemcpyDeviceToDevice, st));
        net_forward(net, m, st, false);
        topk_warp_kernel<<<(m + PT / 32 - 1) / (PT / 32), PT, 0, st>>>(m, O, k, net->z, didx + (long)done * k,
                                                                       dprob ? dprob + (long)done * k : nullptr);
        ROME_CHECK_LAUNCH();
        done += m;
    }
}

void proposal_features_device(RomeProposalNet* net, int P, int cur, const double* Fr, const double* Fi,
                              const double* ctf, float* dfeat, cudaStream_t st) {
    ROME_REQUIRE(net->spec.r_hi + 1 < cur / 2, "radius %.1f too large for image size %d", net->spec.r_hi, cur);
    polar_features_kernel<<<P, PT, sizeof(float) * 2 * net->R * net->A, st>>>(cur, net->R, net->A, net->spec.r_lo,
                                                                            net->spec.r_hi, Fr, Fi, ctf, dfeat);
    ROME_CHECK_LAUNCH();
}
}  // namespace rome

extern "C" int rome_gpu_proposal_features(RomeProposalNet* net, int P, int cur, const double* Fr, const double* Fi,
                                          const double* ctf, int inputs_on_device, float* x_out) {
    if (!net || P <= 0 || !Fr || !Fi || !ctf || !x_out) return ROME_ERR_ARG;
    return guarded(net->ctx, [&] {
        ROME_CUDA(cudaSetDevice(net->ctx->device));
        cudaStream_t st = net->ctx->stream;
        const long F = (long)cur * (cur / 2 + 1);
        const long row_x = 2L * net->R * net->A;
        float* dx = (float*)net->ctx->ws[S_TMP1].get(sizeof(float) * row_x * P);
        const double *dFr = Fr, *dFi = Fi, *dC = ctf;
        if (!inputs_on_device) {
            double* d = net->ctx->ws[S_TMP2].as<double>((size_t)3 * P * F);
            ROME_CUDA(cudaMemcpyAsync(d, Fr, sizeof(double) * P * F, cudaMemcpyHostToDevice, st));
            ROME_CUDA(cudaMemcpyAsync(d + P * F, Fi, sizeof(double) * P * F, cudaMemcpyHostToDevice, st));
            ROME_CUDA(cudaMemcpyAsync(d + 2 * P * F, ctf, sizeof(double) * P * F, cudaMemcpyHostToDevice, st));
            dFr = d;
            dFi = d + P * F;
            dC = d + 2 * P * F;
        }
        proposal_features_device(net, P, cur, dFr, dFi, dC, dx, st);
        ROME_CUDA(cudaMemcpyAsync(x_out, dx, sizeof(float) * row_x * P, cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaStreamSynchronize(st));
        tc_check_error(st, net->ctx->d_err);
    });
}

extern "C" int rome_gpu_proposal_predict(RomeProposalNet* net, int n, const float* x, int k, int* idx, float* prob) {
    if (!net || n <= 0 || !x || k <= 0 || k > net->K * net->A || !idx) return ROME_ERR_ARG;
    return guarded(net->ctx, [&] {
        ROME_CUDA(cudaSetDevice(net->ctx->device));
        cudaStream_t st = net->ctx->stream;
        const long row_x = 2L * net->R * net->A;
        float* dx = (float*)net->ctx->ws[S_TMP1].get(sizeof(float) * row_x * n);
        int* di = (int*)net->ctx->ws[S_TMP0].get((sizeof(int) + sizeof(float)) * (size_t)n * k);
        float* dp = (float*)(di + (size_t)n * k);
        ROME_CUDA(cudaMemcpyAsync(dx, x, sizeof(float) * row_x * n, cudaMemcpyHostToDevice, st));
        proposal_predict_device(net, n, dx, k, di, dp, st);
        ROME_CUDA(cudaMemcpyAsync(idx, di, sizeof(int) * (size_t)n * k, cudaMemcpyDeviceToHost, st));
        if (prob) ROME_CUDA(cudaMemcpyAsync(prob, dp, sizeof(float) * (size_t)n * k, cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaStreamSynchronize(st));
        tc_check_error(st, net->ctx->d_err);
    });
}

extern "C" int rome_gpu_proposal_propose(RomeProposalNet* net, int P, int cur, const double* Fr, const double* Fi,
                                         const double* ctf, int inputs_on_device, int k, int* proposals,
                                         float* mass) {
    if (!net || P <= 0 || !Fr || !Fi || !ctf || k <= 0 || k > 64 || k > net->K * net->A || !proposals)
        return ROME_ERR_ARG;
    return guarded(net->ctx, [&] {
        ROME_CUDA(cudaSetDevice(net->ctx->device));
        cudaStream_t st = net->ctx->stream;
        const long F = (long)cur * (cur / 2 + 1);
        const long row_x = 2L * net->R * net->A;
        const double *dFr = Fr, *dFi = Fi, *dC = ctf;
        if (!inputs_on_device) {
            double* d = net->ctx->ws[S_TMP2].as<double>((size_t)3 * P * F);
            ROME_CUDA(cudaMemcpyAsync(d, Fr, sizeof(double) * P * F, cudaMemcpyHostToDevice, st));
            ROME_CUDA(cudaMemcpyAsync(d + P * F, Fi, sizeof(double) * P * F, cudaMemcpyHostToDevice, st));
            ROME_CUDA(cudaMemcpyAsync(d + 2 * P * F, ctf, sizeof(double) * P * F, cudaMemcpyHostToDevice, st));
            dFr = d;
            dFi = d + P * F;
            dC = d + 2 * P * F;
        }
        Profiler prof(net->ctx);
        prof.begin(ROME_PHASE_PROPOSE);
        float* dx = (float*)net->ctx->ws[S_TMP1].get(sizeof(float) * row_x * P);
        char* buf = (char*)net->ctx->ws[S_TMP0].get((sizeof(int) + sizeof(float)) * (size_t)P * k +
                                                    (sizeof(int) * 2 * k + sizeof(float)) * (size_t)P);
        int* di = (int*)buf;
        float* dp = (float*)(di + (size_t)P * k);
        int* dprop = (int*)(dp + (size_t)P * k);
        float* dmass = (float*)(dprop + (size_t)P * 2 * k);
        proposal_features_device(net, P, cur, dFr, dFi, dC, dx, st);
        proposal_predict_device(net, P, dx, k, di, dp, st);
        expand_proposals_kernel<<<(P + 127) / 128, 128, 0, st>>>(P, k, net->A, di, dp, dprop, dmass);
        ROME_CHECK_LAUNCH();
        // features and the expansion, and top-k per chunk of 4096 (the network's own launches are counted where
        // they are made)
        net->ctx->total_launches += 2 + 1L * ((P + 4095) / 4096);
        net->ctx->phase_launches[ROME_PHASE_PROPOSE] += 2 + 1L * ((P + 4095) / 4096);
        prof.end(ROME_PHASE_PROPOSE);
        ROME_CUDA(cudaMemcpyAsync(proposals, dprop, sizeof(int) * (size_t)P * 2 * k, cudaMemcpyDeviceToHost, st));
        if (mass) ROME_CUDA(cudaMemcpyAsync(mass, dmass, sizeof(float) * P, cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaStreamSynchronize(st));
        prof.collect();
        tc_check_error(st, net->ctx->d_err);
    });
}
