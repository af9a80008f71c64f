// Learned pose proposals for the MAP E-step: a small CNN over the low-pass
// Fourier magnitude of each particle that predicts a distribution over
// (class, psi mod 180 deg), trained on the GPU on (image, posterior) pairs
// produced by the exhaustive E-step itself, with hand-written FP32 forward,
// backward and Adam kernels.  Its top-k (class, psi) pairs (each psi taken
// with psi + 180, which the magnitude cannot tell apart) restrict the
// E-step's search; the exhaustive E-step stays the fallback and the judge.
//
// Network (N samples, S x S input, channels c0..c3, O outputs):
//   x[N][2][S][S] -> conv3x3 s1 + ReLU -> conv3x3 s2 + ReLU
//                 -> conv3x3 s2 + ReLU -> conv3x3 s2 + ReLU -> [N][c3][S/8][S/8]
//                 -> linear -> z[N][O];  loss = mean_n sum_o -t log softmax(z)
// Parameters are one flat FP32 array in the order w0 b0 w1 b1 w2 b2 w3 b3 wf bf
// (w[l]: [c_l][c_{l-1}][3][3], wf: [O][c3 (S/8)^2]), each block starting at a
// multiple of 4 floats (zero padding between blocks).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "common.cuh"
#include "epilogues.cuh"
#include "gemm_simt.cuh"

using namespace rome;

struct RomeProposalNet {
    RomeGpuCtx* ctx = nullptr;
    RomeProposalSpec spec{};
    int ch[5] = {0};     // ch[0] = input channels
    int hw[5] = {0};     // spatial size after each layer
    long off_w[5] = {0}, off_b[5] = {0};  // index 4 = the linear layer
    long nparam = 0;
    int flat = 0;        // c3 * (S/8)^2
    float* params = nullptr;
    float* grads = nullptr;
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    long adam_t = 0;
    // batch buffers (capacity cap_n)
    int cap_n = 0;
    float* act[5] = {nullptr};   // act[0] input, act[l+1] post-ReLU of layer l
    float* dact[5] = {nullptr};
    float* z = nullptr;          // [N][O]
    float* dz = nullptr;
    float* tgt = nullptr;        // [N][O]
    float* tmpA = nullptr;       // transposes for the linear layer
    float* tmpB = nullptr;
    double* loss_acc = nullptr;
    int* idx = nullptr;
};

namespace rome {
namespace {

constexpr int PT = 256;

// ---- convolution 3x3, zero padding 1, stride s, fused bias + ReLU ----
__global__ void __launch_bounds__(PT) conv_fwd_kernel(int Ci, int H, int W, int Co, int Ho, int Wo, int s,
                                                       const float* __restrict__ x, const float* __restrict__ w,
                                                       const float* __restrict__ b, float* __restrict__ y) {
    extern __shared__ float sw[];  // Ci * 9 weights of this output channel
    const int co = blockIdx.y, n = blockIdx.z;
    for (int q = threadIdx.x; q < Ci * 9; q += PT) sw[q] = w[(long)co * Ci * 9 + q];
    __syncthreads();
    const int p = blockIdx.x * PT + threadIdx.x;
    if (p >= Ho * Wo) return;
    const int ho = p / Wo, wo = p - ho * Wo;
    const float* xn = x + (long)n * Ci * H * W;
    float acc = b[co];
    for (int ci = 0; ci < Ci; ci++) {
        const float* xc = xn + (long)ci * H * W;
        const float* wc = sw + ci * 9;
#pragma unroll
        for (int kh = 0; kh < 3; kh++) {
            const int h = ho * s + kh - 1;
            if (h < 0 || h >= H) continue;
#pragma unroll
            for (int kw = 0; kw < 3; kw++) {
                const int ww = wo * s + kw - 1;
                if (ww < 0 || ww >= W) continue;
                acc = fmaf(wc[kh * 3 + kw], xc[h * W + ww], acc);
            }
        }
    }
    y[(((long)n * Co + co) * Ho + ho) * Wo + wo] = fmaxf(acc, 0.f);
}

// dy <- dy * (y > 0): the ReLU's gradient, in place
__global__ void relu_mask_kernel(long n, const float* __restrict__ y, float* __restrict__ dy) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n && !(y[q] > 0.f)) dy[q] = 0.f;
}

// dx[n][ci][h][w] = sum_co sum_taps w[co][ci][kh][kw] dy[n][co][ho][wo], h = s ho + kh - 1
__global__ void __launch_bounds__(PT) conv_bwd_data_kernel(int Ci, int H, int W, int Co, int Ho, int Wo, int s,
                                                            const float* __restrict__ dy, const float* __restrict__ w,
                                                            float* __restrict__ dx) {
    const int ci = blockIdx.y, n = blockIdx.z;
    const int p = blockIdx.x * PT + threadIdx.x;
    if (p >= H * W) return;
    const int h = p / W, ww = p - h * W;
    float acc = 0.f;
    for (int kh = 0; kh < 3; kh++) {
        const int th = h + 1 - kh;
        if (th < 0 || th % s) continue;
        const int ho = th / s;
        if (ho >= Ho) continue;
        for (int kw = 0; kw < 3; kw++) {
            const int tw = ww + 1 - kw;
            if (tw < 0 || tw % s) continue;
            const int wo = tw / s;
            if (wo >= Wo) continue;
            const float* dyp = dy + (long)n * Co * Ho * Wo + (long)ho * Wo + wo;
            const float* wp = w + (long)ci * 9 + kh * 3 + kw;
            for (int co = 0; co < Co; co++) acc = fmaf(wp[(long)co * Ci * 9], dyp[(long)co * Ho * Wo], acc);
        }
    }
    dx[(((long)n * Ci + ci) * H + h) * W + ww] = acc;
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

// dw[co][ci][kh][kw] = sum_{n,ho,wo} dy[n][co][ho][wo] x[n][ci][s ho + kh - 1][s wo + kw - 1]
__global__ void __launch_bounds__(PT) conv_bwd_weight_kernel(int N, int Ci, int H, int W, int Co, int Ho, int Wo,
                                                              int s, const float* __restrict__ x,
                                                              const float* __restrict__ dy, float* __restrict__ dw) {
    __shared__ float sh[32];
    const int co = blockIdx.x, ci = blockIdx.y;
    float acc[9];
#pragma unroll
    for (int k = 0; k < 9; k++) acc[k] = 0.f;
    const long tot = (long)N * Ho * Wo;
    for (long q = threadIdx.x; q < tot; q += PT) {
        const int n = (int)(q / (Ho * Wo));
        const int p = (int)(q - (long)n * Ho * Wo);
        const int ho = p / Wo, wo = p - ho * Wo;
        const float g = dy[((long)n * Co + co) * Ho * Wo + p];
        if (g == 0.f) continue;
        const float* xc = x + ((long)n * Ci + ci) * H * W;
#pragma unroll
        for (int kh = 0; kh < 3; kh++) {
            const int h = ho * s + kh - 1;
            if (h < 0 || h >= H) continue;
#pragma unroll
            for (int kw = 0; kw < 3; kw++) {
                const int ww = wo * s + kw - 1;
                if (ww < 0 || ww >= W) continue;
                acc[kh * 3 + kw] = fmaf(g, xc[h * W + ww], acc[kh * 3 + kw]);
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

// out[c][r] = in[r][c] for r < rows, c < cols; zero for r in [rows, rows_pad)
__global__ void transpose_pad_kernel(int rows, int cols, int rows_pad, const float* __restrict__ in, long ldin,
                                     float* __restrict__ out) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long)rows_pad * cols) return;
    const int c = (int)(q / rows_pad), r = (int)(q - (long)c * rows_pad);
    out[q] = r < rows ? in[(long)r * ldin + c] : 0.f;
}

// out[r][c] = in[r][c] for c < cols, zero for c in [cols, cols_pad)
__global__ void pad_cols_kernel(int rows, int cols, int cols_pad, const float* __restrict__ in,
                                float* __restrict__ out) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long)rows * cols_pad) return;
    const int r = (int)(q / cols_pad), c = (int)(q - (long)r * cols_pad);
    out[q] = c < cols ? in[(long)r * cols + c] : 0.f;
}

__global__ void add_bias_kernel(int N, int O, long ld, const float* __restrict__ b, float* __restrict__ z) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long)N * O) return;
    const int n = (int)(q / O), o = (int)(q - (long)n * O);
    z[(long)n * ld + o] += b[o];
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

// Network input of one particle (see oracle/proposal_oracle.py features()):
// log(1 + |X|) and |CTF| on the centred size x size frequency grid, the
// negative-kx half by Friedel symmetry, each channel normalised.
__global__ void __launch_bounds__(PT) features_kernel(int cur, int size, const double* __restrict__ Fr,
                                                       const double* __restrict__ Fi, const double* __restrict__ ctf,
                                                       float* __restrict__ x) {
    extern __shared__ float sx[];  // 2 * size * size
    __shared__ double shd[32];
    __shared__ double s_mean[2], s_std[2];
    const int i = blockIdx.x, cf = cur / 2 + 1, h = size / 2, n2 = size * size;
    const long base = (long)i * cur * cf;
    for (int q = threadIdx.x; q < n2; q += PT) {
        const int iy = q / size, ix = q - iy * size;
        int kx = ix - h, ky = iy - h;
        if (kx < 0) {
            kx = -kx;
            ky = -ky;
        }
        const int row = ky >= 0 ? ky : ky + cur;
        const long e = base + (long)row * cf + kx;
        const double re = Fr[e], im = Fi[e];
        sx[q] = (float)log1p(sqrt(re * re + im * im));
        sx[n2 + q] = (float)fabs(ctf[e]);
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
// softmax probability of each
__global__ void __launch_bounds__(PT) topk_kernel(int O, int k, const float* __restrict__ z, int* __restrict__ idx,
                                                   float* __restrict__ prob) {
    extern __shared__ unsigned char smraw[];
    const int n2 = 1 << (32 - __clz(O - 1));
    float* key = (float*)smraw;
    int* val = (int*)(key + n2);
    __shared__ float shf[32];
    __shared__ float s_max, s_sum;
    const int r = blockIdx.x;
    const float* zr = z + (long)r * O;
    for (int q = threadIdx.x; q < n2; q += PT) {
        key[q] = q < O ? zr[q] : -INFINITY;
        val[q] = q < O ? q : 0x7fffffff;
    }
    float m = -INFINITY;
    for (int o = threadIdx.x; o < O; o += PT) m = fmaxf(m, zr[o]);
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
    for (int o = threadIdx.x; o < O; o += PT) se += __expf(zr[o] - s_max);
    se = block_sum(se, shf);
    if (threadIdx.x == 0) s_sum = se;
    __syncthreads();
    // bitonic sort, descending by key, ascending index on ties
    for (int kk = 2; kk <= n2; kk <<= 1) {
        for (int j = kk >> 1; j > 0; j >>= 1) {
            for (int q = threadIdx.x; q < n2; q += PT) {
                const int p = q ^ j;
                if (p > q) {
                    const bool desc = (q & kk) == 0;
                    const float a = key[q], b = key[p];
                    const int ia = val[q], ib = val[p];
                    const bool a_first = a > b || (a == b && ia < ib);
                    if (desc ? !a_first : a_first) {
                        key[q] = b;
                        key[p] = a;
                        val[q] = ib;
                        val[p] = ia;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int q = threadIdx.x; q < k; q += PT) {
        idx[(long)r * k + q] = val[q];
        if (prob) prob[(long)r * k + q] = __expf(key[q] - s_max) / s_sum;
    }
}

void net_alloc_batch(RomeProposalNet* net, int n) {
    if (n <= net->cap_n) return;
    auto& sp = net->spec;
    for (int l = 0; l < 5; l++) {
        if (net->act[l]) cudaFree(net->act[l]);
        if (net->dact[l]) cudaFree(net->dact[l]);
        const size_t e = (size_t)n * net->ch[l] * net->hw[l] * net->hw[l];
        ROME_CUDA(cudaMalloc(&net->act[l], sizeof(float) * e));
        ROME_CUDA(cudaMalloc(&net->dact[l], sizeof(float) * e));
    }
    for (float** p : {&net->z, &net->dz, &net->tgt}) {
        if (*p) cudaFree(*p);
        ROME_CUDA(cudaMalloc(p, sizeof(float) * (size_t)n * sp.n_out));
    }
    const int npad = (n + 15) / 16 * 16, opad = (sp.n_out + 15) / 16 * 16;
    const size_t tsz = std::max({(size_t)npad * sp.n_out, (size_t)npad * net->flat, (size_t)opad * net->flat,
                                 (size_t)n * opad});
    for (float** p : {&net->tmpA, &net->tmpB}) {
        if (*p) cudaFree(*p);
        ROME_CUDA(cudaMalloc(p, sizeof(float) * tsz));
    }
    if (net->idx) cudaFree(net->idx);
    ROME_CUDA(cudaMalloc(&net->idx, sizeof(int) * n));
    net->cap_n = n;
}

void net_forward(RomeProposalNet* net, int n, cudaStream_t st) {
    auto& sp = net->spec;
    static const int strides[4] = {1, 2, 2, 2};
    for (int l = 0; l < 4; l++) {
        const int Ci = net->ch[l], H = net->hw[l], Co = net->ch[l + 1], Ho = net->hw[l + 1];
        dim3 grid((Ho * Ho + PT - 1) / PT, Co, n);
        conv_fwd_kernel<<<grid, PT, sizeof(float) * Ci * 9, st>>>(Ci, H, H, Co, Ho, Ho, strides[l], net->act[l],
                                                                 net->params + net->off_w[l],
                                                                 net->params + net->off_b[l], net->act[l + 1]);
        ROME_CHECK_LAUNCH();
    }
    // linear: z[n][o] = act4[n][:] . wf[o][:] + bf[o]
    sgemm_tn(st, n, sp.n_out, net->flat, net->act[4], net->flat, net->params + net->off_w[4], net->flat,
             StoreEpi{net->z, sp.n_out});
    ROME_CHECK_LAUNCH();
    add_bias_kernel<<<(unsigned)(((long)n * sp.n_out + PT - 1) / PT), PT, 0, st>>>(n, sp.n_out, sp.n_out,
                                                                                   net->params + net->off_b[4], net->z);
    ROME_CHECK_LAUNCH();
}

// gradients of the mean loss into net->grads (dz must hold dL/dz)
void net_backward(RomeProposalNet* net, int n, cudaStream_t st) {
    auto& sp = net->spec;
    const int O = sp.n_out, F = net->flat;
    const int npad = (n + 15) / 16 * 16, opad = (O + 15) / 16 * 16;
    // gwf[o][f] = sum_n dz[n][o] act4[n][f]: A = dz^T [O][npad], B = act4^T [F][npad]
    transpose_pad_kernel<<<(unsigned)(((long)npad * O + PT - 1) / PT), PT, 0, st>>>(n, O, npad, net->dz, O, net->tmpA);
    transpose_pad_kernel<<<(unsigned)(((long)npad * F + PT - 1) / PT), PT, 0, st>>>(n, F, npad, net->act[4], F,
                                                                                    net->tmpB);
    ROME_CHECK_LAUNCH();
    sgemm_tn(st, O, F, npad, net->tmpA, npad, net->tmpB, npad, StoreEpi{net->grads + net->off_w[4], F});
    bias_grad_kernel<<<O, PT, 0, st>>>(n, O, 1, net->dz, net->grads + net->off_b[4]);
    ROME_CHECK_LAUNCH();
    // dact4[n][f] = sum_o dz[n][o] wf[o][f]: A = dz with columns padded to opad, B = wf^T [F][opad]
    pad_cols_kernel<<<(unsigned)(((long)n * opad + PT - 1) / PT), PT, 0, st>>>(n, O, opad, net->dz, net->tmpB);
    transpose_pad_kernel<<<(unsigned)(((long)opad * F + PT - 1) / PT), PT, 0, st>>>(O, F, opad,
                                                                                    net->params + net->off_w[4], F,
                                                                                    net->tmpA);
    ROME_CHECK_LAUNCH();
    sgemm_tn(st, n, F, opad, net->tmpB, opad, net->tmpA, opad, StoreEpi{net->dact[4], F});
    ROME_CHECK_LAUNCH();
    static const int strides[4] = {1, 2, 2, 2};
    for (int l = 3; l >= 0; l--) {
        const int Ci = net->ch[l], H = net->hw[l], Co = net->ch[l + 1], Ho = net->hw[l + 1];
        const long ny = (long)n * Co * Ho * Ho;
        relu_mask_kernel<<<(unsigned)((ny + PT - 1) / PT), PT, 0, st>>>(ny, net->act[l + 1], net->dact[l + 1]);
        conv_bwd_weight_kernel<<<dim3(Co, Ci), PT, 0, st>>>(n, Ci, H, H, Co, Ho, Ho, strides[l], net->act[l],
                                                            net->dact[l + 1], net->grads + net->off_w[l]);
        bias_grad_kernel<<<Co, PT, 0, st>>>(n, Co, Ho * Ho, net->dact[l + 1], net->grads + net->off_b[l]);
        if (l > 0) {
            dim3 grid((H * H + PT - 1) / PT, Ci, n);
            conv_bwd_data_kernel<<<grid, PT, 0, st>>>(Ci, H, H, Co, Ho, Ho, strides[l], net->dact[l + 1],
                                                      net->params + net->off_w[l], net->dact[l]);
        }
        ROME_CHECK_LAUNCH();
    }
}

double net_loss_grad(RomeProposalNet* net, int n, cudaStream_t st) {
    ROME_CUDA(cudaMemsetAsync(net->loss_acc, 0, sizeof(double), st));
    net_forward(net, n, st);
    softmax_xent_kernel<<<n, PT, 0, st>>>(n, net->spec.n_out, net->z, net->tgt, net->dz, net->loss_acc);
    ROME_CHECK_LAUNCH();
    net_backward(net, n, st);
    return 0.0;
}

}  // namespace
}  // namespace rome

extern "C" int rome_gpu_proposal_create(RomeGpuCtx* ctx, const RomeProposalSpec* spec, unsigned long long seed,
                                        RomeProposalNet** out) {
    if (!ctx || !spec || !out) return ROME_ERR_ARG;
    *out = nullptr;
    return guarded(ctx, [&] {
        ROME_REQUIRE(spec->size >= 8 && spec->size % 8 == 0 && spec->size <= 64, "input size %d (multiple of 8, <= 64)",
                     spec->size);
        ROME_REQUIRE(spec->n_out > 0 && spec->n_out <= 8192, "n_out %d", spec->n_out);
        for (int l = 0; l < 4; l++) ROME_REQUIRE(spec->channels[l] > 0 && spec->channels[l] <= 128, "channels");
        ROME_CUDA(cudaSetDevice(ctx->device));
        auto* net = new RomeProposalNet();
        net->ctx = ctx;
        net->spec = *spec;
        net->ch[0] = 2;
        net->hw[0] = spec->size;
        for (int l = 0; l < 4; l++) {
            net->ch[l + 1] = spec->channels[l];
            net->hw[l + 1] = l == 0 ? spec->size : (net->hw[l] - 1) / 2 + 1;
        }
        net->flat = net->ch[4] * net->hw[4] * net->hw[4];
        if (net->flat % 16) {
            delete net;
            fail(ROME_ERR_ARG, "flattened size %d must be a multiple of 16", net->hw[4]);
        }
        // every block starts on a 16-byte boundary (vector loads of the linear layer)
        auto a4 = [](long v) { return (v + 3) / 4 * 4; };
        long o = 0;
        for (int l = 0; l < 4; l++) {
            net->off_w[l] = o;
            o = a4(o + (long)net->ch[l + 1] * net->ch[l] * 9);
            net->off_b[l] = o;
            o = a4(o + net->ch[l + 1]);
        }
        net->off_w[4] = o;
        o = a4(o + (long)spec->n_out * net->flat);
        net->off_b[4] = o;
        o = a4(o + spec->n_out);
        net->nparam = o;
        // He-normal weights, zero biases (host RNG, seeded)
        std::vector<float> h(o, 0.f);
        std::mt19937_64 rng(seed);
        for (int l = 0; l < 5; l++) {
            const long nw = (l < 4 ? (long)net->ch[l + 1] * net->ch[l] * 9 : (long)spec->n_out * net->flat);
            const double fan_in = l < 4 ? net->ch[l] * 9.0 : (double)net->flat;
            std::normal_distribution<double> nd(0.0, std::sqrt(2.0 / fan_in) * (l < 4 ? 1.0 : 0.5));
            for (long q = 0; q < nw; q++) h[net->off_w[l] + q] = (float)nd(rng);
        }
        for (float** p : {&net->params, &net->grads, &net->adam_m, &net->adam_v})
            ROME_CUDA(cudaMalloc(p, sizeof(float) * o));
        ROME_CUDA(cudaMemcpy(net->params, h.data(), sizeof(float) * o, cudaMemcpyHostToDevice));
        ROME_CUDA(cudaMemset(net->adam_m, 0, sizeof(float) * o));
        ROME_CUDA(cudaMemset(net->adam_v, 0, sizeof(float) * o));
        ROME_CUDA(cudaMalloc(&net->loss_acc, sizeof(double)));
        *out = net;
    });
}

extern "C" void rome_gpu_proposal_destroy(RomeProposalNet* net) {
    if (!net) return;
    cudaSetDevice(net->ctx->device);
    for (float* p : {net->params, net->grads, net->adam_m, net->adam_v, net->z, net->dz, net->tgt, net->tmpA,
                     net->tmpB})
        if (p) cudaFree(p);
    for (int l = 0; l < 5; l++) {
        if (net->act[l]) cudaFree(net->act[l]);
        if (net->dact[l]) cudaFree(net->dact[l]);
    }
    if (net->loss_acc) cudaFree(net->loss_acc);
    if (net->idx) cudaFree(net->idx);
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
        const long in = (long)n * 2 * net->spec.size * net->spec.size;
        ROME_CUDA(cudaMemcpyAsync(net->act[0], x, sizeof(float) * in, cudaMemcpyHostToDevice, st));
        ROME_CUDA(cudaMemcpyAsync(net->tgt, t, sizeof(float) * (size_t)n * net->spec.n_out, cudaMemcpyHostToDevice,
                                  st));
        net_loss_grad(net, n, st);
        if (loss) ROME_CUDA(cudaMemcpyAsync(loss, net->loss_acc, sizeof(double), cudaMemcpyDeviceToHost, st));
        if (grad) ROME_CUDA(cudaMemcpyAsync(grad, net->grads, sizeof(float) * net->nparam, cudaMemcpyDeviceToHost, st));
        if (logits)
            ROME_CUDA(cudaMemcpyAsync(logits, net->z, sizeof(float) * (size_t)n * net->spec.n_out,
                                      cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaStreamSynchronize(st));
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
        const long row_x = 2L * net->spec.size * net->spec.size, row_t = net->spec.n_out;
        float *dx = nullptr, *dt = nullptr;
        ROME_CUDA(cudaMalloc(&dx, sizeof(float) * row_x * n));
        ROME_CUDA(cudaMalloc(&dt, sizeof(float) * row_t * n));
        ROME_CUDA(cudaMemcpyAsync(dx, x, sizeof(float) * row_x * n, cudaMemcpyHostToDevice, st));
        ROME_CUDA(cudaMemcpyAsync(dt, t, sizeof(float) * row_t * n, cudaMemcpyHostToDevice, st));
        std::vector<int> perm(n);
        std::iota(perm.begin(), perm.end(), 0);
        std::mt19937_64 rng(seed);
        const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
        for (int ep = 0; ep < epochs; ep++) {
            std::shuffle(perm.begin(), perm.end(), rng);
            ROME_CUDA(cudaMemsetAsync(net->loss_acc, 0, sizeof(double), st));
            int nb = 0;
            for (int b0 = 0; b0 + B <= n; b0 += B, nb++) {
                ROME_CUDA(cudaMemcpyAsync(net->idx, perm.data() + b0, sizeof(int) * B, cudaMemcpyHostToDevice, st));
                gather_rows_kernel<<<(unsigned)((B * row_x + PT - 1) / PT), PT, 0, st>>>(B, row_x, net->idx, dx,
                                                                                        net->act[0]);
                gather_rows_kernel<<<(unsigned)((B * row_t + PT - 1) / PT), PT, 0, st>>>(B, row_t, net->idx, dt,
                                                                                        net->tgt);
                ROME_CHECK_LAUNCH();
                net_forward(net, B, st);
                softmax_xent_kernel<<<B, PT, 0, st>>>(B, net->spec.n_out, net->z, net->tgt, net->dz, net->loss_acc);
                ROME_CHECK_LAUNCH();
                net_backward(net, B, st);
                net->adam_t++;
                const float c1 = 1.f - std::pow(b1, (float)net->adam_t), c2 = 1.f - std::pow(b2, (float)net->adam_t);
                adam_kernel<<<(unsigned)((net->nparam + PT - 1) / PT), PT, 0, st>>>(
                    net->nparam, lr, b1, b2, eps, c1, c2, net->grads, net->params, net->adam_m, net->adam_v);
                ROME_CHECK_LAUNCH();
                // the staging copy of the index list must finish before the host refills it
                ROME_CUDA(cudaStreamSynchronize(st));
            }
            double l = 0;
            ROME_CUDA(cudaMemcpyAsync(&l, net->loss_acc, sizeof(double), cudaMemcpyDeviceToHost, st));
            ROME_CUDA(cudaStreamSynchronize(st));
            if (epoch_loss) epoch_loss[ep] = nb ? l / nb : 0.0;
        }
        cudaFree(dx);
        cudaFree(dt);
    });
}

namespace rome {
// logits of n feature rows already on the device, then top-k per row
void proposal_predict_device(RomeProposalNet* net, int n, const float* dfeat, int k, int* didx, float* dprob,
                             cudaStream_t st) {
    int done = 0;
    const long row_x = 2L * net->spec.size * net->spec.size;
    const int chunk = 4096;
    net_alloc_batch(net, std::min(n, chunk));
    while (done < n) {
        const int m = std::min(chunk, n - done);
        ROME_CUDA(cudaMemcpyAsync(net->act[0], dfeat + (long)done * row_x, sizeof(float) * row_x * m,
                                  cudaMemcpyDeviceToDevice, st));
        net_forward(net, m, st);
        const int O = net->spec.n_out;
        const int n2 = 1 << (32 - __builtin_clz((unsigned)(O - 1)));
        const size_t smem = (sizeof(float) + sizeof(int)) * n2;
        ROME_CUDA(cudaFuncSetAttribute(topk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        topk_kernel<<<m, PT, smem, st>>>(O, k, net->z, didx + (long)done * k, dprob ? dprob + (long)done * k : nullptr);
        ROME_CHECK_LAUNCH();
        done += m;
    }
}

void proposal_features_device(RomeProposalNet* net, int P, int cur, const double* Fr, const double* Fi,
                              const double* ctf, float* dfeat, cudaStream_t st) {
    const int S = net->spec.size;
    ROME_REQUIRE(S <= cur, "proposal input size %d exceeds the image size %d", S, cur);
    features_kernel<<<P, PT, sizeof(float) * 2 * S * S, st>>>(cur, S, Fr, Fi, ctf, dfeat);
    ROME_CHECK_LAUNCH();
}
}  // namespace rome

extern "C" int rome_gpu_proposal_features(RomeProposalNet* net, int P, int cur, const double* Fr, const double* Fi,
                                          const double* ctf, float* x_out) {
    if (!net || P <= 0 || !Fr || !Fi || !ctf || !x_out) return ROME_ERR_ARG;
    return guarded(net->ctx, [&] {
        ROME_CUDA(cudaSetDevice(net->ctx->device));
        cudaStream_t st = net->ctx->stream;
        const long F = (long)cur * (cur / 2 + 1);
        const long row_x = 2L * net->spec.size * net->spec.size;
        double* d = net->ctx->ws[S_TMP2].as<double>((size_t)3 * P * F);
        float* dx = (float*)net->ctx->ws[S_TMP1].get(sizeof(float) * row_x * P);
        ROME_CUDA(cudaMemcpyAsync(d, Fr, sizeof(double) * P * F, cudaMemcpyHostToDevice, st));
        ROME_CUDA(cudaMemcpyAsync(d + P * F, Fi, sizeof(double) * P * F, cudaMemcpyHostToDevice, st));
        ROME_CUDA(cudaMemcpyAsync(d + 2 * P * F, ctf, sizeof(double) * P * F, cudaMemcpyHostToDevice, st));
        proposal_features_device(net, P, cur, d, d + P * F, d + 2 * P * F, dx, st);
        ROME_CUDA(cudaMemcpyAsync(x_out, dx, sizeof(float) * row_x * P, cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaStreamSynchronize(st));
    });
}

extern "C" int rome_gpu_proposal_predict(RomeProposalNet* net, int n, const float* x, int k, int* idx, float* prob) {
    if (!net || n <= 0 || !x || k <= 0 || k > net->spec.n_out || !idx) return ROME_ERR_ARG;
    return guarded(net->ctx, [&] {
        ROME_CUDA(cudaSetDevice(net->ctx->device));
        cudaStream_t st = net->ctx->stream;
        const long row_x = 2L * net->spec.size * net->spec.size;
        float* dx = (float*)net->ctx->ws[S_TMP1].get(sizeof(float) * row_x * n);
        int* di = (int*)net->ctx->ws[S_TMP0].get((sizeof(int) + sizeof(float)) * (size_t)n * k);
        float* dp = (float*)(di + (size_t)n * k);
        ROME_CUDA(cudaMemcpyAsync(dx, x, sizeof(float) * row_x * n, cudaMemcpyHostToDevice, st));
        proposal_predict_device(net, n, dx, k, di, dp, st);
        ROME_CUDA(cudaMemcpyAsync(idx, di, sizeof(int) * (size_t)n * k, cudaMemcpyDeviceToHost, st));
        if (prob) ROME_CUDA(cudaMemcpyAsync(prob, dp, sizeof(float) * (size_t)n * k, cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaStreamSynchronize(st));
    });
}
