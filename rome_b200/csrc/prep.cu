// Particle image preparation on the device: ParticleModel::setFourierTransforms
// (src/exp_model.h:397-640) for one pool, entry point rome_gpu_prepare_particles.
//
// Per chunk of images (FP64 throughout, like the reference):
//   translate_center   norm correction, integer translation by the rounded old
//                      offsets without wrap (translate -> applyGeometry,
//                      src/image.h:53-257), CenterFFT (src/image.h:344-380)
//   cuFFT D2Z          the unnormalised transform; the window kernel divides by
//                      n^2 (normalizeComplex, src/fft_base.cpp:103-109) and cuts
//                      to current_size (windowFourierTransform, src/image.h:496-566)
//   noise              the reference's noise spectra (src/exp_model.h:489-532),
//                      one warp per image, with the seeded generator restated
//                      below, written in the column transform's layout; inverse
//                      transform as column DFTs then row C2R (the decomposition
//                      of FFTW's multi-dimensional C2R, which reads only the real
//                      part of the x = 0 and x = n/2 columns)
//   mask               softMaskOutsideMap (src/image.h:571-634) with the noise
//                      image, or the raised-cosine weighted background average
//   cuFFT D2Z          masked transform -> window, power spectrum, highres_Xi2
//   ctf                CTF::getFftwImage (src/ctf.cpp:173-191, src/ctf.h:151-204)
#include <cufft.h>

#include <cmath>
#include <map>
#include <tuple>

#include "common.cuh"

namespace rome {
namespace {

#define ROME_CUFFT(call)                                                                        \
    do {                                                                                        \
        cufftResult r_ = (call);                                                                \
        if (r_ != CUFFT_SUCCESS) ::rome::fail(ROME_ERR_CUDA, "%s:%d %s: cufft error %d", __FILE__, \
                                              __LINE__, #call, (int)r_);                        \
    } while (0)

// per-particle parameter record [P][PP_COUNT] (doubles)
enum {
    PP_NORM = 0,  // NORM
    PP_DX,        // round(XOFF)
    PP_DY,        // round(YOFF)
    PP_DU,        // CTF defocus U, V, angle, voltage, Cs, Q0, B-factor
    PP_DV,
    PP_DANG,
    PP_KV,
    PP_CS,
    PP_Q0,
    PP_BFAC,
    PP_GROUP,
    PP_COUNT = 12
};

// per-particle CTF constants [P][CK_COUNT] (CTF::initialise)
enum { CK_K1 = 0, CK_K2, CK_K3, CK_K4, CK_AVG, CK_DEV, CK_C2, CK_S2, CK_Q0, CK_COUNT };

// cuFFT plans of one (image size, chunk) pair
struct PrepPlan {
    cufftHandle fwd = 0;  // D2Z 2D n x n, batch chunk
    cufftHandle col = 0;  // Z2Z 1D along rows of the (row, image) layout, batch chunk * (n/2+1)
    cufftHandle row = 0;  // Z2D 1D, batch n * chunk
};

struct PrepPlans {
    std::map<std::pair<int, int>, PrepPlan> plans;
    long tick = 0;
    std::map<std::pair<int, int>, long> used;
};

void destroy_plan(PrepPlan& p) {
    if (p.fwd) cufftDestroy(p.fwd);
    if (p.col) cufftDestroy(p.col);
    if (p.row) cufftDestroy(p.row);
    p = PrepPlan{};
}

PrepPlan& get_plan(RomeGpuCtx* ctx, PrepPlans* pp, int n, int chunk) {
    const auto key = std::make_pair(n, chunk);
    pp->used[key] = ++pp->tick;
    auto it = pp->plans.find(key);
    if (it != pp->plans.end()) return it->second;
    // keep a few plan sets (a full chunk and the remainders of recent pools)
    while (pp->plans.size() >= 4) {
        auto old = pp->plans.begin();
        for (auto jt = pp->plans.begin(); jt != pp->plans.end(); ++jt)
            if (pp->used[jt->first] < pp->used[old->first]) old = jt;
        destroy_plan(old->second);
        pp->used.erase(old->first);
        pp->plans.erase(old);
    }
    PrepPlan p;
    const int oF = n / 2 + 1;
    try {
        int dims[2] = {n, n};
        ROME_CUFFT(cufftPlanMany(&p.fwd, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_D2Z, chunk));
        int n1[1] = {n};
        int emb_c[1] = {n};
        ROME_CUFFT(cufftPlanMany(&p.col, 1, n1, emb_c, chunk * oF, 1, emb_c, chunk * oF, 1, CUFFT_Z2Z, chunk * oF));
        int emb_in[1] = {oF}, emb_out[1] = {n};
        ROME_CUFFT(cufftPlanMany(&p.row, 1, n1, emb_in, 1, oF, emb_out, 1, n, CUFFT_Z2D, n * chunk));
        ROME_CUFFT(cufftSetStream(p.fwd, ctx->stream));
        ROME_CUFFT(cufftSetStream(p.col, ctx->stream));
        ROME_CUFFT(cufftSetStream(p.row, ctx->stream));
    } catch (...) {
        destroy_plan(p);
        throw;
    }
    return pp->plans.emplace(key, p).first->second;
}

// ---------------------------------------------------------------------------
// The reference's seeded noise generator.  Random_generator with
// MAP3D_OLD_BASELINE (src/math.h:35, src/math.cpp:361-388) is std::srand /
// std::rand, i.e. glibc's TYPE_3 additive feedback generator: a table of 31
// words r[0] = seed, r[i] = 16807 r[i-1] mod (2^31 - 1); then the words
// y_s = y_{s-31} + y_{s-3} (mod 2^32) with y_{-31+i} = r[(i + 3) mod 31], the
// s-th output being y_s >> 1, and the first 310 outputs discarded.
// Uniforms are (float)rand() / (float)RAND_MAX (RAND_MAX rounds to 2^31), and
// rnd_gaus (src/math.cpp:443-480) is the polar Box-Muller method on them with
// W = pow(U1, 2) + pow(U2, 2) in double rounded to float and the multiplier
// sqrt(-2 log W / W) in double rounded to float.
//
// One warp per image.  Lane j (< 31) holds word j of the window of the last
// 31 words; the next 31 words follow in one step, as
//   y_{k+j} = y_{k+j-31} + y_{k+j-3} = sum_{m >= 0} W[j - 3m] + W[28 + j mod 3],
// a prefix sum of stride 3 over the lanes.  Two steps give 62 outputs, i.e.
// 31 Box-Muller attempts in sequence order, one per lane; a ballot ranks the
// accepted ones, and the m-th accepted attempt of the image fills the m-th
// drawing pixel (its real part from X1, its imaginary part from the cached X2,
// as rnd_gaus returns them on two consecutive calls).
constexpr unsigned kFull = 0xffffffffu;
constexpr long kM31 = 2147483647L;

__device__ __forceinline__ uint32_t glibc_step(uint32_t& W, int lane) {
    uint32_t T = W;
#pragma unroll
    for (int d = 3; d < 31; d *= 2) {  // 3, 6, 12, 24
        const uint32_t v = __shfl_up_sync(kFull, T, d);
        if (lane >= d) T += v;
    }
    const uint32_t y = T + __shfl_sync(kFull, W, 28 + lane % 3);
    W = y;
    return y >> 1;
}

__device__ __forceinline__ float rand_uniform01(uint32_t v) {
    return __fdiv_rn(__uint2float_rn(v), 2147483648.0f);
}

// one Box-Muller attempt: U1, U2 and whether W is inside the unit circle
__device__ __forceinline__ bool polar_attempt(uint32_t v1, uint32_t v2, float& U1, float& U2) {
    U1 = __fadd_rn(-1.0f, __fmul_rn(rand_uniform01(v1), 2.0f));
    U2 = __fadd_rn(-1.0f, __fmul_rn(rand_uniform01(v2), 2.0f));
    const double d1 = (double)U1, d2 = (double)U2;
    const float W = __double2float_rn(__dadd_rn(__dmul_rn(d1, d1), __dmul_rn(d2, d2)));
    return !(W >= 1.0f || W == 0.0f);
}

__device__ __forceinline__ float polar_multiplier(float U1, float U2) {
    const double d1 = (double)U1, d2 = (double)U2;
    const double W = (double)__double2float_rn(__dadd_rn(__dmul_rn(d1, d1), __dmul_rn(d2, d2)));
    return __double2float_rn(__dsqrt_rn(__ddiv_rn(-2.0 * log(W), W)));
}

// Noise spectra of the images of a chunk, written as double2 at
// out[i * si + c * sp + j] (image c, row i, column j): the (row, image) layout
// of the cuFFT column transform (si = chunk * oF, sp = oF) or one spectrum per
// image (si = oF, sp = n * oF) for the fused kernels; drawn in
// the reference's fill order (src/exp_model.h:509-534): row i, column j, real
// then imaginary part; a pixel draws when its shell ires = round(|(i', j)|)
// is < n/2+1 and its sigma sqrt(sigma2_fudge * sigma2_noise[group][ires]),
// rounded to float, is not zero (rnd_gaus returns mu without a draw for a
// zero sigma); the other pixels are zero.  Groups with the same zero shells
// share a pattern: pat_of_group [G]; per pattern, the drawing pixels in fill
// order (draw_pix from draw_start, draw_count of them) and the others
// (zero_pix from zero_start, zero_count).  sigf: [G][n/2+1].
constexpr int kNoiseWarps = 8;

__global__ void __launch_bounds__(kNoiseWarps * 32) noise_spectra_kernel(
    int P, int npix, int oF, uint32_t seed0, const double* __restrict__ part, const int* __restrict__ pat_of_group,
    const int* __restrict__ draw_start, const int* __restrict__ draw_count, const int* __restrict__ draw_pix,
    const int* __restrict__ zero_start, const int* __restrict__ zero_count, const int* __restrict__ zero_pix,
    const unsigned short* __restrict__ ires_tab, const float* __restrict__ sigf, long si, long sp,
    double2* __restrict__ out) {
    const int img = blockIdx.x * kNoiseWarps + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (img >= P) return;  // whole warps leave together
    const int g = (int)part[(size_t)img * PP_COUNT + PP_GROUP], pat = pat_of_group[g];
    const float* sig = sigf + (size_t)g * oF;
    // seeding (srandom_r): lane i holds r[i] = 16807^i r[0] mod (2^31 - 1), i >= 1
    uint32_t seed = seed0 + (uint32_t)img;
    if (seed == 0) seed = 1;
    const int32_t r0 = (int32_t)seed;
    uint32_t init = (uint32_t)r0;
    if (lane >= 1 && lane < 31) {
        long w = (long)r0 % kM31;
        if (w < 0) w += kM31;
        long a = 1;
        for (int i = 0; i < lane; ++i) a = (a * 16807L) % kM31;
        init = (uint32_t)((a * w) % kM31);
    }
    uint32_t W = __shfl_sync(kFull, init, lane < 31 ? (lane + 3) % 31 : 0);
    if (lane == 31) W = 0;
    for (int k = 0; k < 10; ++k) glibc_step(W, lane);  // 310 outputs discarded
    const int need = draw_count[pat];
    const int* dp = draw_pix + draw_start[pat];
    int base = 0;
    while (base < need) {
        const uint32_t A = glibc_step(W, lane), B = glibc_step(W, lane);
        // attempt `lane` uses outputs 2 lane and 2 lane + 1 of the 62
        const int v1 = 2 * lane, v2 = 2 * lane + 1;
        const uint32_t a1 = __shfl_sync(kFull, A, v1 < 31 ? v1 : 0), b1 = __shfl_sync(kFull, B, v1 >= 31 ? v1 - 31 : 0);
        const uint32_t a2 = __shfl_sync(kFull, A, v2 < 31 ? v2 : 0), b2 = __shfl_sync(kFull, B, v2 >= 31 ? v2 - 31 : 0);
        float U1 = 0.f, U2 = 0.f;
        const bool ok = lane < 31 && polar_attempt(v1 < 31 ? a1 : b1, v2 < 31 ? a2 : b2, U1, U2);
        const unsigned mask = __ballot_sync(kFull, ok);
        const int m = base + __popc(mask & ((1u << lane) - 1u));
        if (ok && m < need) {
            const int q = dp[m];
            const float s = sig[ires_tab[q]];
            const float mult = polar_multiplier(U1, U2);
            const float X1 = __fmul_rn(U1, mult), X2 = __fmul_rn(U2, mult);
            const int i = q / oF;
            out[i * si + img * sp + (q - i * oF)] =
                make_double2((double)__fadd_rn(0.0f, __fmul_rn(s, X1)), (double)__fadd_rn(0.0f, __fmul_rn(s, X2)));
        }
        base += __popc(mask);
    }
    const int* zp = zero_pix + zero_start[pat];
    for (int k = lane; k < zero_count[pat]; k += 32) {
        const int q = zp[k], i = q / oF;
        out[i * si + img * sp + (q - i * oF)] = make_double2(0.0, 0.0);
    }
}

// value of the norm-corrected, translated image at (a, b): exp_image after
// `translate(tempImage, exp_image, ori, round(XOFF), round(YOFF), DONT_WRAP)`;
// an integer shift makes applyGeometry's bilinear weights 0 / 1, so it is a
// copy from (a - dy, b - dx) with zeros where that leaves the image
template <typename T>
__device__ __forceinline__ double translated_at(const T* __restrict__ img, int n, int a, int b, int dx, int dy,
                                                int do_norm, double avg, double norm) {
    const int sa = a - dy, sb = b - dx;
    if (sa < 0 || sa >= n || sb < 0 || sb >= n) return 0.0;
    double v = (double)img[(size_t)sa * n + sb];
    if (do_norm) v = __ddiv_rn(__dmul_rn(v, avg), norm);
    return v;
}

// The per-pixel kernels below run a 2D grid: x over the pixels of one image,
// y over the images of the chunk (looping when there are more than 65535).

// CenterFFT(forward) of the translated image: out[i][j] = t[(i - n/2) mod n][(j - n/2) mod n].
// Each thread handles 4 pixels 256 apart (4 loads in flight); blocks of 256.
template <typename T>
__global__ void translate_center_kernel(int chunk, int n, const T* __restrict__ raw, const double* __restrict__ part,
                                        int do_norm, double avg, double* __restrict__ out) {
    const int nn = n * n, h = n / 2;
    for (int p = blockIdx.y; p < chunk; p += gridDim.y) {
        const double* pp = part + (size_t)p * PP_COUNT;
        const int dx = (int)pp[PP_DX], dy = (int)pp[PP_DY];
        const double norm = pp[PP_NORM];
        const T* img = raw + (size_t)p * nn;
        for (int q0 = blockIdx.x * 1024 + threadIdx.x; q0 < nn; q0 += gridDim.x * 1024) {
            double v[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int q = q0 + 256 * k;
                v[k] = 0.0;
                if (q < nn) {
                    const int i = q / n, j = q - (q / n) * n;
                    const int a = i - h < 0 ? i - h + n : i - h, b = j - h < 0 ? j - h + n : j - h;
                    v[k] = translated_at(img, n, a, b, dx, dy, do_norm, avg, norm);
                }
            }
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (q0 + 256 * k < nn) out[(size_t)p * nn + q0 + 256 * k] = v[k];
        }
    }
}

// windowFourierTransform of the normalised transform: F [chunk][n][n/2+1]
// (unnormalised) -> out [chunk][fine][fine/2+1], component / n^2
__global__ void window_kernel(int chunk, int n, int fine, const double2* __restrict__ F, double* __restrict__ out_re,
                              double* __restrict__ out_im) {
    const int oF = n / 2 + 1, fF = fine / 2 + 1, per = fine * fF;
    const double nn = (double)n * (double)n;
    for (int p = blockIdx.y; p < chunk; p += gridDim.y) {
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < per; q += gridDim.x * blockDim.x) {
            const int i = q / fF, j = q - (q / fF) * fF;
            const int ip = i < fF ? i : i - fine;
            const int si = ip < 0 ? ip + n : ip;
            const double2 v = F[((size_t)p * n + si) * oF + j];
            out_re[(size_t)p * per + q] = __ddiv_rn(v.x, nn);
            out_im[(size_t)p * per + q] = __ddiv_rn(v.y, nn);
        }
    }
}

// after the column DFTs: each row's C2R reads only the real part of its x = 0
// and x = n/2 entries (what FFTW's half-complex backward transform does)
__global__ void real_edges_kernel(long rows, int oF, int n, double2* __restrict__ nc) {
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (long)gridDim.x * blockDim.x) {
        nc[r * oF].y = 0.0;
        if ((n & 1) == 0) nc[r * oF + n / 2].y = 0.0;
    }
}

// softMaskOutsideMap's background average (no noise image): sum of w * value
// over the pixels at r >= radius divided by sum of w.  mw: the mask weight of
// every uncentred pixel (< 0 inside the radius, the raised cosine in the edge
// band, > 1 beyond radius + width, where w = 1).  One block of 256 per image.
template <typename T>
__global__ void background_kernel(int n, const T* __restrict__ raw, const double* __restrict__ part, int do_norm,
                                  double avg, const double* __restrict__ mw, double* __restrict__ bg) {
    const int p = blockIdx.x;
    const double* pp = part + (size_t)p * PP_COUNT;
    const T* img = raw + (size_t)p * n * n;
    const int dx = (int)pp[PP_DX], dy = (int)pp[PP_DY];
    double s = 0.0, sw = 0.0;
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
        const double w0 = mw[q];
        if (w0 < 0.0) continue;
        const double w = w0 > 1.0 ? 1.0 : w0;
        const int a = q / n, b = q - (q / n) * n;
        s += w * translated_at(img, n, a, b, dx, dy, do_norm, avg, pp[PP_NORM]);
        sw += w;
    }
    __shared__ double red[2][256];
    red[0][threadIdx.x] = s;
    red[1][threadIdx.x] = sw;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) {
            red[0][threadIdx.x] += red[0][threadIdx.x + k];
            red[1][threadIdx.x] += red[1][threadIdx.x + k];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) bg[p] = red[0][0] / red[1][0];
}

// softMaskOutsideMap of the translated image, written centred (CenterFFT):
// inside the radius the pixel stays, in the edge band it becomes
// (1 - w) * value + w * add, beyond it `add` -- the noise image at the same
// uncentred pixel, or the background average
template <typename T>
__global__ void mask_center_kernel(int chunk, int n, const T* __restrict__ raw, const double* __restrict__ part,
                                   int do_norm, double avg, const double* __restrict__ mw,
                                   const double* __restrict__ noise_img, const double* __restrict__ bg,
                                   double* __restrict__ out) {
    const int nn = n * n, h = n / 2;
    for (int p = blockIdx.y; p < chunk; p += gridDim.y) {
        const double* pp = part + (size_t)p * PP_COUNT;
        const int dx = (int)pp[PP_DX], dy = (int)pp[PP_DY];
        const double norm = pp[PP_NORM];
        const T* img = raw + (size_t)p * nn;
        for (int q0 = blockIdx.x * 1024 + threadIdx.x; q0 < nn; q0 += gridDim.x * 1024) {
            double v[4], w[4], add[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int q = q0 + 256 * k;
                v[k] = 0.0;
                w[k] = -1.0;
                add[k] = 0.0;
                if (q < nn) {
                    const int i = q / n, j = q - (q / n) * n;
                    const int a = i - h < 0 ? i - h + n : i - h, b = j - h < 0 ? j - h + n : j - h;
                    v[k] = translated_at(img, n, a, b, dx, dy, do_norm, avg, norm);
                    w[k] = mw[a * n + b];
                    add[k] = noise_img ? noise_img[((size_t)a * chunk + p) * n + b] : bg[p];
                }
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                double x = v[k];
                if (w[k] >= 0.0) x = w[k] > 1.0 ? add[k] : (1 - w[k]) * v[k] + w[k] * add[k];
                if (q0 + 256 * k < nn) out[(size_t)p * nn + q0 + 256 * k] = x;
            }
        }
    }
}

// power spectrum of the masked, normalised transform over shells 1..n/2
// (the x = 0 column's negative rows skipped) and highres_Xi2, the sum over
// shells >= current_size/2+1.  One block per image; thread s sums shell s
// over its pixels in row-major order (the reference's order within a shell).
// shell_start [oF+1], shell_pix: pixel indices i * oF + j by shell.
__global__ void power_kernel(int n, int fine, const double2* __restrict__ F, const int* __restrict__ shell_start,
                             const int* __restrict__ shell_pix, double* __restrict__ power, double* __restrict__ xi2) {
    const int p = blockIdx.x, oF = n / 2 + 1, fF = fine / 2 + 1;
    const double nn = (double)n * (double)n;
    const double2* f = F + (size_t)p * n * oF;
    extern __shared__ double spec[];
    for (int s = threadIdx.x; s < oF; s += blockDim.x) {
        double acc = 0.0;
        for (int k = shell_start[s]; k < shell_start[s + 1]; ++k) {
            const double2 v = f[shell_pix[k]];
            const double re = __ddiv_rn(v.x, nn), im = __ddiv_rn(v.y, nn);
            acc += re * re + im * im;
        }
        spec[s] = acc;
        power[(size_t)p * oF + s] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double x = 0.0;
        for (int s = fF; s < oF; ++s) x += spec[s];
        xi2[p] = x;
    }
}

// CTF::initialise (src/ctf.cpp:136-171) per particle: [P][CK_COUNT]
__global__ void ctf_constants_kernel(int P, const double* __restrict__ part, double* __restrict__ ck) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    const double* pp = part + (size_t)p * PP_COUNT;
    double* k = ck + (size_t)p * CK_COUNT;
    const double local_cs = pp[PP_CS] * 1e7, local_kv = pp[PP_KV] * 1e3;
    const double rad_az = pp[PP_DANG] * kPi / 180.0;
    const double lambda = 12.2643247 / sqrt(local_kv * (1. + local_kv * 0.978466e-6));
    k[CK_K1] = kPi / 2 * 2 * lambda;
    k[CK_K2] = kPi / 2 * local_cs * lambda * lambda * lambda;
    k[CK_K3] = sqrt(1 - pp[PP_Q0] * pp[PP_Q0]);
    k[CK_K4] = -pp[PP_BFAC] / 4.;
    k[CK_AVG] = -(pp[PP_DU] + pp[PP_DV]) * 0.5;
    k[CK_DEV] = -(pp[PP_DU] - pp[PP_DV]) * 0.5;
    k[CK_C2] = cos(2 * rad_az);
    k[CK_S2] = sin(2 * rad_az);
    k[CK_Q0] = pp[PP_Q0];
}

// CTF::getFftwImage(fine, ori, ori, angpix, do_abs, only_flip, intact_first_peak,
// damping on) (src/ctf.cpp:173-191, getCTF / getDeltaF src/ctf.h:151-204);
// cos(2 (atan2(Y, X) - azimuth)) as ((X^2 - Y^2) cos 2az + 2XY sin 2az) / |u|^2
__global__ void ctf_kernel(int P, int fine, int ori, double angpix, const double* __restrict__ ck, int do_abs,
                           int only_flip, int intact, double* __restrict__ out) {
    const int fF = fine / 2 + 1, per = fine * fF;
    const double xs = (double)ori * angpix;
    for (int p = blockIdx.y; p < P; p += gridDim.y) {
        const double* k = ck + (size_t)p * CK_COUNT;
        const double K1 = k[CK_K1], K2 = k[CK_K2], K3 = k[CK_K3], K4 = k[CK_K4], avg = k[CK_AVG], dev = k[CK_DEV],
                     c2 = k[CK_C2], s2 = k[CK_S2], q0 = k[CK_Q0];
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < per; q += gridDim.x * blockDim.x) {
            const int i = q / fF, j = q - (q / fF) * fF;
            const int ip = i < fF ? i : i - fine;
            const double X = (double)j / xs, Y = (double)ip / xs;
            const double u2 = X * X + Y * Y, u4 = u2 * u2;
            const double deltaf =
                (fabs(X) < 1e-6 && fabs(Y) < 1e-6) ? 0.0 : avg + dev * (((X * X - Y * Y) * c2 + 2 * X * Y * s2) / u2);
            const double arg = K1 * deltaf * u2 + K2 * u4;
            double v;
            if (intact && fabs(arg) < kPi / 2.) {
                v = 1.;
            } else {
                double sn, cs;
                sincos(arg, &sn, &cs);
                v = -(K3 * sn - q0 * cs);
            }
            if (K4 != 0.0) v *= exp(K4 * u2);
            if (do_abs) v = fabs(v);
            else if (only_flip) v = v < 0. ? -1. : 1.;
            out[(size_t)p * per + q] = v;
        }
    }
}

// ---------------------------------------------------------------------------
// Fused preparation for power-of-two sizes n = 32 E (E = 1, 2, 4): one CTA
// holds one image's half-plane spectrum in shared memory, and every 1D
// transform is one warp's: lane l holds elements l + 32 m (m < E); an E-point
// DFT over m, the twiddles W_n^(l k1), then a 32-point radix-2
// decimation-in-frequency DFT across the lanes by shuffles leave element
// k1 + E * bitrev5(l) in lane l.  Two real rows go through one complex
// transform (a + i b), split into their half spectra after it; the inverse
// real transforms take two half rows the same way.  The 2D order is the one
// of FFTW's multi-dimensional real transforms: rows then columns forward,
// columns then rows backward, the backward row transforms reading only the
// real part of the x = 0 and x = n/2 entries.  CenterFFT is the factor
// (-1)^(i + j) on the spectrum (an n/2 shift of an even-sized image).

constexpr int kFusedWarps = 32;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 shfl_xor2(double2 v, int m) {
    return make_double2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

// the warp's length-32E transform; tw[q] = exp(-2 pi i q / (32 E)), conjugated for the inverse (unnormalised).
// In: lane l holds element l + 32 m in v[m].  Out: lane l holds element k1 + E bitrev5(l) in v[k1].
template <int E, bool INV>
__device__ __forceinline__ void warp_fft(double2 (&v)[E], int lane, const double2* __restrict__ tw) {
    constexpr int N = 32 * E;
    auto W = [&](int q) {
        const double2 t = tw[q];
        return INV ? make_double2(t.x, -t.y) : t;
    };
    if constexpr (E == 2) {
        const double2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (E == 4) {
        const double2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        const double2 b0 = cadd(v[1], v[3]), b1 = csub(v[1], v[3]);
        // b1 times -i (forward) or +i (inverse)
        const double2 r = INV ? make_double2(-b1.y, b1.x) : make_double2(b1.y, -b1.x);
        v[0] = cadd(a0, b0);
        v[1] = cadd(a1, r);
        v[2] = csub(a0, b0);
        v[3] = csub(a1, r);
    }
#pragma unroll
    for (int k1 = 1; k1 < E; ++k1) v[k1] = cmul(v[k1], W((lane * k1) & (N - 1)));
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
        const bool upper = lane & s;
        const double2 w = W((lane & (s - 1)) * (N / (2 * s)));
#pragma unroll
        for (int k1 = 0; k1 < E; ++k1) {
            const double2 o = shfl_xor2(v[k1], s);
            v[k1] = upper ? cmul(csub(o, v[k1]), w) : cadd(v[k1], o);
        }
    }
}

__device__ __forceinline__ int bitrev5(int l) { return (int)(__brev((unsigned)l) >> 27); }

// Shared-memory positions.  The transforms leave element k1 + E bitrev5(l)
// in lane l: rows (or scratch entries) 4 apart for consecutive lanes, which
// with 16-byte elements would put 16 lanes on the same banks.  Element
// (row, c) of the spectrum sits at column c ^ ((row >> 2) & 7) of its row (c
// below n/2; the n/2 column stays), scratch entry k at k ^ ((k >> 3) & 7) in
// its group of 8: row-wise, column-wise and bit-reversed accesses then all
// take the minimum of 4 wavefronts per warp.
template <int N>
__device__ __forceinline__ int zidx(int row, int c) {
    constexpr int LD = N / 2 + 1;
    return row * LD + (c < N / 2 ? c ^ ((row >> 2) & 7) : c);
}
__device__ __forceinline__ int sidx(int k) { return (k & ~7) | ((k ^ (k >> 3)) & 7); }

// shared memory of the fused kernels: the spectrum Z [n][n/2+1] (a row also
// holds the n doubles of a real row), per-warp scratch [16][n], twiddles [n],
// the power shells [n/2+1], a reduction area
template <int E>
struct FusedSmem {
    static constexpr int N = 32 * E, LD = N / 2 + 1;
    static constexpr size_t Z = (size_t)N * LD * 16, SCR = (size_t)kFusedWarps * N * 16, TW = (size_t)N * 16,
                            SPEC = ((size_t)LD * 8 + 15) / 16 * 16, RED = 2 * kFusedWarps * 32 * 8;
    static constexpr size_t TOTAL = Z + SCR + TW + SPEC + RED;
};

// forward transform of the n real rows held in Z (row i's doubles at the
// start of its slot), or produced by load_row(i, x), into the half-plane
// spectrum in Z: rows in pairs, then the columns
template <int E, typename LoadRow>
__device__ __forceinline__ void fused_forward(double2* Z, double2* scr, const double2* tw, LoadRow load_row) {
    constexpr int N = 32 * E;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double2* my = scr + warp * N;
    for (int r = warp; r < N / 2; r += kFusedWarps) {
        double2 v[E];
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = make_double2(load_row(2 * r, lane + 32 * m), load_row(2 * r + 1, lane + 32 * m));
        warp_fft<E, false>(v, lane, tw);
#pragma unroll
        for (int k1 = 0; k1 < E; ++k1) my[sidx(k1 + E * bitrev5(lane))] = v[k1];
        __syncwarp();
        for (int k = lane; k <= N / 2; k += 32) {
            const double2 a = my[sidx(k)], b = my[sidx((N - k) & (N - 1))];
            Z[zidx<N>(2 * r, k)] = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
            Z[zidx<N>(2 * r + 1, k)] = make_double2(0.5 * (a.y + b.y), 0.5 * (b.x - a.x));
        }
        __syncwarp();
    }
    __syncthreads();
    // columns 1 .. n/2-1, and columns 0 and n/2 (real after the row pass) as one complex column
    for (int c = warp; c < N / 2; c += kFusedWarps) {
        double2 v[E];
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int row = lane + 32 * m;
            v[m] = c ? Z[zidx<N>(row, c)] : make_double2(Z[zidx<N>(row, 0)].x, Z[zidx<N>(row, N / 2)].x);
        }
        warp_fft<E, false>(v, lane, tw);
        __syncwarp();
        if (c) {
#pragma unroll
            for (int k1 = 0; k1 < E; ++k1) Z[zidx<N>(k1 + E * bitrev5(lane), c)] = v[k1];
        } else {
#pragma unroll
            for (int k1 = 0; k1 < E; ++k1) my[sidx(k1 + E * bitrev5(lane))] = v[k1];
            __syncwarp();
            for (int k = lane; k < N; k += 32) {
                const double2 a = my[sidx(k)], b = my[sidx((N - k) & (N - 1))];
                Z[zidx<N>(k, 0)] = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
                Z[zidx<N>(k, N / 2)] = make_double2(0.5 * (a.y + b.y), 0.5 * (b.x - a.x));
            }
        }
        __syncwarp();
    }
    __syncthreads();
}

// backward transform of the half-plane spectrum in Z into n real rows (in
// place, each row's doubles at the start of its slot), unnormalised
template <int E>
__device__ __forceinline__ void fused_backward(double2* Z, const double2* tw) {
    constexpr int N = 32 * E, LD = N / 2 + 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // columns 1 .. n/2-1; columns 0 and n/2 enter the row transforms by their
    // real parts only, so they go together as one complex column of their
    // Hermitian parts h[k] = (s[k] + conj(s[-k])) / 2 (real inverse transforms)
    for (int c = warp; c < N / 2; c += kFusedWarps) {
        double2 v[E];
        if (c) {
#pragma unroll
            for (int m = 0; m < E; ++m) v[m] = Z[zidx<N>(lane + 32 * m, c)];
        } else {
            double2 s0[E], s1[E];
#pragma unroll
            for (int m = 0; m < E; ++m) {
                s0[m] = Z[zidx<N>(lane + 32 * m, 0)];
                s1[m] = Z[zidx<N>(lane + 32 * m, N / 2)];
            }
            // element n - k of element k = l + 32 m sits in lane (32 - l) & 31, slot E-1-m (slot (E-m) mod E in lane 0)
#pragma unroll
            for (int m = 0; m < E; ++m) {
                double2 t0 = s0[E - 1 - m], t1 = s1[E - 1 - m];
                if (lane == 0) {
                    t0 = s0[(E - m) % E];
                    t1 = s1[(E - m) % E];
                }
                const int from = (32 - lane) & 31;
                const double2 r0 = make_double2(__shfl_sync(0xffffffffu, t0.x, from), __shfl_sync(0xffffffffu, t0.y, from));
                const double2 r1 = make_double2(__shfl_sync(0xffffffffu, t1.x, from), __shfl_sync(0xffffffffu, t1.y, from));
                const double2 h0 = make_double2(0.5 * (s0[m].x + r0.x), 0.5 * (s0[m].y - r0.y));
                const double2 h1 = make_double2(0.5 * (s1[m].x + r1.x), 0.5 * (s1[m].y - r1.y));
                v[m] = make_double2(h0.x - h1.y, h0.y + h1.x);  // h0 + i h1
            }
        }
        warp_fft<E, true>(v, lane, tw);
        __syncwarp();
        if (c) {
#pragma unroll
            for (int k1 = 0; k1 < E; ++k1) Z[zidx<N>(k1 + E * bitrev5(lane), c)] = v[k1];
        } else {
#pragma unroll
            for (int k1 = 0; k1 < E; ++k1) {
                const int row = k1 + E * bitrev5(lane);
                Z[zidx<N>(row, 0)] = make_double2(v[k1].x, 0.0);
                Z[zidx<N>(row, N / 2)] = make_double2(v[k1].y, 0.0);
            }
        }
    }
    __syncthreads();
    for (int r = warp; r < N / 2; r += kFusedWarps) {
        double2 v[E];
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int k = lane + 32 * m;
            double2 a, b;
            if (k <= N / 2) {
                a = Z[zidx<N>(2 * r, k)];
                b = Z[zidx<N>(2 * r + 1, k)];
                if (k == 0 || k == N / 2) a.y = b.y = 0.0;
            } else {
                a = Z[zidx<N>(2 * r, N - k)];
                b = Z[zidx<N>(2 * r + 1, N - k)];
                a.y = -a.y;
                b.y = -b.y;
            }
            v[m] = make_double2(a.x - b.y, a.y + b.x);  // a + i b
        }
        warp_fft<E, true>(v, lane, tw);
        __syncwarp();
        double* ra = (double*)(Z + (2 * r) * LD);
        double* rb = (double*)(Z + (2 * r + 1) * LD);
#pragma unroll
        for (int k1 = 0; k1 < E; ++k1) {
            const int x = k1 + E * bitrev5(lane);
            ra[x] = v[k1].x;
            rb[x] = v[k1].y;
        }
    }
    __syncthreads();
}

// window of the centred, normalised spectrum in Z to [fine][fine/2+1]
template <int E>
__device__ __forceinline__ void fused_window(const double2* Z, int fine, double* __restrict__ re, double* __restrict__ im) {
    constexpr int N = 32 * E;
    const int fF = fine / 2 + 1, per = fine * fF;
    const double nn = (double)N * N;
    for (int q = threadIdx.x; q < per; q += blockDim.x) {
        const int i = q / fF, j = q - (q / fF) * fF;
        const int ip = i < fF ? i : i - fine;
        const int si = ip < 0 ? ip + N : ip;
        const double2 v = Z[zidx<N>(si, j)];
        const double sg = ((si + j) & 1) ? -1.0 : 1.0;
        re[q] = sg * __ddiv_rn(v.x, nn);
        im[q] = sg * __ddiv_rn(v.y, nn);
    }
}

template <int E>
__device__ __forceinline__ void load_twiddles(double2* tw, const double2* __restrict__ gtw) {
    for (int q = threadIdx.x; q < 32 * E; q += blockDim.x) tw[q] = gtw[q];
}

// Fimages_nomask: translate, centre, transform, window, one image per CTA iteration
template <int E, typename T>
__global__ void __launch_bounds__(kFusedWarps * 32) fused_nomask_kernel(int chunk, int fine, const T* __restrict__ raw,
                                                                        const double* __restrict__ part, int do_norm,
                                                                        double avg, const double2* __restrict__ gtw,
                                                                        double* __restrict__ out_re,
                                                                        double* __restrict__ out_im) {
    using L = FusedSmem<E>;
    constexpr int N = 32 * E;
    extern __shared__ __align__(16) unsigned char sm[];
    double2* Z = (double2*)sm;
    double2* scr = (double2*)(sm + L::Z);
    double2* tw = (double2*)(sm + L::Z + L::SCR);
    load_twiddles<E>(tw, gtw);
    __syncthreads();
    const int Ff = fine * (fine / 2 + 1);
    for (int p = blockIdx.x; p < chunk; p += gridDim.x) {
        const double* pp = part + (size_t)p * PP_COUNT;
        const int dx = (int)pp[PP_DX], dy = (int)pp[PP_DY];
        const double norm = pp[PP_NORM];
        const T* img = raw + (size_t)p * N * N;
        fused_forward<E>(Z, scr, tw, [&](int a, int b) { return translated_at(img, N, a, b, dx, dy, do_norm, avg, norm); });
        fused_window<E>(Z, fine, out_re + (size_t)p * Ff, out_im + (size_t)p * Ff);
        __syncthreads();
    }
}

// Fimages_mask: noise image (backward transform of the chunk's noise spectra
// [chunk][n][n/2+1]) or background average, soft mask, transform, window,
// power spectrum and highres_Xi2
template <int E, typename T>
__global__ void __launch_bounds__(kFusedWarps * 32) fused_masked_kernel(
    int chunk, int fine, const T* __restrict__ raw, const double* __restrict__ part, int do_norm, double avg,
    const double2* __restrict__ gtw, const double* __restrict__ mw, const double2* __restrict__ noise,
    const int* __restrict__ shell_start, const int* __restrict__ shell_pix, double* __restrict__ out_re,
    double* __restrict__ out_im, double* __restrict__ power, double* __restrict__ xi2) {
    using L = FusedSmem<E>;
    constexpr int N = 32 * E, LD = N / 2 + 1;
    extern __shared__ __align__(16) unsigned char sm[];
    double2* Z = (double2*)sm;
    double2* scr = (double2*)(sm + L::Z);
    double2* tw = (double2*)(sm + L::Z + L::SCR);
    double* spec = (double*)(sm + L::Z + L::SCR + L::TW);
    double* red = (double*)(sm + L::Z + L::SCR + L::TW + L::SPEC);
    load_twiddles<E>(tw, gtw);
    __syncthreads();
    const int Ff = fine * (fine / 2 + 1), fF = fine / 2 + 1;
    const double nn = (double)N * N;
    for (int p = blockIdx.x; p < chunk; p += gridDim.x) {
        const double* pp = part + (size_t)p * PP_COUNT;
        const int dx = (int)pp[PP_DX], dy = (int)pp[PP_DY];
        const double norm = pp[PP_NORM];
        const T* img = raw + (size_t)p * N * N;
        double bg = 0.0;
        if (noise) {
            const double2* ns = noise + (size_t)p * N * LD;
            for (int q = threadIdx.x; q < N * LD; q += blockDim.x) Z[zidx<N>(q / LD, q % LD)] = ns[q];
            __syncthreads();
            fused_backward<E>(Z, tw);
        } else {
            // softMaskOutsideMap's weighted background average
            double s = 0.0, sw = 0.0;
            for (int q = threadIdx.x; q < N * N; q += blockDim.x) {
                const double w0 = mw[q];
                if (w0 < 0.0) continue;
                const double w = w0 > 1.0 ? 1.0 : w0;
                s += w * translated_at(img, N, q / N, q % N, dx, dy, do_norm, avg, norm);
                sw += w;
            }
            red[threadIdx.x] = s;
            red[blockDim.x + threadIdx.x] = sw;
            __syncthreads();
            for (int k = blockDim.x / 2; k > 0; k >>= 1) {
                if (threadIdx.x < k) {
                    red[threadIdx.x] += red[threadIdx.x + k];
                    red[blockDim.x + threadIdx.x] += red[blockDim.x + threadIdx.x + k];
                }
                __syncthreads();
            }
            bg = red[0] / red[blockDim.x];
            __syncthreads();
        }
        // soft mask into the real rows of Z (uncentred); 4 pixels per thread per step, loads first
        for (int q0 = threadIdx.x; q0 < N * N; q0 += 4 * blockDim.x) {
            double v[4], w[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int q = q0 + u * blockDim.x;
                v[u] = 0.0;
                w[u] = -1.0;
                if (q < N * N) {
                    v[u] = translated_at(img, N, q / N, q % N, dx, dy, do_norm, avg, norm);
                    w[u] = mw[q];
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int q = q0 + u * blockDim.x;
                if (q >= N * N) continue;
                double* row = (double*)(Z + (q / N) * LD);
                double x = v[u];
                if (w[u] >= 0.0) {
                    const double add = noise ? row[q % N] : bg;
                    x = w[u] > 1.0 ? add : (1 - w[u]) * x + w[u] * add;
                }
                row[q % N] = x;
            }
        }
        __syncthreads();
        fused_forward<E>(Z, scr, tw, [&](int a, int b) { return ((const double*)(Z + a * LD))[b]; });
        fused_window<E>(Z, fine, out_re + (size_t)p * Ff, out_im + (size_t)p * Ff);
        if (fine < N) {
            for (int sh = threadIdx.x; sh < LD; sh += blockDim.x) {
                double acc = 0.0;
                for (int k = shell_start[sh]; k < shell_start[sh + 1]; ++k) {
                    const int q = shell_pix[k];  // pixel i * (n/2+1) + j
                    const double2 v = Z[zidx<N>(q / LD, q % LD)];
                    const double re = __ddiv_rn(v.x, nn), im = __ddiv_rn(v.y, nn);
                    acc += re * re + im * im;
                }
                spec[sh] = acc;
                power[(size_t)p * LD + sh] = acc;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                double x = 0.0;
                for (int sh = fF; sh < LD; ++sh) x += spec[sh];
                xi2[p] = x;
            }
        }
        __syncthreads();
    }
}

}  // namespace

namespace {

__global__ void fill_kernel(double* __restrict__ x, size_t n, double v) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) x[i] = v;
}

unsigned grid_for(size_t total, int threads = 256) {
    return (unsigned)std::max<size_t>(1, std::min<size_t>((total + threads - 1) / threads, 148 * 16));
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// 2D grid of the per-pixel kernels: x covers `per_image` elements with 256
// threads, y the images (at most 65535; the kernels loop over the rest)
dim3 grid2(size_t per_image, int images) {
    return dim3((unsigned)std::max<size_t>(1, (per_image + 255) / 256), (unsigned)std::max(1, std::min(images, 65535)));
}

// C round(): halfway cases away from zero
double c_round(double x) { return std::round(x); }

// the host-built tables of the preparation and where they sit in S_PREP_TAB
struct PrepTables {
    bool valid = false;
    std::vector<double> key;  // sizes, mask radius and width, sigma2_fudge, sigma2_noise
    size_t o_ires = 0, o_sig = 0, o_pog = 0, o_dst = 0, o_dcn = 0, o_dpx = 0, o_zst = 0, o_zcn = 0, o_zpx = 0, o_ss = 0,
           o_sp = 0, o_mw = 0, o_tw = 0;
};

struct PrepState {
    PrepPlans plans;
    PrepTables tables;
    // a second stream for the work that does not need the images (noise
    // spectra, CTF images), overlapping the unmasked path on the context's
    cudaStream_t side = nullptr;
    cudaEvent_t ev_ready = nullptr, ev_noise = nullptr, ev_nc_free = nullptr, ev_ctf = nullptr;
};

PrepState* prep_state(RomeGpuCtx* ctx) {
    if (!ctx->prep_plans) ctx->prep_plans = new PrepState();
    auto* ps = (PrepState*)ctx->prep_plans;
    if (!ps->side) {
        ROME_CUDA(cudaStreamCreateWithFlags(&ps->side, cudaStreamNonBlocking));
        for (cudaEvent_t* e : {&ps->ev_ready, &ps->ev_noise, &ps->ev_nc_free, &ps->ev_ctf})
            ROME_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    return ps;
}

void build_tables(RomeGpuCtx* ctx, PrepTables& tb, int n, int fine, int G, bool noise, double radius, double width,
                  double sigma2_fudge, const double* sigma2_noise) {
    const int oF = n / 2 + 1;
    const size_t npix = (size_t)n * oF, nn = (size_t)n * n;
    (void)fine;
    // shell of every half-plane pixel, round(sqrt(i'^2 + j^2)) (src/exp_model.h:514-516)
    std::vector<unsigned short> ires(npix);
    for (int i = 0; i < n; ++i) {
        const int ip = i < oF ? i : i - n;
        for (int j = 0; j < oF; ++j) ires[(size_t)i * oF + j] = (unsigned short)std::round(std::sqrt((double)(ip * ip + j * j)));
    }
    std::vector<float> sigf((size_t)G * oF, 0.f);
    // groups with the same zero-sigma shells share one list of drawing pixels
    std::vector<int> pat_of_group(G, 0), draw_start, draw_count, draw_pix, zero_start, zero_count, zero_pix;
    if (noise) {
        std::map<std::vector<int>, int> patterns;
        for (int g = 0; g < G; ++g) {
            std::vector<int> zero_shells;
            for (int s = 0; s < oF; ++s) {
                const double pw = sigma2_fudge * sigma2_noise[(size_t)g * oF + s];
                ROME_REQUIRE(pw >= 0.0, "sigma2_noise[%d][%d] is negative", g, s);
                sigf[(size_t)g * oF + s] = (float)std::sqrt(pw);
                if (sigf[(size_t)g * oF + s] == 0.f) zero_shells.push_back(s);
            }
            auto it = patterns.find(zero_shells);
            if (it == patterns.end()) {
                const int id = (int)patterns.size();
                it = patterns.emplace(zero_shells, id).first;
                std::vector<char> zs(oF, 0);
                for (int s : zero_shells) zs[s] = 1;
                draw_start.push_back((int)draw_pix.size());
                zero_start.push_back((int)zero_pix.size());
                for (size_t q = 0; q < npix; ++q) {
                    if (ires[q] < oF && !zs[ires[q]]) draw_pix.push_back((int)q);
                    else zero_pix.push_back((int)q);
                }
                draw_count.push_back((int)draw_pix.size() - draw_start.back());
                zero_count.push_back((int)zero_pix.size() - zero_start.back());
            }
            pat_of_group[g] = it->second;
        }
    }
    // shells 1..oF-1 of the power spectrum, pixels in row-major order, the
    // negative rows of the x = 0 column skipped (src/exp_model.h:576-595)
    std::vector<int> shell_start(oF + 1, 0), shell_pix;
    {
        std::vector<std::vector<int>> by(oF);
        for (int i = 0; i < n; ++i) {
            const int ip = i < oF ? i : i - n;
            for (int j = 0; j < oF; ++j) {
                const int s = ires[(size_t)i * oF + j];
                if (s > 0 && s < oF && !(j == 0 && ip < 0)) by[s].push_back(i * oF + j);
            }
        }
        for (int s = 0; s < oF; ++s) {
            shell_start[s + 1] = shell_start[s] + (int)by[s].size();
            shell_pix.insert(shell_pix.end(), by[s].begin(), by[s].end());
        }
    }
    // softMaskOutsideMap's weight of every (uncentred) pixel: < 0 inside the
    // radius, the raised cosine in the edge band, > 1 beyond it
    std::vector<double> mw(nn);
    {
        const double radius_p = radius + width;
        const int origin = -(n / 2);
        for (int a = 0; a < n; ++a)
            for (int b = 0; b < n; ++b) {
                const double r = std::sqrt((double)((a + origin) * (a + origin) + (b + origin) * (b + origin)));
                mw[(size_t)a * n + b] =
                    r < radius ? -1.0 : r <= radius_p ? 0.5 + 0.5 * std::cos(kPi * (radius_p - r) / width) : 2.0;
            }
    }
    size_t bytes = 0;
    auto carve = [&](size_t b) {
        const size_t o = bytes;
        bytes += align256(std::max<size_t>(b, 1));
        return o;
    };
    tb.o_ires = carve(npix * 2);
    tb.o_sig = carve(sigf.size() * 4);
    tb.o_pog = carve((size_t)G * 4);
    tb.o_dst = carve(draw_start.size() * 4);
    tb.o_dcn = carve(draw_count.size() * 4);
    tb.o_dpx = carve(draw_pix.size() * 4);
    tb.o_zst = carve(zero_start.size() * 4);
    tb.o_zcn = carve(zero_count.size() * 4);
    tb.o_zpx = carve(zero_pix.size() * 4);
    tb.o_ss = carve(shell_start.size() * 4);
    tb.o_sp = carve(shell_pix.size() * 4);
    tb.o_mw = carve(nn * 8);
    tb.o_tw = carve((size_t)n * 16);
    char* tab = (char*)ctx->ws[S_PREP_TAB].get(bytes);
    auto up = [&](size_t off, const auto& v) {
        if (!v.empty()) {
            ROME_CUDA(cudaMemcpyAsync(tab + off, v.data(), v.size() * sizeof(v[0]), cudaMemcpyHostToDevice, ctx->stream));
        }
    };
    up(tb.o_ires, ires);
    up(tb.o_sig, sigf);
    up(tb.o_pog, pat_of_group);
    up(tb.o_dst, draw_start);
    up(tb.o_dcn, draw_count);
    up(tb.o_dpx, draw_pix);
    up(tb.o_zst, zero_start);
    up(tb.o_zcn, zero_count);
    up(tb.o_zpx, zero_pix);
    up(tb.o_ss, shell_start);
    up(tb.o_sp, shell_pix);
    up(tb.o_mw, mw);
    // exp(-2 pi i q / n), q < n, for the fused kernels' transforms (host libm)
    std::vector<double2> tw(n);
    for (int q = 0; q < n; ++q)
        tw[q] = make_double2(std::cos(2.0 * kPi * q / n), -std::sin(2.0 * kPi * q / n));
    up(tb.o_tw, tw);
    // the host vectors are pageable: the copies are complete when they return, but wait anyway
    // so that nothing of this call's tables is in flight when the vectors go
    ROME_CUDA(cudaStreamSynchronize(ctx->stream));
}

// one of the fused kernels (masked: the second) for n = 32, 64 or 128, on as
// many CTAs as are resident (each loops over the chunk's images)
template <int E, typename T>
void launch_fused_e(int pc, int fine, const T* raw, const double* pp, int norm_on, double avg, const double2* gtw,
                    double* re, double* im, const double* mw, const double2* noise, const int* ss, const int* sp,
                    double* pow, double* xi2, cudaStream_t st, bool masked) {
    const size_t smem = FusedSmem<E>::TOTAL;
    int per_sm = 0, sms = 0, dev = 0;
    ROME_CUDA(cudaGetDevice(&dev));
    ROME_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (masked) {
        auto k = fused_masked_kernel<E, T>;
        ROME_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        ROME_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kFusedWarps * 32, smem));
        const int grid = std::max(1, std::min(pc, std::max(1, per_sm) * sms));
        k<<<grid, kFusedWarps * 32, smem, st>>>(pc, fine, raw, pp, norm_on, avg, gtw, mw, noise, ss, sp, re, im, pow,
                                                 xi2);
    } else {
        auto k = fused_nomask_kernel<E, T>;
        ROME_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        ROME_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kFusedWarps * 32, smem));
        const int grid = std::max(1, std::min(pc, std::max(1, per_sm) * sms));
        k<<<grid, kFusedWarps * 32, smem, st>>>(pc, fine, raw, pp, norm_on, avg, gtw, re, im);
    }
    ROME_CHECK_LAUNCH();
}

template <typename T>
void launch_fused(int n, int pc, int fine, const T* raw, const double* pp, int norm_on, double avg,
                  const double2* gtw, double* re, double* im, const double* mw, const double2* noise, const int* ss,
                  const int* sp, double* pow, double* xi2, void*, cudaStream_t st, bool masked) {
    if (n == 32)
        launch_fused_e<1, T>(pc, fine, raw, pp, norm_on, avg, gtw, re, im, mw, noise, ss, sp, pow, xi2, st, masked);
    else if (n == 64)
        launch_fused_e<2, T>(pc, fine, raw, pp, norm_on, avg, gtw, re, im, mw, noise, ss, sp, pow, xi2, st, masked);
    else
        launch_fused_e<4, T>(pc, fine, raw, pp, norm_on, avg, gtw, re, im, mw, noise, ss, sp, pow, xi2, st, masked);
}

template <typename T>
void run_prepare(RomeGpuCtx* ctx, const RomePrepIn& in, RomePrepOut& out) {
    const int P = in.nr_images, n = in.ori_size, fine = in.current_size, G = in.nr_groups;
    const int oF = n / 2 + 1, fF = fine / 2 + 1;
    const size_t npix = (size_t)n * oF, Ff = (size_t)fine * fF, nn = (size_t)n * n;
    const bool noise = !in.do_zero_mask;
    cudaStream_t st = ctx->stream;
    Profiler prof(ctx);

    // ---- host side: per-particle parameters, old offsets, tables ----
    std::vector<double> part((size_t)P * PP_COUNT, 0.0);
    for (int p = 0; p < P; ++p) {
        const int g = in.group[p];
        ROME_REQUIRE(g >= 0 && g < G, "particle %d: group %d outside [0, %d)", p, g, G);
        if (in.do_norm_correction) ROME_REQUIRE(in.norm[p] != 0.0, "particle %d: NORM is zero", p);
        if (in.do_ctf_correction) {
            // CTF::initialise's checks (src/ctf.cpp:163-168)
            if (in.ctf_q0[p] < 0. || in.ctf_q0[p] > 1.)
                fail(ROME_ERR_ARG, "particle %d: amplitude contrast Q0 = %g outside [0, 1]", p, in.ctf_q0[p]);
            if (std::fabs(in.ctf_defocus_u[p]) < 1e-6 && std::fabs(in.ctf_defocus_v[p]) < 1e-6 &&
                std::fabs(in.ctf_q0[p]) < 1e-6 && std::fabs(in.ctf_cs[p]) < 1e-6)
                fail(ROME_ERR_ARG, "particle %d: CTF parameters are all zero", p);
        }
        double* r = &part[(size_t)p * PP_COUNT];
        r[PP_NORM] = in.norm[p];
        const double ox = c_round(in.xoff[p]), oy = c_round(in.yoff[p]);
        ROME_REQUIRE(std::fabs(ox) < 1e9 && std::fabs(oy) < 1e9, "particle %d: offset out of range", p);
        out.old_offsetx[p] = ox;
        out.old_offsety[p] = oy;
        r[PP_DX] = ox;
        r[PP_DY] = oy;
        if (in.do_ctf_correction) {
            r[PP_DU] = in.ctf_defocus_u[p];
            r[PP_DV] = in.ctf_defocus_v[p];
            r[PP_DANG] = in.ctf_defocus_angle[p];
            r[PP_KV] = in.ctf_voltage[p];
            r[PP_CS] = in.ctf_cs[p];
            r[PP_Q0] = in.ctf_q0[p];
            r[PP_BFAC] = in.ctf_bfac[p];
        }
        r[PP_GROUP] = g;
    }
    // ---- tables that depend only on the sizes, the mask and sigma2_noise:
    // built on the host and uploaded when those change (once per iteration) ----
    auto* state = prep_state(ctx);
    PrepTables& tb = state->tables;
    const double radius = in.particle_diameter / (2. * in.pixel_size), width = (double)in.width_mask_edge;
    std::vector<double> key = {(double)n, (double)fine, (double)G, noise ? 1.0 : 0.0, radius, width, in.sigma2_fudge};
    if (noise) key.insert(key.end(), in.sigma2_noise, in.sigma2_noise + (size_t)G * oF);
    if (!tb.valid || key != tb.key) {
        tb.valid = false;
        build_tables(ctx, tb, n, fine, G, noise, radius, width, in.sigma2_fudge, in.sigma2_noise);
        tb.key = std::move(key);
        tb.valid = true;
    }
    char* tab = (char*)ctx->ws[S_PREP_TAB].p;
    auto at = [&](size_t off) { return (void*)(tab + off); };
    auto* d_ires = (unsigned short*)at(tb.o_ires);
    auto* d_sig = (float*)at(tb.o_sig);
    auto* d_ss = (int*)at(tb.o_ss);
    auto* d_sp = (int*)at(tb.o_sp);
    auto* d_mw = (double*)at(tb.o_mw);

    // ---- per-call buffers: particle records, CTF constants, per-image sums ----
    size_t call_bytes = 0;
    auto carve = [&](size_t bytes) {
        const size_t o = call_bytes;
        call_bytes += align256(std::max<size_t>(bytes, 1));
        return o;
    };
    const size_t o_part = carve(part.size() * 8), o_ctfk = carve((size_t)P * CK_COUNT * 8), o_bg = carve((size_t)P * 8),
                 o_xi2 = carve((size_t)P * 8), o_pow = carve((size_t)P * oF * 8);
    char* cb = (char*)ctx->ws[S_PREP_PART].get(call_bytes);
    auto* d_part = (double*)(cb + o_part);
    auto* d_ctfk = (double*)(cb + o_ctfk);
    auto* d_bg = (double*)(cb + o_bg);
    auto* d_xi2 = (double*)(cb + o_xi2);
    auto* d_pow = (double*)(cb + o_pow);
    stage_copy(ctx, d_part, part.data(), part.size());

    double *o_re, *o_im, *o_nre, *o_nim, *o_ctf;
    if (out.outputs_on_device) {
        o_re = out.Fimg_real;
        o_im = out.Fimg_imag;
        o_nre = out.Fimg_nomask_real;
        o_nim = out.Fimg_nomask_imag;
        o_ctf = out.Fctf;
    } else {
        double* b = ctx->ws[S_PREP_OUT].as<double>(5 * (size_t)P * Ff);
        o_re = b;
        o_im = b + (size_t)P * Ff;
        o_nre = b + 2 * (size_t)P * Ff;
        o_nim = b + 3 * (size_t)P * Ff;
        o_ctf = b + 4 * (size_t)P * Ff;
    }

    prof.begin(ROME_PHASE_IMAGES);
    // chunks of equal size bounded by the work buffers' footprint
    // power-of-two sizes up to 128 run the fused shared-memory kernels; the
    // others go through cuFFT with FP64 intermediates in HBM
    const bool fused = n == 32 || n == 64 || n == 128;
    const size_t per_img = (fused ? 0 : nn * 8 + npix * 16 + (noise ? nn * 8 : 0)) + (noise ? npix * 16 : 0) +
                           (in.images_on_device ? 0 : nn * sizeof(T)) + 16;
    const size_t budget = ctx->workspace_limit ? ctx->workspace_limit : (size_t)1536 << 20;
    // (cuFFT's 32-bit plans: a chunk holds fewer than 2^31 elements)
    const int cmax = (int)std::max<size_t>(1, std::min<size_t>({(size_t)P, budget / per_img, (size_t)2147483647 / nn}));
    const int nchunk = (P + cmax - 1) / cmax, chunk = (P + nchunk - 1) / nchunk;
    double* d_R = fused ? nullptr : ctx->ws[S_PREP_R].as<double>((size_t)chunk * nn);
    double2* d_C = fused ? nullptr : ctx->ws[S_PREP_C].as<double2>((size_t)chunk * npix);
    double2* d_NC = noise ? ctx->ws[S_PREP_NC].as<double2>((size_t)chunk * npix) : nullptr;
    double* d_NR = noise && !fused ? ctx->ws[S_PREP_NR].as<double>((size_t)chunk * nn) : nullptr;
    const T* d_raw_all = in.images_on_device ? (const T*)in.images : nullptr;
    T* d_raw_chunk = in.images_on_device ? nullptr : ctx->ws[S_PREP_RAW].as<T>((size_t)chunk * nn);
    const int norm_on = in.do_norm_correction ? 1 : 0;
    const uint32_t seed0 = (uint32_t)(in.random_seed + in.first_image);
    const double avg = in.avg_norm_correction;

    // CTF images on the side stream once the particle records are on the device
    cudaStream_t side = state->side;
    ROME_CUDA(cudaEventRecord(state->ev_ready, st));
    ROME_CUDA(cudaStreamWaitEvent(side, state->ev_ready, 0));
    if (in.do_ctf_correction) {
        ctf_constants_kernel<<<(P + 127) / 128, 128, 0, side>>>(P, d_part, d_ctfk);
        ROME_CHECK_LAUNCH();
        prof.launched(ROME_PHASE_IMAGES);
        ctf_kernel<<<grid2(Ff, P), 256, 0, side>>>(P, fine, n, in.pixel_size, d_ctfk, in.ctf_phase_flipped ? 1 : 0,
                                                   in.only_flip_phases ? 1 : 0, in.intact_ctf_first_peak ? 1 : 0,
                                                   o_ctf);
    } else {
        fill_kernel<<<grid_for((size_t)P * Ff), 256, 0, side>>>(o_ctf, (size_t)P * Ff, 1.0);
    }
    ROME_CHECK_LAUNCH();
    prof.launched(ROME_PHASE_IMAGES);
    ROME_CUDA(cudaEventRecord(state->ev_ctf, side));
    ROME_CUDA(cudaEventRecord(state->ev_nc_free, st));

    for (int c0 = 0; c0 < P; c0 += chunk) {
        const int pc = std::min(chunk, P - c0);
        const double* pp = d_part + (size_t)c0 * PP_COUNT;
        // this chunk's noise spectra on the side stream, once the previous chunk's are consumed
        if (noise) {
            ROME_CUDA(cudaStreamWaitEvent(side, state->ev_nc_free, 0));
            noise_spectra_kernel<<<(pc + kNoiseWarps - 1) / kNoiseWarps, kNoiseWarps * 32, 0, side>>>(
                pc, (int)npix, oF, seed0 + (uint32_t)c0, pp, (const int*)at(tb.o_pog), (const int*)at(tb.o_dst),
                (const int*)at(tb.o_dcn), (const int*)at(tb.o_dpx), (const int*)at(tb.o_zst), (const int*)at(tb.o_zcn),
                (const int*)at(tb.o_zpx), d_ires, d_sig, fused ? (long)oF : (long)pc * oF, fused ? (long)npix : (long)oF,
                d_NC);
            ROME_CHECK_LAUNCH();
            ROME_CUDA(cudaEventRecord(state->ev_noise, side));
            prof.launched(ROME_PHASE_IMAGES);
        }
        const T* raw;
        if (in.images_on_device) {
            raw = d_raw_all + (size_t)c0 * nn;
        } else {
            ROME_CUDA(cudaMemcpyAsync(d_raw_chunk, (const T*)in.images + (size_t)c0 * nn, (size_t)pc * nn * sizeof(T),
                                      cudaMemcpyHostToDevice, st));
            raw = d_raw_chunk;
        }
        if (fused) {
            const auto* gtw = (const double2*)at(tb.o_tw);
            launch_fused<T>(n, pc, fine, raw, pp, norm_on, avg, gtw, o_nre + (size_t)c0 * Ff, o_nim + (size_t)c0 * Ff,
                            nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, st, false);
            if (noise) ROME_CUDA(cudaStreamWaitEvent(st, state->ev_noise, 0));
            launch_fused<T>(n, pc, fine, raw, pp, norm_on, avg, gtw, o_re + (size_t)c0 * Ff, o_im + (size_t)c0 * Ff,
                            d_mw, noise ? d_NC : nullptr, d_ss, d_sp, d_pow + (size_t)c0 * oF, d_xi2 + c0, nullptr, st,
                            true);
            if (noise) ROME_CUDA(cudaEventRecord(state->ev_nc_free, st));
            prof.launched(ROME_PHASE_IMAGES, 2);
            continue;
        }
        PrepPlan& plan = get_plan(ctx, &state->plans, n, pc);
        // unmasked image
        translate_center_kernel<T><<<grid2((nn + 3) / 4, pc), 256, 0, st>>>(pc, n, raw, pp, norm_on, avg, d_R);
        ROME_CHECK_LAUNCH();
        ROME_CUFFT(cufftExecD2Z(plan.fwd, d_R, (cufftDoubleComplex*)d_C));
        window_kernel<<<grid2(Ff, pc), 256, 0, st>>>(pc, n, fine, d_C, o_nre + (size_t)c0 * Ff, o_nim + (size_t)c0 * Ff);
        ROME_CHECK_LAUNCH();
        prof.launched(ROME_PHASE_IMAGES, 2);
        // noise image or background average
        if (noise) {
            ROME_CUDA(cudaStreamWaitEvent(st, state->ev_noise, 0));
            ROME_CUFFT(cufftExecZ2Z(plan.col, (cufftDoubleComplex*)d_NC, (cufftDoubleComplex*)d_NC, CUFFT_INVERSE));
            real_edges_kernel<<<grid_for((size_t)n * pc), 256, 0, st>>>((long)n * pc, oF, n, d_NC);
            ROME_CHECK_LAUNCH();
            ROME_CUFFT(cufftExecZ2D(plan.row, (cufftDoubleComplex*)d_NC, d_NR));
            ROME_CUDA(cudaEventRecord(state->ev_nc_free, st));
            prof.launched(ROME_PHASE_IMAGES);
        } else {
            background_kernel<T><<<pc, 256, 0, st>>>(n, raw, pp, norm_on, avg, d_mw, d_bg + c0);
            ROME_CHECK_LAUNCH();
            prof.launched(ROME_PHASE_IMAGES);
        }
        mask_center_kernel<T><<<grid2((nn + 3) / 4, pc), 256, 0, st>>>(pc, n, raw, pp, norm_on, avg, d_mw, d_NR,
                                                                       d_bg + c0, d_R);
        ROME_CHECK_LAUNCH();
        ROME_CUFFT(cufftExecD2Z(plan.fwd, d_R, (cufftDoubleComplex*)d_C));
        window_kernel<<<grid2(Ff, pc), 256, 0, st>>>(pc, n, fine, d_C, o_re + (size_t)c0 * Ff, o_im + (size_t)c0 * Ff);
        ROME_CHECK_LAUNCH();
        prof.launched(ROME_PHASE_IMAGES, 2);
        if (fine < n) {
            power_kernel<<<pc, 128, oF * sizeof(double), st>>>(n, fine, d_C, d_ss, d_sp, d_pow + (size_t)c0 * oF,
                                                                d_xi2 + c0);
            ROME_CHECK_LAUNCH();
            prof.launched(ROME_PHASE_IMAGES);
        }
    }
    if (fine >= n) {
        ROME_CUDA(cudaMemsetAsync(d_xi2, 0, (size_t)P * 8, st));
        ROME_CUDA(cudaMemsetAsync(d_pow, 0, (size_t)P * oF * 8, st));
    }
    ROME_CUDA(cudaStreamWaitEvent(st, state->ev_ctf, 0));
    prof.end(ROME_PHASE_IMAGES);
    // algorithmic traffic: images in, the five output arrays and the power spectra out
    prof.add_bytes(ROME_PHASE_IMAGES, (double)P * ((double)nn * sizeof(T) + 5.0 * Ff * 8 + oF * 8.0));

    ROME_CUDA(cudaMemcpyAsync(out.highres_Xi2, d_xi2, (size_t)P * 8, cudaMemcpyDeviceToHost, st));
    if (out.power_imgs)
        ROME_CUDA(cudaMemcpyAsync(out.power_imgs, d_pow, (size_t)P * oF * 8, cudaMemcpyDeviceToHost, st));
    if (!out.outputs_on_device) {
        double* dsts[5] = {out.Fimg_real, out.Fimg_imag, out.Fimg_nomask_real, out.Fimg_nomask_imag, out.Fctf};
        double* srcs[5] = {o_re, o_im, o_nre, o_nim, o_ctf};
        for (int k = 0; k < 5; ++k)
            ROME_CUDA(cudaMemcpyAsync(dsts[k], srcs[k], (size_t)P * Ff * 8, cudaMemcpyDeviceToHost, st));
    }
    ROME_CUDA(cudaStreamSynchronize(st));
    prof.collect();
}

}  // namespace

void prep_release(RomeGpuCtx* ctx) {
    if (!ctx || !ctx->prep_plans) return;
    auto* ps = (PrepState*)ctx->prep_plans;
    for (auto& kv : ps->plans.plans) destroy_plan(kv.second);
    if (ps->side) {
        cudaStreamSynchronize(ps->side);
        cudaStreamDestroy(ps->side);
        for (cudaEvent_t e : {ps->ev_ready, ps->ev_noise, ps->ev_nc_free, ps->ev_ctf})
            if (e) cudaEventDestroy(e);
    }
    delete ps;
    ctx->prep_plans = nullptr;
}

}  // namespace rome

using namespace rome;

extern "C" int rome_gpu_prepare_particles(RomeGpuCtx* ctx, const RomePrepIn* in, RomePrepOut* out) {
    if (!ctx) return ROME_ERR_ARG;
    return guarded(ctx, [&] {
        ROME_REQUIRE(in && out, "null argument");
        const RomePrepIn& a = *in;
        ROME_REQUIRE(a.nr_images >= 0, "nr_images %d", a.nr_images);
        if (a.nr_images == 0) return;
        ROME_REQUIRE(a.ori_size >= 2 && a.ori_size % 2 == 0 && a.ori_size <= 4096, "ori_size %d: even sizes 2..4096",
                     a.ori_size);
        ROME_REQUIRE(a.current_size >= 1 && a.current_size <= a.ori_size, "current_size %d outside [1, ori_size]",
                     a.current_size);
        ROME_REQUIRE(a.nr_groups >= 1, "nr_groups %d", a.nr_groups);
        ROME_REQUIRE(a.image_type == 0 || a.image_type == 1, "image_type %d", a.image_type);
        ROME_REQUIRE(a.images && a.norm && a.xoff && a.yoff && a.group && a.sigma2_noise, "missing input array");
        ROME_REQUIRE(!a.do_ctf_correction || (a.ctf_defocus_u && a.ctf_defocus_v && a.ctf_defocus_angle &&
                                              a.ctf_voltage && a.ctf_cs && a.ctf_q0 && a.ctf_bfac),
                     "missing CTF parameters");
        ROME_REQUIRE(out->Fimg_real && out->Fimg_imag && out->Fimg_nomask_real && out->Fimg_nomask_imag && out->Fctf &&
                         out->highres_Xi2 && out->old_offsetx && out->old_offsety,
                     "missing output array");
        ROME_REQUIRE(a.pixel_size > 0 && a.width_mask_edge >= 0, "pixel_size %g, width_mask_edge %d", a.pixel_size,
                     a.width_mask_edge);
        if (!a.do_zero_mask) {
            // Random_generator::init(seed) seeds from the clock for seed < 0:
            // not reproducible, so not supported
            const long s0 = (long)a.random_seed + a.first_image, s1 = s0 + a.nr_images - 1;
            ROME_REQUIRE(s0 >= 0 && s1 <= 2147483647L, "noise seeds %ld..%ld outside [0, 2^31)", s0, s1);
        }
        ROME_CUDA(cudaSetDevice(ctx->device));
        arena_reset(ctx);
        if (a.image_type == 0)
            run_prepare<double>(ctx, a, *out);
        else
            run_prepare<float>(ctx, a, *out);
    });
}
