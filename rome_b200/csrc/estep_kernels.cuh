// Device kernels of the MAP E-step (2D).  Each kernel names the reference
// loop it replaces.  FP64 arithmetic that must reproduce the reference's
// operation order uses explicit round-to-nearest intrinsics (no fused
// multiply-add); everything else is free to fuse.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cfloat>
#include <climits>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "epilogues.cuh"

namespace rome {
// internal linkage: every translation unit that launches these kernels gets its own copy
namespace {

template <typename TVal>
__device__ TVal block_reduce_sum(TVal v, TVal* sh);

// ---------------------------------------------------------------------------
// shiftImageInFourierTransform for one coefficient (src/image.h:1530-1547):
// tabulated cos/sin at index (int)(|dotp| / sampling) % 5000 and the
// three-multiplication complex product.
__device__ __forceinline__ double2 table_shift(double x, double y, double2 sh, double2 v, const double2* __restrict__ tab,
                                               double sampling) {
    if (fabs(sh.x) < 1e-6 && fabs(sh.y) < 1e-6) return v;  // ROME_EQUAL_ACCURACY shortcut
    const double two_pi = 2 * kPi;
    double dotp = dmul(two_pi, dadd(dmul(x, sh.x), dmul(y, sh.y)));
    int idx = ((int)__ddiv_rn(fabs(dotp), sampling)) % 5000;
    double2 cs = __ldg(tab + idx);
    double a = cs.x;
    double b = dotp < 0 ? -cs.y : cs.y;
    double ac = dmul(a, v.x), bd = dmul(b, v.y);
    double ab_cd = dmul(dadd(a, b), dadd(v.x, v.y));
    return make_double2(dsub(ac, bd), dsub(dsub(ab_cd, ac), bd));
}

// The table index depends only on the translation and the pixel, so a pass
// tabulates (a, b) = (cos, +-sin) once per (translation, pixel) and every
// particle reuses it: ph[t][n].  apply_phase is the same three-multiplication
// product as table_shift; translations below ROME_EQUAL_ACCURACY leave the
// coefficient untouched exactly as the reference's early return does.
__device__ __forceinline__ double2 apply_phase(double2 sh, double2 ab, double2 v) {
    if (fabs(sh.x) < 1e-6 && fabs(sh.y) < 1e-6) return v;
    double ac = dmul(ab.x, v.x), bd = dmul(ab.y, v.y);
    double ab_cd = dmul(dadd(ab.x, ab.y), dadd(v.x, v.y));
    return make_double2(dsub(ac, bd), dsub(dsub(ab_cd, ac), bd));
}

__global__ void phase_table_kernel(int T, int F, int csF, int cs, const double2* __restrict__ shifts,
                                   const double2* __restrict__ tab, double sampling, double2* __restrict__ ph) {
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long)T * F) return;
    int t = (int)(q / F), n = (int)(q - (long)t * F);
    int row = n / csF;
    double x = (double)(n - row * csF), y = (double)(row < csF ? row : row - cs);
    const double2 sh = shifts[t];
    const double two_pi = 2 * kPi;
    double dotp = dmul(two_pi, dadd(dmul(x, sh.x), dmul(y, sh.y)));
    int idx = ((int)__ddiv_rn(fabs(dotp), sampling)) % 5000;
    double2 cs2 = tab[idx];
    ph[q] = make_double2(cs2.x, dotp < 0 ? -cs2.y : cs2.y);
}

// Table index of every (translation, active pixel): the same index the
// reference's shiftImageInFourierTransform picks, as 16 bits, with the sign
// of dotp in bit 15 (src/image.h:1530-1537).  Identity translations (below
// ROME_EQUAL_ACCURACY) are marked with 0xFFFF.
__global__ void phase_index_kernel(int T, int Kact, int csF, int cs, const int* __restrict__ act,
                                   const double2* __restrict__ shifts, double sampling,
                                   unsigned short* __restrict__ pidx) {
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long)T * Kact) return;
    int t = (int)(q / Kact), a = (int)(q - (long)t * Kact);
    const double2 sh = shifts[t];
    if (fabs(sh.x) < 1e-6 && fabs(sh.y) < 1e-6) {
        pidx[q] = 0xFFFF;
        return;
    }
    int n = act[a];
    int row = n / csF;
    double x = (double)(n - row * csF), y = (double)(row < csF ? row : row - cs);
    const double two_pi = 2 * kPi;
    double dotp = dmul(two_pi, dadd(dmul(x, sh.x), dmul(y, sh.y)));
    int idx = ((int)__ddiv_rn(fabs(dotp), sampling)) % 5000;
    pidx[q] = (unsigned short)(idx | (dotp < 0 ? 0x8000 : 0));
}

// Cross-term A operand of one particle for every translation: a = Minvsigma2
// * ctf * X_t on the active pixels, with the table phase applied in FP32
// (the operand is stored in FP32 or BF16, so FP32 products keep it exact to
// its own rounding), and S = sum_n Minvsigma2 |X|^2 over all pixels in FP64
// (a phase shift leaves |X|^2 unchanged up to rounding, so S is the same
// for every translation).  One CTA per particle; the 5000-entry table is
// staged in shared memory as float2.  Minv null: no Minvsigma2 weighting
// (the cross-correlation mode's signal product).  pscale (per particle,
// may be null): the group's intensity scale, which multiplies the
// reference (applyCtfToClass, src/map3d_optimizer.cpp:1054-1066) and so
// the cross term once.
template <int NT>
__global__ void __launch_bounds__(NT)
    shift_operand2_kernel(int P, int T, int F, int Kact, int Kp, const double2* __restrict__ Fimg,
                          const double* __restrict__ lctf, const double* __restrict__ Minv, int apply_ctf,
                          const int* __restrict__ act, const unsigned short* __restrict__ pidx,
                          const double2* __restrict__ tab, void* __restrict__ Aop, float* __restrict__ S,
                          int precision, const double* __restrict__ pscale = nullptr) {
    __shared__ float2 stab[5000];
    __shared__ double red[32];
    const int i = blockIdx.x;
    for (int q = threadIdx.x; q < 5000; q += NT) stab[q] = make_float2((float)tab[q].x, (float)tab[q].y);
    const double2* X = Fimg + (long)i * F;
    const double* M = Minv ? Minv + (long)i * F : nullptr;
    const double* C = lctf + (long)i * F;
    const double sc = pscale ? pscale[i] : 1.0;
    double s = 0.0;
    for (int n = threadIdx.x; n < F; n += NT) {
        double2 v = X[n];
        s += (M ? M[n] : 1.0) * (v.x * v.x + v.y * v.y);
    }
    s = block_reduce_sum(s, red);  // includes a __syncthreads after the table fill
    const long M2 = (long)P * T;
    __nv_bfloat16* Ah = (__nv_bfloat16*)Aop;
    __nv_bfloat16* Al = Ah + M2 * Kp;
    for (int a = threadIdx.x; a < Kp / 2; a += NT) {
        float2 xw = make_float2(0.f, 0.f);
        if (a < Kact) {
            int n = act[a];
            const double m = M ? M[n] : 1.0;
            double w = (apply_ctf ? m * C[n] : m) * sc;
            xw = make_float2((float)(w * X[n].x), (float)(w * X[n].y));
        }
        for (int t = 0; t < T; t++) {
            float fr = 0.f, fi = 0.f;
            if (a < Kact) {
                unsigned short pi = pidx[(long)t * Kact + a];
                if (pi == 0xFFFF) {
                    fr = xw.x;
                    fi = xw.y;
                } else {
                    float2 cs = stab[pi & 0x7FFF];
                    float sn = (pi & 0x8000) ? -cs.y : cs.y;
                    fr = cs.x * xw.x - sn * xw.y;
                    fi = cs.x * xw.y + sn * xw.x;
                }
            }
            long o = ((long)i * T + t) * Kp + 2 * a;
            if (precision == ROME_PREC_FP32) {
                *(float2*)((float*)Aop + o) = make_float2(fr, fi);
            } else {
                __nv_bfloat162 h2 = __floats2bfloat162_rn(fr, fi);
                *(__nv_bfloat162*)(Ah + o) = h2;
                if (precision == ROME_PREC_BF16X3) {
                    float2 hf = __bfloat1622float2(h2);
                    *(__nv_bfloat162*)(Al + o) = __floats2bfloat162_rn(fr - hf.x, fi - hf.y);
                }
            }
        }
    }
    if (threadIdx.x == 0)
        for (int t = 0; t < T; t++) S[(long)i * T + t] = (float)s;
}

// coordinates of half-plane pixel n of a size x (size/2+1) FFTW image
__device__ __forceinline__ void pixel_xy(int n, int rowlen, int size, double& x, double& y) {
    int row = n / rowlen;
    x = (double)(n - row * rowlen);
    y = (double)(row < rowlen ? row : row - size);
}

// convertSquaredDifferencesToWeights (src/map2d_optimizer.cpp:1113-1131):
// pdf_orientation * pdf_offset * exp(-(diff2 - min_diff2)), zero beyond 700
// and for hypotheses that were not computed (stored as +inf).
__device__ __forceinline__ double hyp_weight(float d, double mn, double pdir, double po) {
    if (!(d < INFINITY)) return 0.0;
    double w = pdir * po;
    double diff = (double)d - mn;
    if (diff > 700.) return 0.0;
    return w * exp(-diff);
}

// ---------------------------------------------------------------------------
// ParticleModel::preShiftedImagesCtfsAndInvSigma2s, per-particle part
// (src/exp_model.cpp:1015-1103): window the fine-size image and CTF to the
// pass size (windowFourierTransform / windowTransform, src/image.h:419-568)
// and build Minvsigma2 = 1/(sigma2_fudge * sigma2_noise[ires]), 0 at ires <= 0.
// rows: optional input row of each particle (a subset of a staged pool).
// The restricted tensor-core search's per-particle operands come out of the
// same pass when xw is given (the restricted_prep_kernel arithmetic, in its
// order): xw[i][a] = Minvsigma2 * ctf * X and w2[i][a] = Minvsigma2 * ctf^2 at
// the active pixels a = actidx[n] (zero up to Kh), S[i] = sum_n Minvsigma2 |X|^2.
struct RestrictedOut {
    float2* xw = nullptr;
    float* w2 = nullptr;
    float* S = nullptr;
    const int* actidx = nullptr;
    int Kact = 0, Kh = 0, apply_ctf = 0;
};

__global__ void prep_particles_kernel(int P, int cur, int cs, const double* __restrict__ Fr,
                                      const double* __restrict__ Fi, const double* __restrict__ ctf_fine,
                                      const int* __restrict__ Mresol, const double* __restrict__ sigma2,
                                      const int* __restrict__ group, int oriF, double fudge, double2* __restrict__ Fimg,
                                      double* __restrict__ lctf, double* __restrict__ Minv,
                                      const int* __restrict__ rows = nullptr, RestrictedOut ro = RestrictedOut{}) {
    __shared__ double red[32];
    const int i = blockIdx.x;
    const long ri = rows ? rows[i] : i;
    const int curF = cur / 2 + 1, curF2 = cur * curF, csF = cs / 2 + 1, F = cs * csF;
    const double* s2 = sigma2 + (long)group[i] * oriF;
    double s = 0.0;
    for (int n = threadIdx.x; n < F; n += blockDim.x) {
        int oi = n / csF, j = n - oi * csF;
        int ip = oi < csF ? oi : oi - cs;
        int in_i = ip < 0 ? ip + cur : ip;
        long src = ri * curF2 + (long)in_i * curF + j;
        long dst = (long)i * F + n;
        const double2 X = make_double2(Fr[src], Fi[src]);
        const double c = ctf_fine[src];
        Fimg[dst] = X;
        lctf[dst] = c;
        int ires = Mresol[n];
        const double m = ires > 0 ? 1. / (fudge * s2[ires]) : 0.;
        Minv[dst] = m;
        if (ro.xw) {
            s += m * (X.x * X.x + X.y * X.y);
            const int a = ro.actidx[n];
            if (a >= 0) {
                const double cc = ro.apply_ctf ? c : 1.0;
                const double wd = ro.apply_ctf ? m * c : m;
                ro.xw[(long)i * ro.Kh + a] = make_float2((float)(wd * X.x), (float)(wd * X.y));
                ro.w2[(long)i * ro.Kh + a] = (float)(m * cc * cc);
            }
        }
    }
    if (!ro.xw) return;
    for (int a = ro.Kact + threadIdx.x; a < ro.Kh; a += blockDim.x) {
        ro.xw[(long)i * ro.Kh + a] = make_float2(0.f, 0.f);
        ro.w2[(long)i * ro.Kh + a] = 0.f;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) t += red[q];
        ro.S[i] = (float)t;
    }
}

// MLModel::calculatePdfOffset (src/ml_model.h:231-242) for every particle,
// class and coarse translation: the offset is the coarse translation plus
// the particle's rounded old offset (src/map2d_optimizer.cpp:1116-1121).
__global__ void pdf_offset_kernel(int P, int K, int ntr, const double2* __restrict__ oldoff,
                                  const double2* __restrict__ trans, const double* __restrict__ priorx,
                                  const double* __restrict__ priory, double sigma2_offset,
                                  double* __restrict__ poff) {
    const int i = blockIdx.x;
    const double2 oo = oldoff[i];
    for (int q = threadIdx.x; q < K * ntr; q += blockDim.x) {
        int k = q / ntr, t = q - k * ntr;
        double ox = trans[t].x + oo.x, oy = trans[t].y + oo.y;
        double dx = ox - priorx[k], dy = oy - priory[k];
        double tdiff2 = dadd(dmul(dx, dx), dmul(dy, dy));
        double po;
        if (sigma2_offset < 0.0001) po = (tdiff2 > 0.) ? 0. : 1.;
        else po = exp(tdiff2 / (-2. * sigma2_offset)) / (2. * kPi * sigma2_offset);
        poff[(long)i * K * ntr + q] = po;
    }
}

// Rot_significant (getReferenceAllOrientations, src/map2d_optimizer.cpp:856-880
// and isSignificantAnyParticleAnyTranslation, :2048-2061) per (class, psi).
__global__ void rot_sig_kernel(int nkp, int P, int ntr, long ncoarse, const char* __restrict__ mcoarse,
                               char* __restrict__ rotsig) {
    int kp = blockIdx.x * blockDim.x + threadIdx.x;
    if (kp >= nkp) return;
    char any = 1;
    if (mcoarse) {
        any = 0;
        for (int i = 0; i < P && !any; i++)
            for (int t = 0; t < ntr; t++)
                if (mcoarse[(long)i * ncoarse + (long)kp * ntr + t]) {
                    any = 1;
                    break;
                }
    }
    rotsig[kp] = any;
}

__global__ void jvalid_kernel(int J, int nrot, int nor, const int* __restrict__ class_ok,
                              const char* __restrict__ rotsig, int* __restrict__ jvalid) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= J) return;
    jvalid[j] = class_ok[j / nrot] && rotsig[j / nor];
}

// ---------------------------------------------------------------------------
// MyProjector::rotate2D (src/reconstruct.cpp:823-958) for every
// orientation j = (class, psi, over_rot), evaluated only on the active
// pixels (r^2 <= my_r_max^2; every other coefficient of the projection is
// zero).  Writes the FP64 projection, the GEMM B operand and |P|^2.
__global__ void project2d_kernel(int J, int Kact, int Kp, int Kq, int cs, int csF, int my_r_max, int pad, int padF,
                                 int nrot, const double2* __restrict__ proj_data, long vox,
                                 const double4* __restrict__ rot, const int* __restrict__ act,
                                 const int* __restrict__ jvalid, double2* __restrict__ P_out, float* __restrict__ Q,
                                 void* __restrict__ Bop, int precision) {
    const int j = blockIdx.x;
    const bool ok = jvalid[j] != 0;
    const double4 A = rot[j];
    const double2* data = proj_data + (long)(j / nrot) * vox;
    const int shift = -(int)((float)pad / 2.0f);
    for (int a = threadIdx.x; a < Kp / 2; a += blockDim.x) {
        double2 v = make_double2(0.0, 0.0);
        if (ok && a < Kact) {
            int n = act[a];
            int row = n / csF;
            int x = n - row * csF;
            int y = row <= my_r_max ? row : row - cs;
            double xp = dadd(dmul(A.x, (double)x), dmul(A.y, (double)y));
            double yp = dadd(dmul(A.z, (double)x), dmul(A.w, (double)y));
            bool neg = xp < 0;
            if (neg) {
                xp = -xp;
                yp = -yp;
            }
            int x0 = (int)floor(xp);
            double fx = dsub(xp, (double)x0);
            int y0 = (int)floor(yp);
            double fy = dsub(yp, (double)y0);
            y0 -= shift;
            int y1 = y0 + 1;
            double2 d00 = data[(long)y0 * padF + x0], d01 = data[(long)y0 * padF + x0 + 1];
            double2 d10 = data[(long)y1 * padF + x0], d11 = data[(long)y1 * padF + x0 + 1];
            double dx0r = dadd(d00.x, dmul(dsub(d01.x, d00.x), fx));
            double dx0i = dadd(d00.y, dmul(dsub(d01.y, d00.y), fx));
            double dx1r = dadd(d10.x, dmul(dsub(d11.x, d10.x), fx));
            double dx1i = dadd(d10.y, dmul(dsub(d11.y, d10.y), fx));
            v.x = dadd(dx0r, dmul(dsub(dx1r, dx0r), fy));
            v.y = dadd(dx0i, dmul(dsub(dx1i, dx0i), fy));
            if (neg) v.y = -1.0 * v.y;
        }
        if (a < Kact) P_out[(long)j * Kact + a] = v;
        if (a < Kq) Q[(long)j * Kq + a] = (float)(v.x * v.x + v.y * v.y);
        long o = (long)j * Kp + 2 * a;
        if (precision == ROME_PREC_FP32) {
            float2* B = (float2*)((float*)Bop + o);
            *B = make_float2((float)v.x, (float)v.y);
        } else {
            __nv_bfloat16* Bh = (__nv_bfloat16*)Bop;
            __nv_bfloat16* Bl = Bh + (long)J * Kp;
            float fr = (float)v.x, fi = (float)v.y;
            __nv_bfloat16 hr = __float2bfloat16_rn(fr), hi = __float2bfloat16_rn(fi);
            Bh[o] = hr;
            Bh[o + 1] = hi;
            if (precision == ROME_PREC_BF16X3) {
                Bl[o] = __float2bfloat16_rn(fr - __bfloat162float(hr));
                Bl[o + 1] = __float2bfloat16_rn(fi - __bfloat162float(hi));
            }
        }
    }
    for (int a = Kp / 2 + threadIdx.x; a < Kq; a += blockDim.x) Q[(long)j * Kq + a] = 0.f;
}

// ---------------------------------------------------------------------------
// Shifted images (exp_Fimgs_shifted, src/exp_model.cpp:1057-1076) turned into
// the cross-term A operand a = Minvsigma2 * ctf * X_t on the active pixels,
// and S_it = sum_n Minvsigma2 |X_t|^2 over all pixels.
__global__ void shift_operand_kernel(int P, int T, int F, int csF, int cs, int Kact, int Kp,
                                     const double2* __restrict__ Fimg, const double* __restrict__ lctf,
                                     const double* __restrict__ Minv, int apply_ctf, const int* __restrict__ act,
                                     const double2* __restrict__ shifts, const double2* __restrict__ ph,
                                     void* __restrict__ Aop, float* __restrict__ S, int precision) {
    const int t = blockIdx.x, i = blockIdx.y;
    const long r = (long)i * T + t;
    const double2 sh = shifts[t];
    const double2* X = Fimg + (long)i * F;
    const double* M = Minv + (long)i * F;
    const double* C = lctf + (long)i * F;
    const double2* pht = ph + (long)t * F;
    double s = 0.0;
    // S over every pixel of the pass image
    for (int n = threadIdx.x; n < F; n += blockDim.x) {
        double2 v = apply_phase(sh, pht[n], X[n]);
        s += M[n] * (v.x * v.x + v.y * v.y);
    }
    // A operand on the active pixels (zero padded to Kp)
    const long M2 = (long)P * T;
    for (int a = threadIdx.x; a < Kp / 2; a += blockDim.x) {
        float fr = 0.f, fi = 0.f;
        if (a < Kact) {
            int n = act[a];
            double2 v = apply_phase(sh, pht[n], X[n]);
            double w = apply_ctf ? M[n] * C[n] : M[n];
            fr = (float)(w * v.x);
            fi = (float)(w * v.y);
        }
        long o = r * Kp + 2 * a;
        if (precision == ROME_PREC_FP32) {
            *(float2*)((float*)Aop + o) = make_float2(fr, fi);
        } else {
            __nv_bfloat16* Ah = (__nv_bfloat16*)Aop;
            __nv_bfloat16* Al = Ah + M2 * Kp;
            __nv_bfloat16 hr = __float2bfloat16_rn(fr), hi = __float2bfloat16_rn(fi);
            Ah[o] = hr;
            Ah[o + 1] = hi;
            if (precision == ROME_PREC_BF16X3) {
                Al[o] = __float2bfloat16_rn(fr - __bfloat162float(hr));
                Al[o + 1] = __float2bfloat16_rn(fi - __bfloat162float(hi));
            }
        }
    }
    // block reduction of S
    __shared__ double red[32];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
        if (threadIdx.x == 0) S[r] = (float)s;
    }
}

// norm-term operand Minvsigma2 * ctf^2 on the active pixels (Minv null:
// ctf^2 alone, the reference power of the cross-correlation mode); times
// the square of the particle's intensity scale when pscale is given
__global__ void w2_kernel(int P, int Kact, int Kq, const int* __restrict__ act, const double* __restrict__ lctf,
                          const double* __restrict__ Minv, int F, int apply_ctf, float* __restrict__ W2,
                          const double* __restrict__ pscale = nullptr) {
    const int i = blockIdx.x;
    const double sc = pscale ? pscale[i] : 1.0;
    for (int a = threadIdx.x; a < Kq; a += blockDim.x) {
        float v = 0.f;
        if (a < Kact) {
            long n = (long)i * F + act[a];
            double c = (apply_ctf ? lctf[n] : 1.0) * sc;
            v = (float)((Minv ? Minv[n] : 1.0) * c * c);
        }
        W2[(long)i * Kq + a] = v;
    }
}

// Layout of the hypothesis index e of one particle (exp_Mweight order).
// Hypothesis layout of one particle's row.  Dense rows (every pass of 2D,
// the coarse pass of 3D) hold e = j * T + t with j = (k, psi, over_rot) and
// t = (trans, over_trans); k indexes pdf_direction and k / ndir the class of
// the offset prior (3D folds the direction into k: k = class * ndir + dir).
// Ragged rows (the 3D fine pass, the restricted 2D search) hold epr
// hypotheses per entry r; ent[i * ent_stride + r] = (k, coarse translation),
// or (k, -1) when the entry's hypotheses are its translations; x < 0 marks
// padding, and the row order is already the reference's loop order.
struct PostLayout {
    int T, notr, nor, npsi, ntr, K;
    int ndir = 1;
    const int2* ent = nullptr;
    int ent_stride = 0;
    // ragged rows without padding: particle i's entries are roff[i] .. roff[i + 1] - 1 (each epr
    // hypotheses), so its row starts at roff[i] * epr and ent[roff[i] + r] describes entry r
    const int* roff = nullptr;
    int epr = 0;
    int list_zeros = 0;  // 3D: computed zero weights take part in the sorted walk
};

__device__ __forceinline__ void decode_e(long e, const PostLayout& L, int& k, int& itr, long& loop_order) {
    int j = (int)(e / L.T), t = (int)(e - (long)j * L.T);
    int nrot = L.npsi * L.nor;
    k = j / nrot;
    int rr = j - k * nrot;
    int ipsi = rr / L.nor, ior = rr - ipsi * L.nor;
    itr = t / L.notr;
    int iotr = t - itr * L.notr;
    // order of the reference's weight loop: class, psi, trans, over_rot, over_trans
    loop_order = ((((long)k * L.npsi + ipsi) * L.ntr + itr) * L.nor + ior) * L.notr + iotr;
}

// prior pdf_orientation and pdf_offset of hypothesis e in particle i's row
// (po points at the particle's [class][ntr] offset priors); false for padding
__device__ __forceinline__ bool hyp_prior(long e, int i, const PostLayout& L, const double* __restrict__ pdir,
                                          const double* __restrict__ po, double& pd, double& pof, long& lo) {
    int k, itr;
    if (L.ent) {
        const int2 en = L.ent[(L.roff ? (long)L.roff[i] : (long)i * L.ent_stride) + e / L.epr];
        if (en.x < 0) return false;
        k = en.x;
        // y < 0: the entry's hypotheses are its translations (restricted 2D search)
        itr = en.y >= 0 ? en.y : (int)(e % L.epr) / L.notr;
        lo = e;
    } else {
        decode_e(e, L, k, itr, lo);
    }
    pd = pdir[k];
    pof = po[(k / L.ndir) * L.ntr + itr];
    return true;
}

template <typename TVal>
__device__ TVal block_reduce_max(TVal v, TVal* sh) {
    for (int off = 16; off > 0; off >>= 1) v = max(v, __shfl_down_sync(0xffffffffu, v, off));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    TVal r = v;
    if (threadIdx.x < 32) {
        r = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : sh[0];
        for (int off = 16; off > 0; off >>= 1) r = max(r, __shfl_down_sync(0xffffffffu, r, off));
        if (threadIdx.x == 0) sh[0] = r;
    }
    __syncthreads();
    r = sh[0];
    __syncthreads();
    return r;
}

template <typename TVal>
__device__ TVal block_reduce_sum(TVal v, TVal* sh) {
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    TVal r = 0;
    if (threadIdx.x < 32) {
        r = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : (TVal)0;
        for (int off = 16; off > 0; off >>= 1) r += __shfl_down_sync(0xffffffffu, r, off);
        if (threadIdx.x == 0) sh[0] = r;
    }
    __syncthreads();
    r = sh[0];
    __syncthreads();
    return r;
}

// backProjection preparation (src/map2d_optimizer.cpp:1670-1737): origin of
// Minvsigma2 restored, Minvsigma2 -> 1 without MAP, CTF -> 1 without CTF
// correction, then CTF times the group's intensity scale with scale
// correction (pscale, src/map3d_optimizer.cpp:2274-2282); nomask image times
// ctf*Minvsigma2 and Mctf2 = ctf^2*Minvsigma2.
__global__ void bp_prep_kernel(int P, int F, const double* __restrict__ Fnr, const double* __restrict__ Fni,
                               const double* __restrict__ lctf, double* __restrict__ Minv,
                               const double* __restrict__ sigma2, const int* __restrict__ group, int oriF, double fudge,
                               int do_map, int do_ctf, double2* __restrict__ Fnm, double* __restrict__ Mctf2,
                               const int* __restrict__ rows = nullptr, const double* __restrict__ pscale = nullptr) {
    const int i = blockIdx.x;
    const long ri = rows ? rows[i] : i;
    for (int n = threadIdx.x; n < F; n += blockDim.x) {
        long q = (long)i * F + n, qi = ri * F + n;
        double m = Minv[q];
        if (n == 0) m = 1. / (fudge * sigma2[(long)group[i] * oriF + 0]);
        if (!do_map) m = 1.0;
        double c = do_ctf ? lctf[q] : 1.0;
        if (pscale) c = dmul(c, pscale[i]);
        double mc = dmul(c, m);
        Fnm[q] = make_double2(dmul(Fnr[qi], mc), dmul(Fni[qi], mc));
        Mctf2[q] = dmul(c, mc);
    }
}

// ---------------------------------------------------------------------------
// Significant hypotheses as a compact list.  updateOtherParams and
// backProjection only touch hypotheses with weight >= significant_weight
// (src/map2d_optimizer.cpp:1469, :1594, :1800); each particle writes its own
// contiguous segment of (hypothesis, weight / sum_weight) records.
struct SigEntry {
    int i;     // particle
    int e;     // hypothesis index in the exp_Mweight layout
    double w;  // weight / exp_sum_weight
};

// counting sort of the list by orientation j = e / T
__global__ void count_by_j_kernel(int n, int T, const SigEntry* __restrict__ list, int* __restrict__ cnt) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) atomicAdd(&cnt[list[q].e / T], 1);
}

// exclusive scan of cnt[0..n) into off[0..n], one CTA
__global__ void __launch_bounds__(1024) exclusive_scan_kernel(int n, const int* __restrict__ cnt, int* __restrict__ off) {
    __shared__ int sh[1024];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int b = 0; b < n; b += 1024) {
        int q = b + threadIdx.x;
        int v = q < n ? cnt[q] : 0;
        sh[threadIdx.x] = v;
        __syncthreads();
        for (int s = 1; s < 1024; s <<= 1) {
            int t = threadIdx.x >= s ? sh[threadIdx.x - s] : 0;
            __syncthreads();
            sh[threadIdx.x] += t;
            __syncthreads();
        }
        if (q < n) off[q] = carry + sh[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry += sh[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) off[n] = carry;
}

__global__ void scatter_by_j_kernel(int n, int T, const SigEntry* __restrict__ list, const int* __restrict__ off,
                                    int* __restrict__ fill, SigEntry* __restrict__ sorted) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    SigEntry s = list[q];
    int j = s.e / T;
    sorted[off[j] + atomicAdd(&fill[j], 1)] = s;
}

// updateOtherParams over the particle's list segment (see wsum_kernel)
template <int NT, int PIX>
__global__ void __launch_bounds__(NT, 4)
    wsum_list_kernel(int T, int nrot, int K, int F, int csF, int cs, int oriF, const SigEntry* __restrict__ list,
                     const int* __restrict__ seg, const double2* __restrict__ Fimg, const double* __restrict__ lctf,
                     int apply_ctf, const double2* __restrict__ proj, const int* __restrict__ actidx, int Kact,
                     const double2* __restrict__ shifts, const double2* __restrict__ ph,
                     const int* __restrict__ Mresol, const int* __restrict__ group, const double2* __restrict__ oldoff,
                     const double2* __restrict__ trans, const double* __restrict__ priorx,
                     const double* __restrict__ priory, double* __restrict__ wsn, double* __restrict__ normcorr,
                     double* __restrict__ wk) {
    const int i = blockIdx.y;
    const int n0 = blockIdx.x * NT * PIX;
    const int s0 = seg[2 * i], ns = seg[2 * i + 1];
    __shared__ double spec[1024];
    __shared__ double red[32];
    for (int q = threadIdx.x; q < oriF && q < 1024; q += NT) spec[q] = 0.0;
    __syncthreads();
    double acc[PIX];
    int ires_p[PIX];
    double xs[PIX], ys[PIX], cp[PIX];
    double2 Xp[PIX];
    int ap[PIX];
#pragma unroll
    for (int p = 0; p < PIX; p++) {
        acc[p] = 0.0;
        int n = n0 + threadIdx.x + p * NT;
        ires_p[p] = n < F ? Mresol[n] : -1;
        if (ires_p[p] > -1) {
            pixel_xy(n, csF, cs, xs[p], ys[p]);
            Xp[p] = Fimg[(long)i * F + n];
            cp[p] = lctf[(long)i * F + n];
            ap[p] = actidx[n];
        }
    }
    double sumwd = 0.0;
    const int g = group[i];
    const double2 oo = oldoff[i];
    for (int q = 0; q < ns; q++) {
        const SigEntry s = list[s0 + q];
        const int j = s.e / T, t = s.e - j * T;
        const double w = s.w;
        const double2 sh = shifts[t];
        const double2* Pj = proj + (long)j * Kact;
#pragma unroll
        for (int p = 0; p < PIX; p++) {
            if (ires_p[p] > -1) {
                double2 v = apply_phase(sh, ph[(long)t * F + n0 + threadIdx.x + p * NT], Xp[p]);
                double2 pv = ap[p] >= 0 ? Pj[ap[p]] : make_double2(0.0, 0.0);
                double pr = apply_ctf ? dmul(pv.x, cp[p]) : pv.x;
                double pim = apply_ctf ? dmul(pv.y, cp[p]) : pv.y;
                double dr = dsub(pr, v.x), di = dsub(pim, v.y);
                double wd = dmul(w, dadd(dmul(dr, dr), dmul(di, di)));
                acc[p] += wd;
                sumwd += wd;
            }
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            int k = j / nrot;
            double2 tr = trans[t];
            atomicAdd(&wk[0 * K + k], w);
            atomicAdd(&wk[1 * K + k], w);
            atomicAdd(&wk[2 * K + k], w * (oo.x + tr.x));
            atomicAdd(&wk[3 * K + k], w * (oo.y + tr.y));
            double ox = priorx[k] - oo.x - tr.x, oy = priory[k] - oo.y - tr.y;
            atomicAdd(&wk[5 * K + g], w);
            atomicAdd(&wk[4 * K + k], w * (ox * ox + oy * oy));
        }
    }
#pragma unroll
    for (int p = 0; p < PIX; p++)
        if (ires_p[p] > -1 && ires_p[p] < 1024 && acc[p] != 0.0) atomicAdd(&spec[ires_p[p]], acc[p]);
    sumwd = block_reduce_sum(sumwd, red);
    __syncthreads();
    for (int q = threadIdx.x; q < oriF && q < 1024; q += NT)
        if (spec[q] != 0.0) atomicAdd(&wsn[(long)g * oriF + q], spec[q]);
    if (threadIdx.x == 0 && sumwd != 0.0) atomicAdd(&normcorr[i], sumwd);
}

// backProjection over the orientation's list segment (see bp_kernel)
template <int NT, int PIX>
__global__ void __launch_bounds__(NT, 4)
    bp_list_kernel(int T, int nrot, int F, int csF, int cs, const SigEntry* __restrict__ sorted,
                   const int* __restrict__ off, const double2* __restrict__ Fnm, const double* __restrict__ Mctf2,
                   const double2* __restrict__ shifts, const double2* __restrict__ ph,
                   const double4* __restrict__ rot, int r_max, int pad, int padF, double2* __restrict__ bp_data,
                   double* __restrict__ bp_weight, long vox, int j0) {
    const int j = j0 + blockIdx.y;  // launched in chunks of at most 65,535 orientations (grid y limit)
    const int s0 = off[j], ns = off[j + 1] - s0;
    if (ns == 0) return;
    const int n0 = blockIdx.x * NT * PIX;
    const int k = j / nrot;
    double sr[PIX], si[PIX], sw[PIX], xs[PIX], ys[PIX];
    bool on[PIX];
    const int max_r2 = r_max * r_max;
#pragma unroll
    for (int p = 0; p < PIX; p++) {
        sr[p] = si[p] = sw[p] = 0.0;
        int n = n0 + threadIdx.x + p * NT;
        on[p] = false;
        if (n < F) {
            int row = n / csF, x = n - row * csF;
            int y = row, first_x = 0;
            bool rowok = true;
            if (row <= r_max) {
                y = row;
                first_x = 0;
            } else if (row >= cs - r_max) {
                y = row - cs;
                first_x = 1;
            } else
                rowok = false;
            on[p] = rowok && x >= first_x && x <= r_max && x * x + y * y <= max_r2;
            xs[p] = (double)x;
            ys[p] = (double)(row < csF ? row : row - cs);
        }
    }
    for (int q = 0; q < ns; q++) {
        const SigEntry s = sorted[s0 + q];
        const int t = s.e - j * T;
        const double w = s.w;
        const double2 sh = shifts[t];
#pragma unroll
        for (int p = 0; p < PIX; p++) {
            if (on[p]) {
                int n = n0 + threadIdx.x + p * NT;
                double2 v = apply_phase(sh, ph[(long)t * F + n], Fnm[(long)s.i * F + n]);
                sr[p] = dadd(sr[p], dmul(v.x, w));
                si[p] = dadd(si[p], dmul(v.y, w));
                sw[p] = dadd(sw[p], dmul(Mctf2[(long)s.i * F + n], w));
            }
        }
    }
    const double4 A = rot[j];
    const int shift = -(int)((float)pad / 2.0f);
    double2* D = bp_data + (long)k * vox;
    double* W = bp_weight + (long)k * vox;
#pragma unroll
    for (int p = 0; p < PIX; p++) {
        if (!on[p]) continue;
        double mw = sw[p];
        if (!(mw > 0.)) continue;
        double x = xs[p], y = ys[p];
        double vr = sr[p], vi = si[p];
        double xp = dadd(dmul(A.x, x), dmul(A.y, y));
        double yp = dadd(dmul(A.z, x), dmul(A.w, y));
        if (xp < 0) {
            xp = -xp;
            yp = -yp;
            vi = -1 * vi;
        }
        int x0 = (int)floor(xp);
        double fx = dsub(xp, (double)x0);
        int y0 = (int)floor(yp);
        double fy = dsub(yp, (double)y0);
        y0 -= shift;
        int y1 = y0 + 1;
        double mfx = dsub(1., fx), mfy = dsub(1., fy);
        double dd00 = dmul(mfy, mfx), dd01 = dmul(mfy, fx), dd10 = dmul(fy, mfx), dd11 = dmul(fy, fx);
        double* t00 = (double*)(D + (long)y0 * padF + x0);
        double* t10 = (double*)(D + (long)y1 * padF + x0);
        atomicAdd(t00 + 0, dmul(dd00, vr));
        atomicAdd(t00 + 1, dmul(dd00, vi));
        atomicAdd(t00 + 2, dmul(dd01, vr));
        atomicAdd(t00 + 3, dmul(dd01, vi));
        atomicAdd(t10 + 0, dmul(dd10, vr));
        atomicAdd(t10 + 1, dmul(dd10, vi));
        atomicAdd(t10 + 2, dmul(dd11, vr));
        atomicAdd(t10 + 3, dmul(dd11, vi));
        double* w00 = W + (long)y0 * padF + x0;
        double* w10 = W + (long)y1 * padF + x0;
        atomicAdd(w00 + 0, dmul(dd00, mw));
        atomicAdd(w00 + 1, dmul(dd01, mw));
        atomicAdd(w10 + 0, dmul(dd10, mw));
        atomicAdd(w10 + 1, dmul(dd11, mw));
    }
}

}  // namespace
}  // namespace rome
