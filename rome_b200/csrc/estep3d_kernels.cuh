// Kernels of the MAP3D E-step that have no 2D counterpart: Fourier-slice
// projection from and back-projection into 3D volumes, the compaction of
// coarse-significant points into the fine pass, and the fine-pass squared
// differences over those points only.
#pragma once

#include "estep_kernels.cuh"

namespace rome {
// internal linkage: every translation unit that launches these kernels gets its own copy
namespace {

// Slice-to-volume map of one orientation: (xp, yp, zp) = Ainv * (x, y) with
// Ainv[i][j] = A[j][i] * padding_factor (MyProjector::project,
// src/reconstruct.cpp:265-276), A = Euler_angles2matrix(rot, tilt, psi).
struct Rot3 {
    double a00, a01, a10, a11, a20, a21;
};

__device__ __forceinline__ double lin_interp(double a, double l, double h) { return dadd(l, dmul(dsub(h, l), a)); }

// MyProjector::project / projectOneTile (src/reconstruct.cpp:226-624),
// trilinear branch, at slice pixel (x, y); data is [pad][pad][pad/2+1].
__device__ __forceinline__ double2 project3d_point(const double2* __restrict__ data, int pad, int padF,
                                                   const Rot3& A, int x, int y) {
    const int shift = -(int)((float)pad / 2.0f);
    double xp = dadd(dmul(A.a00, (double)x), dmul(A.a01, (double)y));
    double yp = dadd(dmul(A.a10, (double)x), dmul(A.a11, (double)y));
    double zp = dadd(dmul(A.a20, (double)x), dmul(A.a21, (double)y));
    const bool neg = xp < 0;
    if (neg) {
        xp = -xp;
        yp = -yp;
        zp = -zp;
    }
    const int x0 = (int)floor(xp);
    const double fx = dsub(xp, (double)x0);
    int y0 = (int)floor(yp);
    const double fy = dsub(yp, (double)y0);
    y0 -= shift;
    int z0 = (int)floor(zp);
    const double fz = dsub(zp, (double)z0);
    z0 -= shift;
    const long py = padF, pz = (long)pad * padF;
    const double2* p000 = data + z0 * pz + y0 * py + x0;
    const double2* p010 = p000 + py;
    const double2* p100 = p000 + pz;
    const double2* p110 = p100 + py;
    const double2 d000 = p000[0], d001 = p000[1], d010 = p010[0], d011 = p010[1];
    const double2 d100 = p100[0], d101 = p100[1], d110 = p110[0], d111 = p110[1];
    const double dx00r = lin_interp(fx, d000.x, d001.x), dx00i = lin_interp(fx, d000.y, d001.y);
    const double dx01r = lin_interp(fx, d100.x, d101.x), dx01i = lin_interp(fx, d100.y, d101.y);
    const double dx10r = lin_interp(fx, d010.x, d011.x), dx10i = lin_interp(fx, d010.y, d011.y);
    const double dx11r = lin_interp(fx, d110.x, d111.x), dx11i = lin_interp(fx, d110.y, d111.y);
    const double dxy0r = lin_interp(fy, dx00r, dx10r), dxy0i = lin_interp(fy, dx00i, dx10i);
    const double dxy1r = lin_interp(fy, dx01r, dx11r), dxy1i = lin_interp(fy, dx01i, dx11i);
    double2 v = make_double2(lin_interp(fz, dxy0r, dxy1r), lin_interp(fz, dxy0i, dxy1i));
    if (neg) v.y = -1.0 * v.y;
    return v;
}

// one projected coefficient into the requested outputs of project3d_kernel
__device__ __forceinline__ void project3d_store(int j, int a, double2 v, int J, int Kact, int Kp, int Kq,
                                                double2* __restrict__ P_out, float* __restrict__ Q,
                                                void* __restrict__ Bop, int precision) {
    if (P_out && a < Kact) P_out[(long)j * Kact + a] = v;
    if (Q && a < Kq) Q[(long)j * Kq + a] = (float)(v.x * v.x + v.y * v.y);
    if (!Bop) return;
    const long o = (long)j * Kp + 2 * a;
    if (precision == ROME_PREC_FP32) {
        *(float2*)((float*)Bop + o) = make_float2((float)v.x, (float)v.y);
    } else {
        __nv_bfloat16* Bh = (__nv_bfloat16*)Bop;
        __nv_bfloat16* Bl = Bh + (long)J * Kp;
        const float fr = (float)v.x, fi = (float)v.y;
        const __nv_bfloat16 hr = __float2bfloat16_rn(fr), hi = __float2bfloat16_rn(fi);
        Bh[o] = hr;
        Bh[o + 1] = hi;
        if (precision == ROME_PREC_BF16X3) {
            Bl[o] = __float2bfloat16_rn(fr - __bfloat162float(hr));
            Bl[o + 1] = __float2bfloat16_rn(fi - __bfloat162float(hi));
        }
    }
}

// Projections of J orientations on the active pixels (r^2 <= my_r_max^2;
// every other coefficient of the slice is zero).  jclass[j] selects the
// class volume.  Writes, each optional: the FP64 projection [J][Kact], |P|^2
// as the norm-term operand [J][Kq] and the cross-term B operand [J][Kp]
// (FP32 re/im interleaved, or BF16 hi/lo planes as the 2D projector).
__global__ void project3d_kernel(int J, int Kact, int Kp, int Kq, int cs, int csF, int my_r_max, int pad, int padF,
                                 const int* __restrict__ jclass, const double2* __restrict__ proj_data, long vox,
                                 const Rot3* __restrict__ rot, const int* __restrict__ act,
                                 const int* __restrict__ jvalid, double2* __restrict__ P_out, float* __restrict__ Q,
                                 void* __restrict__ Bop, int precision) {
    const int j = blockIdx.x;
    const bool ok = jvalid == nullptr || jvalid[j] != 0;
    const Rot3 A = rot[j];
    const double2* data = proj_data + (long)jclass[j] * vox;
    auto point = [&](int a) {
        double2 v = make_double2(0.0, 0.0);
        if (ok && a < Kact) {
            const int n = act[a];
            const int row = n / csF;
            const int x = n - row * csF;
            const int y = row <= my_r_max ? row : row - cs;
            v = project3d_point(data, pad, padF, A, x, y);
        }
        return v;
    };
    // two pixels per thread per step: both pixels' 8 voxel loads are in flight before either is interpolated
    for (int a0 = threadIdx.x; a0 < Kp / 2; a0 += 2 * blockDim.x) {
        const int a1 = a0 + blockDim.x;
        const double2 v0 = point(a0);
        const double2 v1 = a1 < Kp / 2 ? point(a1) : make_double2(0.0, 0.0);
        for (int h = 0; h < 2; h++) {
            const int a = h ? a1 : a0;
            if (a >= Kp / 2) break;
            const double2 v = h ? v1 : v0;
            project3d_store(j, a, v, J, Kact, Kp, Kq, P_out, Q, Bop, precision);
        }
    }
    if (Q)
        for (int a = Kp / 2 + threadIdx.x; a < Kq; a += blockDim.x) Q[(long)j * Kq + a] = 0.f;
}

// ---------------------------------------------------------------------------
// Cross-correlation mode: the norm of each particle's masked image at the
// pass size, sqrt(sum_n |X_n|^2) over every coefficient of the window
// (exp_local_sqrtXi2, src/exp_model.cpp:1037-1045).  One CTA per particle.
__global__ void sqrt_xi2_kernel(int F, const double2* __restrict__ Fimg, double* __restrict__ out) {
    __shared__ double red[32];
    const int i = blockIdx.x;
    const double2* X = Fimg + (long)i * F;
    double s = 0.0;
    for (int n = threadIdx.x; n < F; n += blockDim.x) s += X[n].x * X[n].x + X[n].y * X[n].y;
    s = block_reduce_sum(s, red);
    if (threadIdx.x == 0) out[i] = sqrt(s);
}

// ---------------------------------------------------------------------------
// Fine pass: the coarse-significant points of every particle, in the
// reference's list order (class, dir, psi, coarse translation ascending:
// getAllSquaredDifferencesFine, src/map3d_optimizer.cpp:1261-1372, visits
// exp_Mcoarse_significant in exactly this order).

// Significant coarse points per particle (Mcoarse_significant holds 0 or 1
// per byte): 16 bytes per load when the rows are 16-byte aligned.
__global__ void mcoarse_count_kernel(long ncoarse, const char* __restrict__ mcoarse, int* __restrict__ cnt) {
    __shared__ int red[32];
    const int i = blockIdx.x;
    const char* m = mcoarse + (long)i * ncoarse;
    int c = 0;
    if ((ncoarse & 15) == 0) {
        const uint4* m4 = (const uint4*)m;
        for (long q = threadIdx.x; q < ncoarse / 16; q += blockDim.x) {
            const uint4 v = m4[q];
            c += __popc(v.x) + __popc(v.y) + __popc(v.z) + __popc(v.w);
        }
    } else {
        for (long e = threadIdx.x; e < ncoarse; e += blockDim.x) c += m[e] != 0;
    }
    c = block_reduce_sum(c, red);
    if (threadIdx.x == 0) cnt[i] = c;
}

// Orientations some particle needs (exp_Rot_significant,
// isSignificantAnyParticleAnyTranslation, src/map3d_optimizer.cpp:956-985,
// :2801-2814) from the list of coarse-significant points (coarse index e =
// jc * ntr + itr): the same set the dense Mcoarse_significant marks.
__global__ void rotsig_from_list_kernel(int n, int ntr, const SigEntry* __restrict__ list, char* __restrict__ rotsig) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) rotsig[list[q].e / ntr] = 1;
}

// Ordered compaction of particle i's significant coarse points e = jc * ntr
// + itr into (a) the fine-pass entries fe[off[i] + r] = (i, r, u, itr), u
// the compact index of orientation jc among the orientations some particle
// needs, and (b) the row-layout prior index ent[off[i] + r] =
// (jc / npsi, itr), the pdf_direction index (class * ndir + dir) and the
// coarse translation.  Each thread scans 16
// bytes per step (one block-wide scan of the counts per 8 KB of the row).
constexpr int FE_THREADS = 512;
__global__ void __launch_bounds__(FE_THREADS)
    fine_entries_kernel(long ncoarse, int ntr, int npsi, const char* __restrict__ mcoarse, const int* __restrict__ off,
                        const int* __restrict__ ucompact, int4* __restrict__ fe, int2* __restrict__ ent) {
    __shared__ int wsum[FE_THREADS / 32 + 1];
    const int i = blockIdx.x;
    const char* m = mcoarse + (long)i * ncoarse;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool vec = (ncoarse & 15) == 0;
    const int per = vec ? 16 : 1;  // bytes per thread per step
    int base = 0;
    for (long c0 = 0; c0 < ncoarse; c0 += (long)FE_THREADS * per) {
        const long e0 = c0 + (long)threadIdx.x * per;
        uint4 v = make_uint4(0, 0, 0, 0);
        int cnt = 0;
        if (e0 < ncoarse) {
            if (vec) {
                v = *(const uint4*)(m + e0);
                cnt = __popc(v.x) + __popc(v.y) + __popc(v.z) + __popc(v.w);
            } else {
                v.x = m[e0] != 0;
                cnt = (int)v.x;
            }
        }
        // block-wide exclusive scan of the counts
        int incl = cnt;
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            int w = lane < FE_THREADS / 32 ? wsum[lane] : 0;
            int x = w;
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += t;
            }
            if (lane < FE_THREADS / 32) wsum[lane] = x - w;  // exclusive warp offsets
            if (lane == FE_THREADS / 32 - 1) wsum[FE_THREADS / 32] = x;  // block total
        }
        __syncthreads();
        if (cnt) {
            int r = base + wsum[warp] + incl - cnt;
            const unsigned words[4] = {v.x, v.y, v.z, v.w};
            for (int b = 0; b < per; b++) {
                if (!((words[b >> 2] >> (8 * (b & 3))) & 0xFF)) continue;
                const long e = e0 + b;
                const int jc = (int)(e / ntr), itr = (int)(e - (long)jc * ntr);
                fe[off[i] + r] = make_int4(i, r, ucompact[jc], itr);
                ent[off[i] + r] = make_int2(jc / npsi, itr);
                r++;
            }
        }
        base += wsum[FE_THREADS / 32];
        __syncthreads();
    }
}

// The (particle, coarse translation) pairs the fine pass needs: flag[i *
// ntr + itr] for every coarse-significant point.
__global__ void fine_pair_flag_kernel(int E, int ntr, const int4* __restrict__ fe, int* __restrict__ flag) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < E) flag[fe[q].x * ntr + fe[q].w] = 1;
}

// pair index -> particle * ntr + coarse translation (pid = exclusive scan of the flags)
__global__ void fine_pair_list_kernel(int n, const int* __restrict__ flag, const int* __restrict__ pid,
                                      int* __restrict__ pair_of) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n && flag[q]) pair_of[pid[q]] = q;
}

// Fine-pass A operand of the needed (particle, coarse translation) pairs
// only: rows pair * notr + t for the notr over-translations of the pair's
// coarse translation (the rows shift_operand2_kernel would write at i * Tf +
// itr * notr + t, same arithmetic, FP32), and S of each row.  One CTA per
// pair slot; slots beyond the number of pairs (npairs[0]) return.
template <int NT>
__global__ void __launch_bounds__(NT)
    fine_pair_operand_kernel(const int* __restrict__ npairs, const int* __restrict__ pair_of, int ntr, int notr, int F,
                             int Kact, int Kp, const double2* __restrict__ Fimg, const double* __restrict__ lctf,
                             const double* __restrict__ Minv, int apply_ctf, const int* __restrict__ act,
                             const unsigned short* __restrict__ pidx, const double2* __restrict__ tab,
                             float* __restrict__ A, float* __restrict__ S, const double* __restrict__ pscale) {
    const int p = blockIdx.x;
    if (p >= npairs[0]) return;
    __shared__ float2 stab[5000];
    __shared__ double red[32];
    const int q = pair_of[p], i = q / ntr, itr = q - i * ntr;
    for (int k = threadIdx.x; k < 5000; k += NT) stab[k] = make_float2((float)tab[k].x, (float)tab[k].y);
    const double2* X = Fimg + (long)i * F;
    const double* M = Minv ? Minv + (long)i * F : nullptr;  // null: cross-correlation mode, no weighting
    const double* C = lctf + (long)i * F;
    const double sc = pscale ? pscale[i] : 1.0;  // the group's intensity scale on the reference
    double s = 0.0;
    for (int n = threadIdx.x; n < F; n += NT) {
        const double2 v = X[n];
        s += (M ? M[n] : 1.0) * (v.x * v.x + v.y * v.y);
    }
    s = block_reduce_sum(s, red);
    for (int a = threadIdx.x; a < Kp / 2; a += NT) {
        float2 xw = make_float2(0.f, 0.f);
        if (a < Kact) {
            const int n = act[a];
            const double m = M ? M[n] : 1.0;
            const double w = (apply_ctf ? m * C[n] : m) * sc;
            xw = make_float2((float)(w * X[n].x), (float)(w * X[n].y));
        }
        for (int t = 0; t < notr; t++) {
            float fr = 0.f, fi = 0.f;
            if (a < Kact) {
                const unsigned short pi = pidx[(long)(itr * notr + t) * Kact + a];
                if (pi == 0xFFFF) {
                    fr = xw.x;
                    fi = xw.y;
                } else {
                    const float2 cs = stab[pi & 0x7FFF];
                    const float sn = (pi & 0x8000) ? -cs.y : cs.y;
                    fr = cs.x * xw.x - sn * xw.y;
                    fi = cs.x * xw.y + sn * xw.x;
                }
            }
            *(float2*)(A + ((long)p * notr + t) * Kp + 2 * a) = make_float2(fr, fi);
        }
    }
    if (threadIdx.x < notr) S[(long)p * notr + threadIdx.x] = (float)s;
}

// Fine-pass squared differences of one coarse-significant point: nor fine
// orientations (u * nor + o) x notr fine translations (itr * notr + t),
// written at [off[i] + r][o * notr + t] of the unpadded ragged rows (the ihidden order
// itrans -> over_rot -> over_trans of the reference's lists,
// src/map3d_optimizer.cpp:1340-1358).  A holds the shifted images of the
// needed (particle, coarse translation) pairs only, pair pid[i * ntr + itr].  diff2 = (N - 2 C + S + Xi2) / 2 with
// the cross term C = <A_(i,t), B_(u,o)>, the norm term N = <W2_i, Q_(u,o)>
// (FP32 products, FP64 block sums) and the per-particle minimum folded in.
template <int NT, int NOR, int NOTR>
__global__ void __launch_bounds__(NT)
    fine_diff2_kernel(int ntr, int Kp, int Kq, const int4* __restrict__ fe, const int* __restrict__ pid,
                      const float* __restrict__ A, const float* __restrict__ B, const float* __restrict__ W2,
                      const float* __restrict__ Q, const float* __restrict__ S, const double* __restrict__ xi2,
                      float* __restrict__ diff2, unsigned* __restrict__ rowmin, const double* __restrict__ ccx) {
    constexpr int NH = NOR * NOTR;
    static_assert(NH == 32, "one warp holds the 32 sub-hypotheses of a point");
    __shared__ double red[NT / 32][NH + NOR];
    const int4 en = fe[blockIdx.x];
    const int i = en.x, u = en.z, itr = en.w;
    const long arow = (long)pid[i * ntr + itr] * NOTR;  // the pair's rows of the compacted A operand
    const float2* Ar[NOTR];
    const float2* Br[NOR];
    const float* Qr[NOR];
#pragma unroll
    for (int t = 0; t < NOTR; t++) Ar[t] = (const float2*)(A + (arow + t) * Kp);
#pragma unroll
    for (int o = 0; o < NOR; o++) {
        Br[o] = (const float2*)(B + ((long)u * NOR + o) * Kp);
        Qr[o] = Q + ((long)u * NOR + o) * Kq;
    }
    const float* w2 = W2 + (long)i * Kq;
    float c[NH], nn[NOR];
#pragma unroll
    for (int h = 0; h < NH; h++) c[h] = 0.f;
#pragma unroll
    for (int o = 0; o < NOR; o++) nn[o] = 0.f;
    for (int a = threadIdx.x; a < Kp / 2; a += NT) {
        float2 av[NOTR];
#pragma unroll
        for (int t = 0; t < NOTR; t++) av[t] = Ar[t][a];
#pragma unroll
        for (int o = 0; o < NOR; o++) {
            const float2 b = Br[o][a];
#pragma unroll
            for (int t = 0; t < NOTR; t++) c[o * NOTR + t] += av[t].x * b.x + av[t].y * b.y;
        }
    }
    for (int a = threadIdx.x; a < Kq; a += NT) {
        const float w = w2[a];
#pragma unroll
        for (int o = 0; o < NOR; o++) nn[o] += w * Qr[o][a];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int h = 0; h < NH + NOR; h++) {
        double v = h < NH ? (double)c[h] : (double)nn[h - NH];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) red[warp][h] = v;
    }
    __syncthreads();
    if (threadIdx.x < NH) {
        const int h = threadIdx.x, o = h / NOTR, t = h - o * NOTR;
        double cs = 0.0, ns = 0.0;
        for (int w = 0; w < NT / 32; w++) {
            cs += red[w][h];
            ns += red[w][NH + o];
        }
        // cross-correlation mode (ccx = the particle's image norms): -C / (sqrt(N) * |X|), get_diff,
        // src/map3d_optimizer.cpp:1086-1102
        const float v = ccx ? (float)(-cs / (sqrt(ns) * ccx[i]))
                            : (float)(0.5 * (ns - 2.0 * cs + (double)S[arow + t] + xi2[i]));
        diff2[(long)blockIdx.x * NH + h] = v;  // point blockIdx.x = off[i] + r of the ragged rows
        float m = v;
        for (int off = 16; off > 0; off >>= 1) m = fminf(m, __shfl_down_sync(0xffffffffu, m, off));
        if (h == 0) atomicMin(&rowmin[i], float_key(m));
    }
}

// The significant fine hypotheses of the walk, re-indexed from the ragged
// row position e = r * NH + o * notr + t to the dense position over the
// fine orientations and translations, e' = (u * nor + o) * Tf + itr * notr + t,
// so that the wsum and back-projection kernels can group them by orientation.
__global__ void fine_list_dense_kernel(int n, int nor, int notr, int Tf, int stride, const int4* __restrict__ fe,
                                       const int* __restrict__ off, SigEntry* __restrict__ list) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    SigEntry s = list[q];
    const int nh = nor * notr;
    const int r = s.e / nh, h = s.e - r * nh, o = h / notr, t = h - o * notr;
    const int4 en = fe[off[s.i] + r];
    s.e = (en.z * nor + o) * Tf + en.w * notr + t;
    list[q] = s;
}

// ---------------------------------------------------------------------------
// updateOtherParams (src/map3d_optimizer.cpp:2059-2236 and
// CoarseAndFineSearch::updateModel :1484-1602) over each particle's list
// segment of significant fine hypotheses: wsum_sigma2_noise per resolution
// shell of the particle's group, the norm-correction sum, sumw_group,
// wsum_pdf_class, wsum_pdf_direction[class][dir] and wsum_sigma2_offset.
// jcd[j] = class * ndir + dir of fine orientation j.  wk: [0,K) pdf_class,
// [K, K + K*ndir) pdf_direction, then sigma2_offset, then [G] sumw_group.
// SCALE (intensity-scale correction): the reference is Frefctf times the
// particle's scale sc.pscale[i], and the pixels of the shells whose
// data_vs_prior of the hypothesis' class exceeds 3 also add
// w * Re(Frefctf conj(X)) and w * |Frefctf|^2 to the particle's XA and AA
// spectra (get_wdiff2 'S' pixels, src/map3d_optimizer.cpp:1488-1502).
struct ScaleSums {
    const double* pscale = nullptr;  // [P]
    const double* dvp = nullptr;     // data_vs_prior_class [K][oriF]
    double* xa = nullptr;            // [P][oriF]
    double* aa = nullptr;            // [P][oriF]
};
template <int NT, int PIX, bool SCALE>
__global__ void __launch_bounds__(NT)
    wsum3d_list_kernel(int T, int K, int ndir, int F, int csF, int cs, int oriF, const SigEntry* __restrict__ list,
                       const int* __restrict__ seg, const int* __restrict__ jcd, const double2* __restrict__ Fimg,
                       const double* __restrict__ lctf, int apply_ctf, const double2* __restrict__ proj,
                       const int* __restrict__ actidx, int Kact, const double2* __restrict__ shifts,
                       const double2* __restrict__ ph, const int* __restrict__ Mresol, const int* __restrict__ group,
                       const double2* __restrict__ oldoff, const double2* __restrict__ trans,
                       const double* __restrict__ priorx, const double* __restrict__ priory,
                       double* __restrict__ wsn, double* __restrict__ normcorr, double* __restrict__ wk, int chunk,
                       ScaleSums sc) {
    const int i = blockIdx.y;
    const int n0 = blockIdx.x * NT * PIX;
    // blockIdx.z takes entries [z * chunk, (z + 1) * chunk) of the particle's segment, so that a particle
    // with many significant hypotheses is spread over many CTAs (all sums below are atomic)
    const int z0 = blockIdx.z * chunk;
    if (z0 >= seg[2 * i + 1]) return;
    const int s0 = seg[2 * i] + z0, ns = min(chunk, seg[2 * i + 1] - z0);
    __shared__ double spec[1024];
    __shared__ double red[32];
    __shared__ double sxa[SCALE ? 1024 : 1], saa[SCALE ? 1024 : 1];
    for (int q = threadIdx.x; q < oriF && q < 1024; q += NT) {
        spec[q] = 0.0;
        if (SCALE) sxa[q] = saa[q] = 0.0;
    }
    __syncthreads();
    double acc[PIX], axa[SCALE ? PIX : 1], aaa[SCALE ? PIX : 1];
    int ires_p[PIX];
    double2 Xp[PIX];
    double cp[PIX];
    int ap[PIX];
    const double psc = SCALE ? sc.pscale[i] : 1.0;
#pragma unroll
    for (int p = 0; p < PIX; p++) {
        acc[p] = 0.0;
        if (SCALE) axa[p] = aaa[p] = 0.0;
        const int n = n0 + threadIdx.x + p * NT;
        ires_p[p] = n < F ? Mresol[n] : -1;
        if (ires_p[p] > -1) {
            Xp[p] = Fimg[(long)i * F + n];
            cp[p] = lctf[(long)i * F + n];
            ap[p] = actidx[n];
        }
    }
    double sumwd = 0.0;
    const int g = group[i];
    const double2 oo = oldoff[i];
    const int KD = K * ndir;
    for (int q = 0; q < ns; q++) {
        const SigEntry s = list[s0 + q];
        const int j = s.e / T, t = s.e - j * T;
        const double w = s.w;
        const double2 sh = shifts[t];
        const double2* Pj = proj + (long)j * Kact;
        const double* dv = SCALE ? sc.dvp + (long)(jcd[j] / ndir) * oriF : nullptr;
#pragma unroll
        for (int p = 0; p < PIX; p++) {
            if (ires_p[p] > -1) {
                const double2 v = apply_phase(sh, ph[(long)t * F + n0 + threadIdx.x + p * NT], Xp[p]);
                const double2 pv = ap[p] >= 0 ? Pj[ap[p]] : make_double2(0.0, 0.0);
                double pr = apply_ctf ? dmul(pv.x, cp[p]) : pv.x;
                double pim = apply_ctf ? dmul(pv.y, cp[p]) : pv.y;
                if (SCALE) {
                    pr = dmul(pr, psc);
                    pim = dmul(pim, psc);
                }
                const double dr = dsub(pr, v.x), di = dsub(pim, v.y);
                const double wd = dmul(w, dadd(dmul(dr, dr), dmul(di, di)));
                acc[p] += wd;
                sumwd += wd;
                if (SCALE && dv[ires_p[p]] > 3.) {
                    axa[p] += dmul(w, dadd(dmul(pr, v.x), dmul(pim, v.y)));
                    aaa[p] += dmul(w, dadd(dmul(pr, pr), dmul(pim, pim)));
                }
            }
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            const int cd = jcd[j], k = cd / ndir;
            const double2 tr = trans[t];
            atomicAdd(&wk[k], w);
            atomicAdd(&wk[K + cd], w);
            atomicAdd(&wk[K + KD + 1 + g], w);
            const double ox = priorx[k] - oo.x - tr.x, oy = priory[k] - oo.y - tr.y;
            atomicAdd(&wk[K + KD], w * (ox * ox + oy * oy));
        }
    }
#pragma unroll
    for (int p = 0; p < PIX; p++) {
        if (ires_p[p] > -1 && ires_p[p] < 1024 && acc[p] != 0.0) atomicAdd(&spec[ires_p[p]], acc[p]);
        if (SCALE && ires_p[p] > -1 && ires_p[p] < 1024 && (axa[p] != 0.0 || aaa[p] != 0.0)) {
            atomicAdd(&sxa[ires_p[p]], axa[p]);
            atomicAdd(&saa[ires_p[p]], aaa[p]);
        }
    }
    sumwd = block_reduce_sum(sumwd, red);
    __syncthreads();
    for (int q = threadIdx.x; q < oriF && q < 1024; q += NT) {
        if (spec[q] != 0.0) atomicAdd(&wsn[(long)g * oriF + q], spec[q]);
        if (SCALE && sxa[q] != 0.0) atomicAdd(&sc.xa[(long)i * oriF + q], sxa[q]);
        if (SCALE && saa[q] != 0.0) atomicAdd(&sc.aa[(long)i * oriF + q], saa[q]);
    }
    if (threadIdx.x == 0 && sumwd != 0.0) atomicAdd(&normcorr[i], sumwd);
}

// Trilinear scatter of one slice coefficient (x, y) with value (vr, vi) and
// weight mw into a class volume: MyBackProjector::backproject
// (src/reconstruct.cpp:977-1164) for one pixel, with the reference's
// operation order.  A is Ainv = A^T * padding; points with xp < 0 go to
// their Friedel mate (negated coordinates, conjugated value).
__device__ __forceinline__ void bp3d_scatter(const Rot3& A, double x, double y, double vr, double vi, double mw,
                                             int pad, int padF, double2* __restrict__ D, double* __restrict__ W) {
    const int shift = -(int)((float)pad / 2.0f);
    const long py = padF, pz = (long)pad * padF;
    double xp = dadd(dmul(A.a00, x), dmul(A.a01, y));
    double yp = dadd(dmul(A.a10, x), dmul(A.a11, y));
    double zp = dadd(dmul(A.a20, x), dmul(A.a21, y));
    if (xp < 0) {
        xp = -xp;
        yp = -yp;
        zp = -zp;
        vi = -vi;
    }
    const int x0 = (int)floor(xp);
    const double fx = dsub(xp, (double)x0);
    int y0 = (int)floor(yp);
    const double fy = dsub(yp, (double)y0);
    y0 -= shift;
    int z0 = (int)floor(zp);
    const double fz = dsub(zp, (double)z0);
    z0 -= shift;
    const double mfx = dsub(1., fx), mfy = dsub(1., fy), mfz = dsub(1., fz);
    const double dd[8] = {dmul(dmul(mfz, mfy), mfx), dmul(dmul(mfz, mfy), fx), dmul(dmul(mfz, fy), mfx),
                          dmul(dmul(mfz, fy), fx),   dmul(dmul(fz, mfy), mfx), dmul(dmul(fz, mfy), fx),
                          dmul(dmul(fz, fy), mfx),   dmul(dmul(fz, fy), fx)};
    const long b000 = z0 * pz + y0 * py + x0;
    const long base[4] = {b000, b000 + py, b000 + pz, b000 + pz + py};  // (z0,y0) (z0,y1) (z1,y0) (z1,y1)
#pragma unroll
    for (int c = 0; c < 4; c++) {
        double* td = (double*)(D + base[c]);
        atomicAdd(td + 0, dmul(dd[2 * c], vr));
        atomicAdd(td + 1, dmul(dd[2 * c], vi));
        atomicAdd(td + 2, dmul(dd[2 * c + 1], vr));
        atomicAdd(td + 3, dmul(dd[2 * c + 1], vi));
        atomicAdd(W + base[c], dmul(dd[2 * c], mw));
        atomicAdd(W + base[c] + 1, dmul(dd[2 * c + 1], mw));
    }
}

// backProjection (src/map3d_optimizer.cpp:2360-2479): per fine orientation,
// the weighted sum of the significant shifted nomask images (times ctf *
// Minvsigma2) and of ctf^2 * Minvsigma2, then MyBackProjector::backproject
// (src/reconstruct.cpp:977-1164, trilinear) into the class volume.  The
// reference back-projects each particle's slice; summing the slices of one
// orientation first changes only the FP64 rounding.
template <int NT, int PIX>
__global__ void __launch_bounds__(NT)
    bp3d_list_kernel(int T, int F, int csF, int cs, const SigEntry* __restrict__ sorted, const int* __restrict__ off,
                     const int* __restrict__ jclass, const double2* __restrict__ Fnm, const double* __restrict__ Mctf2,
                     const double2* __restrict__ shifts, const double2* __restrict__ ph, const Rot3* __restrict__ rot,
                     int r_max, int pad, int padF, double2* __restrict__ bp_data, double* __restrict__ bp_weight,
                     long vox, int j0) {
    const int j = j0 + blockIdx.y;  // launched in chunks of at most 65,535 orientations (grid y limit)
    const int s0 = off[j], ns = off[j + 1] - s0;
    if (ns == 0) return;
    const int n0 = blockIdx.x * NT * PIX;
    double sr[PIX], si[PIX], sw[PIX];
    int xs[PIX], ys[PIX];
    bool on[PIX];
    const int max_r2 = r_max * r_max;
#pragma unroll
    for (int p = 0; p < PIX; p++) {
        sr[p] = si[p] = sw[p] = 0.0;
        const int n = n0 + threadIdx.x + p * NT;
        on[p] = false;
        xs[p] = ys[p] = 0;
        if (n < F) {
            const int row = n / csF, x = n - row * csF;
            int y = row, first_x = 0;
            bool rowok = true;
            if (row <= r_max) {
                y = row;
                first_x = 0;
            } else if (row >= cs - r_max) {
                y = row - cs;
                first_x = 1;  // x == 0 column stored twice in FFTW order: only once here
            } else
                rowok = false;
            on[p] = rowok && x >= first_x && x <= r_max && x * x + y * y <= max_r2;
            xs[p] = x;
            ys[p] = y;
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
                const int n = n0 + threadIdx.x + p * NT;
                const double2 v = apply_phase(sh, ph[(long)t * F + n], Fnm[(long)s.i * F + n]);
                sr[p] = dadd(sr[p], dmul(v.x, w));
                si[p] = dadd(si[p], dmul(v.y, w));
                sw[p] = dadd(sw[p], dmul(Mctf2[(long)s.i * F + n], w));
            }
        }
    }
    const Rot3 A = rot[j];
    double2* D = bp_data + (long)jclass[j] * vox;
    double* W = bp_weight + (long)jclass[j] * vox;
#pragma unroll
    for (int p = 0; p < PIX; p++) {
        if (!on[p]) continue;
        const double mw = sw[p];
        if (!(mw > 0.)) continue;
        bp3d_scatter(A, (double)xs[p], (double)ys[p], sr[p], si[p], mw, pad, padF, D, W);
    }
}

// Back-projection of whole particle images at known poses: the per-image
// loop of rome_reconstruct (apps/rome_reconstruct.cpp:160-330).  Image i's
// spectrum is shifted by its own offset with the tabulated phases of
// shiftImageInFourierTransform (src/image.h:1478-1575: dotp, index
// (int)(|dotp| / sampling) % 5000, sign of dotp on the sine), multiplied by
// its CTF, and scattered with weight CTF^2 (unit value and weight without
// CTF) through MyBackProjector::backproject (src/reconstruct.cpp:977-1164).
// One block row per image, PIX pixels per thread; block row y works on
// image order[y], so that images whose slices share voxels run at the same
// time and their atomics meet in L2.
template <int NT, int PIX>
__global__ void __launch_bounds__(NT)
    bp_images_kernel(int F, int csF, int cs, const int* __restrict__ order, const double* __restrict__ Fre,
                     const double* __restrict__ Fim, const double* __restrict__ Fctf,
                     const double2* __restrict__ shifts, const double2* __restrict__ tab, double sampling,
                     const Rot3* __restrict__ rot, int r_max, int pad, int padF, double2* __restrict__ D,
                     double* __restrict__ W) {
    const long i = order[blockIdx.y];
    const double2 sh = shifts[i];
    const Rot3 A = rot[i];
    const int max_r2 = r_max * r_max;
    const double two_pi = 2 * kPi;
#pragma unroll
    for (int p = 0; p < PIX; p++) {
        const int n = blockIdx.x * NT * PIX + threadIdx.x + p * NT;
        if (n >= F) continue;
        const int row = n / csF, x = n - row * csF;
        int y;
        if (row <= r_max) {
            y = row;
            if (x > r_max) continue;
        } else if (row >= cs - r_max) {
            y = row - cs;
            if (x < 1 || x > r_max) continue;  // x == 0 column stored twice in FFTW order: only once here
        } else
            continue;
        if (x * x + y * y > max_r2) continue;
        const double c = Fctf ? Fctf[i * F + n] : 1.0;
        const double mw = Fctf ? dmul(c, c) : 1.0;
        if (!(mw > 0.)) continue;
        const double2 v = make_double2(Fre[i * F + n], Fim[i * F + n]);
        const double dotp = dmul(two_pi, dadd(dmul((double)x, sh.x), dmul((double)y, sh.y)));
        const int idx = ((int)__ddiv_rn(fabs(dotp), sampling)) % 5000;
        const double2 cs2 = tab[idx];
        const double2 s = apply_phase(sh, make_double2(cs2.x, dotp < 0 ? -cs2.y : cs2.y), v);
        const double vr = Fctf ? dmul(s.x, c) : s.x, vi = Fctf ? dmul(s.y, c) : s.y;
        bp3d_scatter(A, (double)x, (double)y, vr, vi, mw, pad, padF, D, W);
    }
}

}  // namespace
}  // namespace rome
