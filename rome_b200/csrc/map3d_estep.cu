// MAP3D E-step for one pool of particles on sm_100a.
//
// Replaces Map3dOptimizer_old::expectationSomeParticles
// (src/map3d_optimizer.cpp:883-953) minus storeWeightedSums.
//
// Coarse pass (coarse_size, nr_over_rot = nr_over_trans = 1): every
// hypothesis (class, dir, psi, trans) whose class and direction have a
// positive prior, laid out densely like the 2D pass with the direction
// folded into the class index (k = class * ndir + dir): 3D Fourier-slice
// projections (project3d_kernel), the cross term on the tensor cores (or
// FP32 CUDA cores) with the fused diff2 epilogue, then the FP64 posterior
// and significance walk.
//
// Fine pass (current_size, 8 over-rotations x 4 over-translations): only
// the coarse-significant (orientation, translation) points of each
// particle, compacted in the reference's list order; the squared
// differences of their 32 sub-hypotheses (fine_diff2_kernel), the posterior
// over the ragged rows, then updateOtherParams and backProjection over the
// significant fine hypotheses.
//
// Cross-correlation mode replaces the squared difference by the negative
// normalised correlation and the posterior by the single best hypothesis;
// intensity-scale correction multiplies the references (and the
// back-projection's CTF) by each particle's group scale and adds the XA/AA
// spectra to updateOtherParams.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "estep3d_kernels.cuh"
#include "restricted_kernels.cuh"
#include "restricted_tc.cuh"
#include "estep_kernels.cuh"
#include "gemm_simt.cuh"
#include "gemm_tc.cuh"
#include "select_kernels.cuh"

using namespace rome;

namespace rome {
namespace {

template <typename T>
T* upload3(RomeGpuCtx* ctx, Slot s, const T* host, size_t n) {
    T* d = ctx->ws[s].as<T>(n);
    stage_copy(ctx, d, host, n);
    return d;
}

// Euler_angles2matrix (src/math.cpp:86-115); the projector and the
// back-projector use Ainv[i][j] = A[j][i] * padding (src/reconstruct.cpp:265-276).
Rot3 rot3_inv(double rot, double tilt, double psi, int padding) {
    const double d2r = 3.14159265358979323846 / 180.;
    const double alpha = rot * d2r, beta = tilt * d2r, gamma = psi * d2r;
    const double ca = cos(alpha), cb = cos(beta), cg = cos(gamma);
    const double sa = sin(alpha), sb = sin(beta), sg = sin(gamma);
    const double cc = cb * ca, cs = cb * sa, sc = sb * ca, ss = sb * sa;
    const double A00 = cg * cc - sg * sa, A01 = cg * cs + sg * ca, A02 = -cg * sb;
    const double A10 = -sg * cc - cg * sa, A11 = -sg * cs + cg * ca, A12 = sg * sb;
    (void)sc;
    (void)ss;
    const double p = (double)padding;
    return Rot3{A00 * p, A10 * p, A01 * p, A11 * p, A02 * p, A12 * p};
}

struct Pass {
    int cs, csF, F, Kact, Kp, Kq, my_r_max;
};

// active pixels of a pass: the support of the projection, r^2 <= my_r_max^2
// (src/reconstruct.cpp:278-299)
Pass active_pixels(int cs, int r_max, std::vector<int>& act, std::vector<int>& actidx) {
    Pass g{};
    g.cs = cs;
    g.csF = cs / 2 + 1;
    g.F = cs * g.csF;
    g.my_r_max = std::min(r_max, cs / 2);
    act.clear();
    actidx.assign(g.F, -1);
    for (int row = 0; row < cs; row++) {
        int y;
        if (row <= g.my_r_max) y = row;
        else if (row >= cs - g.my_r_max) y = row - cs;
        else continue;
        for (int x = 0; x <= g.my_r_max; x++)
            if (x * x + y * y <= g.my_r_max * g.my_r_max) {
                actidx[row * g.csF + x] = (int)act.size();
                act.push_back(row * g.csF + x);
            }
    }
    g.Kact = (int)act.size();
    g.Kp = ((2 * g.Kact + 63) / 64) * 64;
    g.Kq = ((g.Kact + 15) / 16) * 16;
    return g;
}

}  // namespace
}  // namespace rome

extern "C" int rome_gpu_map3d_estep_pool(RomeGpuCtx* ctx, const RomeMap3dPool* in, RomeMap3dPoolOut* out) {
    if (!ctx || !in || !out) return ROME_ERR_ARG;
    return guarded(ctx, [&] {
        if (!ctx->proj || ctx->ref_dim != 3) fail(ROME_ERR_STATE, "3D projectors not set (rome_gpu_set_projectors)");
        ROME_CUDA(cudaSetDevice(ctx->device));
        arena_reset(ctx);
        ctx->proj_key.clear();  // this call reuses the 2D projection slots
        const int P = in->nr_images, K = in->nr_classes, ori = in->ori_size, cur = in->current_size;
        const int ndir = in->nr_dir, npsi = in->nr_psi, ntr = in->nr_trans, G = in->nr_groups, oriF = ori / 2 + 1;
        ROME_REQUIRE(P > 0 && K == ctx->nr_classes && ori == ctx->ori_size, "pool/projector mismatch");
        ROME_REQUIRE(cur > 0 && cur <= ori && cur % 2 == 0, "bad current_size %d", cur);
        ROME_REQUIRE(in->coarse_size > 0 && in->coarse_size <= cur && in->coarse_size % 2 == 0, "bad coarse_size %d",
                     in->coarse_size);
        if (in->adaptive_oversampling != 1)
            fail(ROME_ERR_UNSUPPORTED, "3D E-step needs adaptive_oversampling 1 (got %d)", in->adaptive_oversampling);
        ROME_REQUIRE(in->iclass_min >= 0 && in->iclass_max < K && in->iclass_min <= in->iclass_max, "bad class range");
        ROME_REQUIRE(ctx->r_max == std::min(cur / 2, ori / 2), "projector r_max %d does not match current_size %d",
                     ctx->r_max, cur);
        ROME_REQUIRE(in->Fimg_real && in->Fimg_imag && in->Fimg_nomask_real && in->Fimg_nomask_imag && in->Fctf,
                     "missing particle images");
        ROME_REQUIRE(ndir > 0 && npsi > 0 && ntr > 0 && G > 0, "empty sampling");
        for (int p = 0; p < 2; p++)
            ROME_REQUIRE(in->angles[p] && in->over_trans_x[p] && in->over_trans_y[p], "missing sampling tables (pass %d)",
                         p);
        ROME_REQUIRE(in->Mresol_coarse && in->Mresol_fine && in->pdf_direction && in->pdf_class, "missing model arrays");
        ROME_CUDA(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        const int curF2 = cur * (cur / 2 + 1);
        const int KD = K * ndir;
        const int Jc = KD * npsi;                  // coarse orientations (class, dir, psi)
        const long ncoarse = (long)Jc * ntr;       // coarse hypotheses per particle
        const int NOR = 8, NOTR = 4, NH = NOR * NOTR;
        const bool apply_ctf = in->do_ctf_correction && in->refs_are_ctf_corrected;
        const bool tc = ctx->precision != ROME_PREC_FP32;
        Profiler prof(ctx);
        // optional coarse-pass restriction (learned proposals): validated on the host
        const bool restricted = in->proposals != nullptr;
        const int nprop = restricted ? in->nr_proposals : 0;
        // cross-correlation mode (-firstiter_cc in iteration 1, -always_cc): normalised signal products
        // instead of squared differences, and the best hypothesis alone instead of the posterior
        const bool ccm = in->do_cross_correlation != 0;
        if (ccm && restricted) fail(ROME_ERR_UNSUPPORTED, "cross-correlation mode with proposals");
        // intensity-scale correction: per-particle scale of its group (check_scale, map3d_optimizer.cpp:1000-1018)
        const bool scl = in->do_scale_correction != 0;
        if (scl && restricted) fail(ROME_ERR_UNSUPPORTED, "scale correction with proposals");
        std::vector<double> hscale;
        if (scl) {
            ROME_REQUIRE(in->scale_correction && in->data_vs_prior_class,
                         "scale correction needs scale_correction and data_vs_prior_class");
            hscale.resize(P);
            for (int i = 0; i < P; i++) {
                const int gi = in->group[i];
                ROME_REQUIRE(gi >= 0 && gi < G, "group %d of particle %d out of range", gi, i);
                double sc = in->scale_correction[gi];
                if (std::isnan(sc) || std::isinf(sc)) fail(ROME_ERR_NUMERIC, "Scale is Nan or Inf (group %d)", gi + 1);
                if (sc > 10000.) fail(ROME_ERR_NUMERIC, "scale correction %g of group %d is very high", sc, gi + 1);
                hscale[i] = sc < 0.001 ? 0.001 : sc;
            }
        }
        int* dProp = nullptr;
        if (restricted) {
            ROME_REQUIRE(nprop > 0 && nprop <= Jc, "nr_proposals %d (1..%d)", nprop, Jc);
            ROME_REQUIRE(!out->coarse_diff2, "coarse_diff2 checkpoints are not available with proposals");
            for (int i = 0; i < P; i++) {
                const int* pr = in->proposals + (size_t)i * nprop;
                for (int q = 0; q < nprop; q++) {
                    ROME_REQUIRE(pr[q] >= 0 && pr[q] < Jc, "proposal %d of particle %d out of range", pr[q], i);
                    ROME_REQUIRE(q == 0 || pr[q] > pr[q - 1], "proposals of particle %d not ascending", i);
                }
            }
            dProp = upload3(ctx, S_PROP, in->proposals, (size_t)P * nprop);
        }

        // ---- particle data at current_size ----
        const double *dFr, *dFi, *dFnr, *dFni, *dCtf;
        if (in->inputs_on_device) {
            dFr = in->Fimg_real;
            dFi = in->Fimg_imag;
            dFnr = in->Fimg_nomask_real;
            dFni = in->Fimg_nomask_imag;
            dCtf = in->Fctf;
        } else {
            double* base = ctx->ws[S_TMP0].as<double>((size_t)P * curF2 * 5);
            const double* src[5] = {in->Fimg_real, in->Fimg_imag, in->Fimg_nomask_real, in->Fimg_nomask_imag,
                                    in->Fctf};
            for (int q = 0; q < 5; q++)
                ROME_CUDA(cudaMemcpyAsync(base + (size_t)q * P * curF2, src[q], sizeof(double) * P * curF2,
                                          cudaMemcpyHostToDevice, st));
            dFr = base;
            dFi = base + (size_t)P * curF2;
            dFnr = base + (size_t)2 * P * curF2;
            dFni = base + (size_t)3 * P * curF2;
            dCtf = base + (size_t)4 * P * curF2;
        }
        double* dSig2 = upload3(ctx, S_SIG2, in->sigma2_noise, (size_t)G * oriF);
        int* dGroup = upload3(ctx, S_GROUP, in->group, (size_t)P);
        double* dXi2 = upload3(ctx, S_XI2, in->highres_Xi2, (size_t)P);
        double* dScale = nullptr;  // [P] scales, then XA [P][oriF], AA [P][oriF]
        ScaleSums ssum;
        if (scl) {
            dScale = ctx->ws[S_PSCALE].as<double>((size_t)P * (1 + 2 * oriF) + (size_t)K * oriF);
            stage_copy(ctx, dScale, hscale.data(), (size_t)P);
            double* dDvp = dScale + (size_t)P * (1 + 2 * oriF);
            stage_copy(ctx, dDvp, in->data_vs_prior_class, (size_t)K * oriF);
            ROME_CUDA(cudaMemsetAsync(dScale + P, 0, sizeof(double) * 2 * P * oriF, st));
            ssum = ScaleSums{dScale, dDvp, dScale + P, dScale + P + (size_t)P * oriF};
        }
        // model values: pdf_direction [K*ndir], prior offsets [K] x 2
        std::vector<double> hcls((size_t)KD + 2 * K);
        for (int q = 0; q < KD; q++) hcls[q] = in->pdf_direction[q];
        for (int k = 0; k < K; k++) {
            hcls[KD + k] = in->prior_offsetx_class[k];
            hcls[KD + K + k] = in->prior_offsety_class[k];
        }
        double* dCls = upload3(ctx, S_PDIR, hcls.data(), hcls.size());
        const double* dPdir = dCls;
        const double* dPriorX = dCls + KD;
        const double* dPriorY = dCls + KD + K;
        std::vector<double2> hoff(P);
        for (int i = 0; i < P; i++) hoff[i] = make_double2(in->old_offsetx[i], in->old_offsety[i]);
        double2* dOld = upload3(ctx, S_OLDOFF, hoff.data(), hoff.size());
        std::vector<double2> htc(ntr);
        for (int t = 0; t < ntr; t++) htc[t] = make_double2(in->trans_x[t], in->trans_y[t]);
        double2* dTrC = upload3(ctx, S_TMP1, htc.data(), htc.size());
        double* dPoff = ctx->ws[S_POFF].as<double>((size_t)P * K * ntr);
        prof.begin(ROME_PHASE_PREP);
        pdf_offset_kernel<<<P, 128, 0, st>>>(P, K, ntr, dOld, dTrC, dPriorX, dPriorY, in->sigma2_offset, dPoff);
        ROME_CHECK_LAUNCH();
        prof.launched(ROME_PHASE_PREP);
        prof.end(ROME_PHASE_PREP);
        // (class, dir) pairs the reference visits (map3d_optimizer.cpp:1205-1206, :1279-1280)
        std::vector<int> hcd_ok(KD);
        for (int q = 0; q < KD; q++) {
            const int k = q / ndir;
            hcd_ok[q] = k >= in->iclass_min && k <= in->iclass_max && in->pdf_class[k] > 0. && in->pdf_direction[q] > 0.;
        }

        double* dPart = ctx->ws[S_PART].as<double>((size_t)P * 8);
        int* dPartI = ctx->ws[S_PARTI].as<int>((size_t)P * 8);
        char* dMcoarse = ctx->ws[S_MCOARSE].as<char>((size_t)P * ncoarse);
        int* dSeg = ctx->ws[S_SEG].as<int>((size_t)2 * P);
        std::vector<double> h_min(P), h_sum(P), h_sig(P), h_nsig(P);
        std::vector<double> hpart((size_t)P * 8);
        std::vector<int> hparti((size_t)P * 8);

        // the coarse pass's significant list (coarse index per entry) outlives the pass
        int nsig0 = 0;
        const SigEntry* dList0 = nullptr;

        // ================= pass 0: coarse, dense =================
        {
            std::vector<int> act, actidx;
            const Pass g = active_pixels(in->coarse_size, ctx->r_max, act, actidx);
            const int cs = g.cs, T = ntr, J = Jc;
            const long X = (long)J * T;
            int* dAct = upload3(ctx, S_ACT, act.data(), act.size());
            int* dMres = upload3(ctx, S_MRES, in->Mresol_coarse, (size_t)g.F);
            std::vector<int> hj((size_t)2 * J);  // jvalid, jclass
            std::vector<Rot3> hrot(J);
            for (int j = 0; j < J; j++) {
                const int cd = j / npsi, dp = j % (ndir * npsi);
                hj[j] = hcd_ok[cd];
                hj[J + j] = cd / ndir;
                const double* a = in->angles[0] + (size_t)dp * 3;
                hrot[j] = rot3_inv(a[0], a[1], a[2], ctx->padding);
            }
            int* dJ = upload3(ctx, S_JVALID, hj.data(), hj.size());
            Rot3* dRot = upload3(ctx, S_ROTM, hrot.data(), hrot.size());
            std::vector<double2> hsh(T);
            for (int t = 0; t < T; t++)
                hsh[t] = make_double2(in->over_trans_x[0][t] / (-ori), in->over_trans_y[0][t] / (-ori));
            double2* dShift = upload3(ctx, S_SHIFT, hsh.data(), hsh.size());

            double2* dFimg = ctx->ws[S_FIMG].as<double2>((size_t)P * g.F);
            double* dLctf = ctx->ws[S_CTF].as<double>((size_t)P * g.F);
            double* dMinv = ctx->ws[S_MINV].as<double>((size_t)P * g.F);
            prof.begin(ROME_PHASE_PREP);
            prep_particles_kernel<<<P, 256, 0, st>>>(P, cur, cs, dFr, dFi, dCtf, dMres, dSig2, dGroup, oriF,
                                                      in->sigma2_fudge, dFimg, dLctf, dMinv);
            ROME_CHECK_LAUNCH();
            prof.launched(ROME_PHASE_PREP);
            double* dSx = nullptr;
            if (ccm) {
                dSx = ctx->ws[S_CCX].as<double>((size_t)P);
                sqrt_xi2_kernel<<<P, 256, 0, st>>>(g.F, dFimg, dSx);
                ROME_CHECK_LAUNCH();
                prof.launched(ROME_PHASE_PREP);
            }
            prof.end(ROME_PHASE_PREP);

            float* dQ = ctx->ws[S_Q].as<float>((size_t)J * g.Kq);
            void* dB = ctx->ws[S_B].get((size_t)J * g.Kp * 4);
            prof.begin(ROME_PHASE_PROJECT);
            project3d_kernel<<<J, 128, 0, st>>>(J, g.Kact, g.Kp, g.Kq, cs, g.csF, g.my_r_max, ctx->pad_size,
                                                 ctx->pad_size / 2 + 1, dJ + J, ctx->proj, ctx->vox, dRot, dAct, dJ,
                                                 nullptr, dQ, dB, ctx->precision);
            ROME_CHECK_LAUNCH();
            prof.launched(ROME_PHASE_PROJECT);
            // algorithmic bytes: the class volumes read once, |P|^2 and the cross-term operand written
            prof.add_bytes(ROME_PHASE_PROJECT, (double)K * ctx->vox * 16 + (double)J * g.Kq * 4 +
                                                   (double)J * g.Kp * (ctx->precision == ROME_PREC_BF16 ? 2 : 4));
            prof.end(ROME_PHASE_PROJECT);

            const long M = (long)P * T;
            // restricted search on the tensor cores: no shifted images (a [TN][Kp] phase operand instead)
            const bool rtc = restricted && tc && T <= 256;
            const int Kh = g.Kp / 2;
            void* dA = nullptr;
            float* dS = ctx->ws[S_S].as<float>((size_t)M);
            float* dW2 = nullptr;
            float2* dXw = nullptr;
            float* dW2h = nullptr;
            void* dSh = nullptr;
            unsigned short* dPidx = ctx->ws[S_PIDX].as<unsigned short>((size_t)T * g.Kact);
            prof.begin(ROME_PHASE_SHIFT);
            phase_index_kernel<<<(unsigned)(((long)T * g.Kact + 255) / 256), 256, 0, st>>>(
                T, g.Kact, g.csF, cs, dAct, dShift, ctx->shift_sampling, dPidx);
            ROME_CHECK_LAUNCH();
            if (rtc) {
                char* buf = (char*)ctx->ws[S_A].get((size_t)P * Kh * (sizeof(float2) + sizeof(float)));
                dXw = (float2*)buf;
                dW2h = (float*)(buf + (size_t)P * Kh * sizeof(float2));
                dSh = ctx->ws[S_NORM].get((size_t)2 * restricted_tile_tn(T) * g.Kp * 2);
                restricted_prep(st, P, g.F, g.Kact, Kh, dFimg, dLctf, dMinv, apply_ctf ? 1 : 0, dAct, dXw, dW2h, dS);
                restricted_shift_operand(st, T, g.Kact, g.Kp, dPidx, ctx->d_shift_tab, ctx->precision, dSh);
            } else {
                dA = ctx->ws[S_A].get((size_t)M * g.Kp * 4);
                dW2 = ctx->ws[S_W2].as<float>((size_t)P * g.Kq);
                // cross-correlation mode: no Minvsigma2 in either operand
                const double* dMw = ccm ? nullptr : dMinv;
                shift_operand2_kernel<256><<<P, 256, 0, st>>>(P, T, g.F, g.Kact, g.Kp, dFimg, dLctf, dMw,
                                                               apply_ctf ? 1 : 0, dAct, dPidx, ctx->d_shift_tab, dA,
                                                               dS, ctx->precision, dScale);
                ROME_CHECK_LAUNCH();
                w2_kernel<<<P, 256, 0, st>>>(P, g.Kact, g.Kq, dAct, dLctf, dMw, g.F, apply_ctf ? 1 : 0, dW2, dScale);
                ROME_CHECK_LAUNCH();
            }
            prof.launched(ROME_PHASE_SHIFT, 3);
            prof.end(ROME_PHASE_SHIFT);

            unsigned* dRowMin = ctx->ws[S_ROWMIN].as<unsigned>((size_t)P);
            ROME_CUDA(cudaMemsetAsync(dRowMin, 0xFF, sizeof(unsigned) * P, st));
            const long Xrow = restricted ? (long)nprop * T : X;  // hypotheses per particle row
            float* dDiff2 = ctx->ws[S_DIFF2].as<float>((size_t)P * Xrow);
            if (!restricted) {
                float* dNorm = ctx->ws[S_NORM].as<float>((size_t)P * J);
                prof.begin(ROME_PHASE_NORM_GEMM);
                if (!tc) {
                    sgemm_tn(st, P, J, g.Kq, dW2, g.Kq, dQ, g.Kq, StoreEpi{dNorm, J});
                    ROME_CHECK_LAUNCH();
                    prof.launched(ROME_PHASE_NORM_GEMM);
                } else {
                    const int Kq64 = ((g.Kact + 63) / 64) * 64;
                    void* dW2b = ctx->ws[S_W2B].get((size_t)P * Kq64 * 4);
                    void* dQb = ctx->ws[S_QB].get((size_t)J * Kq64 * 4);
                    split_bf16(st, dW2, P, g.Kact, g.Kq, Kq64, dW2b);
                    split_bf16(st, dQ, J, g.Kact, g.Kq, Kq64, dQb);
                    tc_store_gemm(st, P, J, Kq64, dW2b, dQb, dNorm, J, ctx->d_err);
                    prof.launched(ROME_PHASE_NORM_GEMM, 3);
                }
                prof.add_flops(ROME_PHASE_NORM_GEMM, 2.0 * P * J * g.Kact);
                prof.end(ROME_PHASE_NORM_GEMM);

                Diff2Epi epi{dDiff2, dNorm, dS, dXi2, dJ, T, J, X, 1, 1, ntr, ncoarse, nullptr, dRowMin, dSx};
                prof.begin(ROME_PHASE_CROSS_GEMM);
                if (!tc) sgemm_tn(st, (int)M, J, g.Kp, (const float*)dA, g.Kp, (const float*)dB, g.Kp, epi);
                else tc_diff2_gemm(st, (int)M, J, g.Kp, dA, dB, ctx->precision, epi, ctx->d_err);
                ROME_CHECK_LAUNCH();
                prof.launched(ROME_PHASE_CROSS_GEMM);
                prof.add_flops(ROME_PHASE_CROSS_GEMM, 4.0 * (double)M * J * g.Kact);
                prof.add_bytes(ROME_PHASE_CROSS_GEMM, 4.0 * (double)M * J);  // diff2 written once
                prof.end(ROME_PHASE_CROSS_GEMM);
            } else {
                // ---- restricted coarse search: only the proposed orientations ----
                prof.begin(ROME_PHASE_RESTRICTED);
                if (rtc) {
                    restricted_tc_diff2(st, ctx->precision, P, nprop, T, g.Kp, dProp, dJ, dXw, dW2h, dB, J, dSh, dS,
                                        dXi2, Xrow, dDiff2, dRowMin, ctx->d_err);
                } else {
                    dim3 grid((nprop + RS_QQ - 1) / RS_QQ, (T + RS_TQ - 1) / RS_TQ, P);
                    if (ctx->precision == ROME_PREC_FP32)
                        restricted_diff2_kernel<ROME_PREC_FP32><<<grid, RS_THREADS, 0, st>>>(
                            T, g.Kp, g.Kq, nprop, M, J, dProp, dJ, dA, dB, dW2, dQ, dS, dXi2, Xrow, dDiff2, dRowMin);
                    else if (ctx->precision == ROME_PREC_BF16)
                        restricted_diff2_kernel<ROME_PREC_BF16><<<grid, RS_THREADS, 0, st>>>(
                            T, g.Kp, g.Kq, nprop, M, J, dProp, dJ, dA, dB, dW2, dQ, dS, dXi2, Xrow, dDiff2, dRowMin);
                    else
                        restricted_diff2_kernel<ROME_PREC_BF16X3><<<grid, RS_THREADS, 0, st>>>(
                            T, g.Kp, g.Kq, nprop, M, J, dProp, dJ, dA, dB, dW2, dQ, dS, dXi2, Xrow, dDiff2, dRowMin);
                    ROME_CHECK_LAUNCH();
                }
                prof.launched(ROME_PHASE_RESTRICTED);
                prof.add_flops(ROME_PHASE_RESTRICTED, 4.0 * (double)P * Xrow * g.Kact);
                prof.end(ROME_PHASE_RESTRICTED);
            }

            // posterior, walk, coarse-significant points
            PostLayout Lp{T, 1, 1, npsi, ntr, K};
            Lp.ndir = ndir;
            Lp.list_zeros = 1;
            if (restricted) {
                // ragged rows: the prior of row position q * T + t comes from proposal q
                int2* dEnt = ctx->ws[S_FENT].as<int2>((size_t)P * nprop);
                restricted_entries_kernel<<<(unsigned)(((long)P * nprop + 255) / 256), 256, 0, st>>>(
                    (long)P * nprop, npsi, dProp, dEnt);
                ROME_CHECK_LAUNCH();
                Lp.ent = dEnt;
                Lp.ent_stride = nprop;
                Lp.epr = T;
            }
            int* dCounter = ctx->ws[S_LISTCNT].as<int>(4);
            int listcap = std::max(1024, P * 64), nsig = 0;
            SigEntry* dList = nullptr;
            prof.begin(ROME_PHASE_POSTERIOR);
            prof.add_bytes(ROME_PHASE_POSTERIOR, 4.0 * (double)P * Xrow);  // diff2 read once
            for (;;) {
                dList = ctx->ws[S_SIGLIST].as<SigEntry>((size_t)listcap);
                SelectResult sr = ccm ? run_select_cc(st, P, Xrow, Lp, dDiff2, dPart, dPartI, nullptr, dList,
                                                      dCounter, listcap, dSeg)
                                      : run_select(ctx, st, 0, P, Xrow, Lp, dDiff2, dPdir, dPoff, in->adaptive_fraction,
                                                   dPart, dPartI, nullptr, nullptr, dList, dCounter, listcap, dSeg,
                                                   dRowMin);
                prof.launched(ROME_PHASE_POSTERIOR, sr.launches);
                nsig = sr.nlist;
                if (sr.nlist <= listcap) break;
                listcap = sr.nlist;
            }
            if (restricted && nsig > 0) {
                // row position q * T + t -> dense coarse hypothesis j * T + t
                restricted_list_dense_kernel<<<(nsig + 255) / 256, 256, 0, st>>>(nsig, T, nprop, dProp, dList);
                ROME_CHECK_LAUNCH();
            }
            if (out->post_coarse) {
                double* dMarg = ctx->ws[S_TMP2].as<double>((size_t)P * J);
                ROME_CUDA(cudaMemsetAsync(dMarg, 0, sizeof(double) * P * J, st));
                if (nsig > 0) {
                    post_marginal_kernel<<<(nsig + 255) / 256, 256, 0, st>>>(nsig, T, 1, J, dList, dMarg);
                    ROME_CHECK_LAUNCH();
                }
                ROME_CUDA(cudaMemcpyAsync(out->post_coarse, dMarg, sizeof(double) * P * J, cudaMemcpyDeviceToHost,
                                          st));
            }
            nsig0 = nsig;
            dList0 = dList;
            ROME_CUDA(cudaMemsetAsync(dMcoarse, 0, (size_t)P * ncoarse, st));
            if (nsig > 0) {
                mcoarse_from_list_kernel<<<(nsig + 255) / 256, 256, 0, st>>>(nsig, X, dList, dMcoarse);
                ROME_CHECK_LAUNCH();
                prof.launched(ROME_PHASE_POSTERIOR);
            }
            prof.end(ROME_PHASE_POSTERIOR);
            if (tc) tc_check_error(st, ctx->d_err);

            ROME_CUDA(cudaMemcpyAsync(hpart.data(), dPart, sizeof(double) * P * 8, cudaMemcpyDeviceToHost, st));
            ROME_CUDA(cudaMemcpyAsync(hparti.data(), dPartI, sizeof(int) * P * 8, cudaMemcpyDeviceToHost, st));
            if (out->coarse_diff2) {
                std::vector<float> hd((size_t)P * X);
                ROME_CUDA(cudaMemcpyAsync(hd.data(), dDiff2, sizeof(float) * hd.size(), cudaMemcpyDeviceToHost, st));
                ROME_CUDA(cudaStreamSynchronize(st));
                for (size_t q = 0; q < hd.size(); q++)
                    out->coarse_diff2[q] = hd[q] < INFINITY ? (double)hd[q] : (double)INT_MIN;
            }
            if (out->Mcoarse_significant)
                ROME_CUDA(cudaMemcpyAsync(out->Mcoarse_significant, dMcoarse, (size_t)P * ncoarse,
                                          cudaMemcpyDeviceToHost, st));
            ROME_CUDA(cudaStreamSynchronize(st));
            for (int i = 0; i < P; i++) {
                h_min[i] = hpart[i * 8 + 0];
                h_sum[i] = hpart[i * 8 + 1];
                h_sig[i] = hpart[i * 8 + 2];
                h_nsig[i] = hparti[i * 8 + 1];
                if (h_nsig[i] == 0) fail(ROME_ERR_NUMERIC, "my_nr_significant_coarse_samples == 0 for particle %d", i);
                if (out->pass_min_diff2[0]) out->pass_min_diff2[0][i] = h_min[i];
                if (out->pass_sum_weight[0]) out->pass_sum_weight[0][i] = h_sum[i];
                if (out->pass_significant_weight[0]) out->pass_significant_weight[0][i] = h_sig[i];
            }
        }

        // ================= pass 1: fine, over the coarse-significant points =================
        std::vector<int> act, actidx;
        const Pass g = active_pixels(cur, ctx->r_max, act, actidx);
        const int Tf = ntr * NOTR;
        int* dAct = upload3(ctx, S_ACT, act.data(), act.size());
        int* dActIdx = upload3(ctx, S_ACTIDX, actidx.data(), actidx.size());
        int* dMresF = upload3(ctx, S_MRES, in->Mresol_fine, (size_t)g.F);

        // orientations some particle needs (getReferenceAllOrientations, :956-985)
        char* dRotSig = ctx->ws[S_ROTSIG].as<char>((size_t)Jc);
        ROME_CUDA(cudaMemsetAsync(dRotSig, 0, (size_t)Jc, st));
        if (nsig0 > 0) {
            rotsig_from_list_kernel<<<(nsig0 + 255) / 256, 256, 0, st>>>(nsig0, ntr, dList0, dRotSig);
            ROME_CHECK_LAUNCH();
            prof.launched(ROME_PHASE_PROJECT);
        }
        std::vector<char> hrs(Jc);
        ROME_CUDA(cudaMemcpyAsync(hrs.data(), dRotSig, Jc, cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaStreamSynchronize(st));
        std::vector<int> uj, ucompact(Jc, -1);
        for (int jc = 0; jc < Jc; jc++)
            if (hrs[jc] && hcd_ok[jc / npsi]) {
                ucompact[jc] = (int)uj.size();
                uj.push_back(jc);
            }
        const int nU = (int)uj.size(), Jf = nU * NOR;
        ROME_REQUIRE(nU > 0, "no significant coarse orientation");
        {
            // the fine projections of the pool live on the device together (FP64 slice, |P|^2 and operand
            // rows per fine orientation): refuse pools whose union of significant orientations would not fit
            std::vector<int> a2, ai2;
            const Pass gf = active_pixels(cur, ctx->r_max, a2, ai2);
            const double nb[3] = {(double)nU * NOR * gf.Kact * 16, (double)nU * NOR * gf.Kq * 4,
                                  (double)nU * NOR * gf.Kp * 4};
            const Slot sl[3] = {S_PROJ, S_Q, S_B};
            double need = 0.0, held = 0.0;
            bool grows = false;
            for (int q = 0; q < 3; q++) {
                need += nb[q];
                held += (double)ctx->ws[sl[q]].bytes;
                grows |= nb[q] > (double)ctx->ws[sl[q]].bytes;
            }
            if (grows) {  // only a pool that enlarges the buffers can run out (they are freed, then reallocated)
                size_t free_b = 0, total_b = 0;
                ROME_CUDA(cudaMemGetInfo(&free_b, &total_b));
                if (need > 0.8 * ((double)free_b + held))
                    fail(ROME_ERR_OOM, "fine pass: %d significant coarse orientations need %.1f GB of projections "
                         "(%.1f GB free); use smaller pools", nU, need / 1e9, ((double)free_b + held) / 1e9);
            }
        }
        int* dUcomp = upload3(ctx, S_TMP2, ucompact.data(), ucompact.size());
        std::vector<int> hjf((size_t)2 * Jf);  // jclass, jcd
        std::vector<Rot3> hrotf(Jf);
        for (int u = 0; u < nU; u++) {
            const int jc = uj[u], cd = jc / npsi, dp = jc % (ndir * npsi);
            for (int o = 0; o < NOR; o++) {
                const int jf = u * NOR + o;
                hjf[jf] = cd / ndir;
                hjf[Jf + jf] = cd;
                const double* a = in->angles[1] + ((size_t)dp * NOR + o) * 3;
                hrotf[jf] = rot3_inv(a[0], a[1], a[2], ctx->padding);
            }
        }
        int* dJf = upload3(ctx, S_JVALID, hjf.data(), hjf.size());
        Rot3* dRotF = upload3(ctx, S_ROTM, hrotf.data(), hrotf.size());
        std::vector<double2> hsh(Tf), htr(Tf);
        for (int t = 0; t < Tf; t++) {
            hsh[t] = make_double2(in->over_trans_x[1][t] / (-ori), in->over_trans_y[1][t] / (-ori));
            htr[t] = make_double2(in->over_trans_x[1][t], in->over_trans_y[1][t]);
        }
        double2* dShift = upload3(ctx, S_SHIFT, hsh.data(), hsh.size());
        double2* dTr = upload3(ctx, S_TRANS, htr.data(), htr.size());
        double2* dPh = ctx->ws[S_PHASE].as<double2>((size_t)Tf * g.F);
        prof.begin(ROME_PHASE_SHIFT);
        phase_table_kernel<<<(unsigned)(((long)Tf * g.F + 255) / 256), 256, 0, st>>>(
            Tf, g.F, g.csF, cur, dShift, ctx->d_shift_tab, ctx->shift_sampling, dPh);
        ROME_CHECK_LAUNCH();
        prof.launched(ROME_PHASE_SHIFT);
        prof.end(ROME_PHASE_SHIFT);

        double2* dFimg = ctx->ws[S_FIMG].as<double2>((size_t)P * g.F);
        double* dLctf = ctx->ws[S_CTF].as<double>((size_t)P * g.F);
        double* dMinv = ctx->ws[S_MINV].as<double>((size_t)P * g.F);
        prof.begin(ROME_PHASE_PREP);
        prep_particles_kernel<<<P, 256, 0, st>>>(P, cur, cur, dFr, dFi, dCtf, dMresF, dSig2, dGroup, oriF,
                                                  in->sigma2_fudge, dFimg, dLctf, dMinv);
        ROME_CHECK_LAUNCH();
        prof.launched(ROME_PHASE_PREP);
        double* dSx = nullptr;
        if (ccm) {
            dSx = ctx->ws[S_CCX].as<double>((size_t)P);
            sqrt_xi2_kernel<<<P, 256, 0, st>>>(g.F, dFimg, dSx);
            ROME_CHECK_LAUNCH();
            prof.launched(ROME_PHASE_PREP);
        }
        const double* dMw = ccm ? nullptr : dMinv;  // operands without Minvsigma2 in cross-correlation mode
        prof.end(ROME_PHASE_PREP);

        // fine projections: FP64 for wsum/backprojection, FP32 operands for diff2
        double2* dProj = ctx->ws[S_PROJ].as<double2>((size_t)Jf * g.Kact);
        float* dQ = ctx->ws[S_Q].as<float>((size_t)Jf * g.Kq);
        float* dB = ctx->ws[S_B].as<float>((size_t)Jf * g.Kp);
        prof.begin(ROME_PHASE_PROJECT);
        project3d_kernel<<<Jf, 128, 0, st>>>(Jf, g.Kact, g.Kp, g.Kq, cur, g.csF, g.my_r_max, ctx->pad_size,
                                              ctx->pad_size / 2 + 1, dJf, ctx->proj, ctx->vox, dRotF, dAct, nullptr,
                                              dProj, dQ, dB, ROME_PREC_FP32);
        ROME_CHECK_LAUNCH();
        prof.launched(ROME_PHASE_PROJECT);
        // algorithmic bytes: the class volumes read once, FP64 projections, |P|^2 and FP32 operand written
        prof.add_bytes(ROME_PHASE_PROJECT, (double)K * ctx->vox * 16 +
                                               (double)Jf * ((double)g.Kact * 16 + (double)g.Kq * 4 + (double)g.Kp * 4));
        prof.end(ROME_PHASE_PROJECT);

        float* dW2 = ctx->ws[S_W2].as<float>((size_t)P * g.Kq);
        unsigned short* dPidx = ctx->ws[S_PIDX].as<unsigned short>((size_t)Tf * g.Kact);
        prof.begin(ROME_PHASE_SHIFT);
        phase_index_kernel<<<(unsigned)(((long)Tf * g.Kact + 255) / 256), 256, 0, st>>>(
            Tf, g.Kact, g.csF, cur, dAct, dShift, ctx->shift_sampling, dPidx);
        ROME_CHECK_LAUNCH();
        w2_kernel<<<P, 256, 0, st>>>(P, g.Kact, g.Kq, dAct, dLctf, dMw, g.F, apply_ctf ? 1 : 0, dW2, dScale);
        ROME_CHECK_LAUNCH();
        prof.launched(ROME_PHASE_SHIFT, 2);
        prof.end(ROME_PHASE_SHIFT);

        // compaction of the coarse-significant points
        int* dCnt = ctx->ws[S_OFFJ].as<int>((size_t)2 * P + 2);
        int* dOffP = dCnt + P;
        mcoarse_count_kernel<<<P, 256, 0, st>>>(ncoarse, dMcoarse, dCnt);
        ROME_CHECK_LAUNCH();
        std::vector<int> hcnt(P), hoffp(P + 1);
        ROME_CUDA(cudaMemcpyAsync(hcnt.data(), dCnt, sizeof(int) * P, cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaStreamSynchronize(st));
        int stride = 1;
        hoffp[0] = 0;
        for (int i = 0; i < P; i++) {
            hoffp[i + 1] = hoffp[i] + hcnt[i];
            stride = std::max(stride, hcnt[i]);
        }
        const int E = hoffp[P];
        stage_copy(ctx, dOffP, hoffp.data(), (size_t)P + 1);
        int4* dFe = ctx->ws[S_FE].as<int4>((size_t)std::max(E, 1));
        int2* dEnt = ctx->ws[S_FENT].as<int2>((size_t)std::max(E, 1));
        fine_entries_kernel<<<P, FE_THREADS, 0, st>>>(ncoarse, ntr, npsi, dMcoarse, dOffP, dUcomp, dFe, dEnt);
        ROME_CHECK_LAUNCH();
        prof.launched(ROME_PHASE_PROJECT, 2);

        // shifted images of the (particle, coarse translation) pairs the points need, NOTR rows each
        const int NPT = P * ntr;
        int* dPairFlag = ctx->ws[S_PAIRS].as<int>((size_t)3 * NPT + 2);
        int* dPairId = dPairFlag + NPT;       // exclusive scan of the flags, [NPT + 1] (last: the count)
        int* dPairOf = dPairId + NPT + 1;     // pair -> particle * ntr + coarse translation
        const int pair_cap = std::max(1, std::min(E, NPT));
        float* dA = ctx->ws[S_A].as<float>((size_t)pair_cap * NOTR * g.Kp);
        float* dS = ctx->ws[S_S].as<float>((size_t)pair_cap * NOTR);
        prof.begin(ROME_PHASE_SHIFT);
        ROME_CUDA(cudaMemsetAsync(dPairFlag, 0, sizeof(int) * NPT, st));
        if (E > 0) {
            fine_pair_flag_kernel<<<(E + 255) / 256, 256, 0, st>>>(E, ntr, dFe, dPairFlag);
            ROME_CHECK_LAUNCH();
        }
        exclusive_scan_kernel<<<1, 1024, 0, st>>>(NPT, dPairFlag, dPairId);
        ROME_CHECK_LAUNCH();
        fine_pair_list_kernel<<<(NPT + 255) / 256, 256, 0, st>>>(NPT, dPairFlag, dPairId, dPairOf);
        ROME_CHECK_LAUNCH();
        fine_pair_operand_kernel<256><<<pair_cap, 256, 0, st>>>(dPairId + NPT, dPairOf, ntr, NOTR, g.F, g.Kact, g.Kp,
                                                                dFimg, dLctf, dMw, apply_ctf ? 1 : 0, dAct, dPidx,
                                                                ctx->d_shift_tab, dA, dS, dScale);
        ROME_CHECK_LAUNCH();
        prof.launched(ROME_PHASE_SHIFT, 4);
        prof.add_bytes(ROME_PHASE_SHIFT, 4.0 * pair_cap * NOTR * g.Kp);
        prof.end(ROME_PHASE_SHIFT);

        // fine squared differences in ragged rows without padding: particle i's row is points
        // off[i] .. off[i + 1] - 1, NH sub-hypotheses each (every entry is written by the kernel);
        // Xf, the longest row, sizes the selection's scratch
        const long Xf = (long)stride * NH;
        float* dDiff2 = ctx->ws[S_DIFF2].as<float>((size_t)std::max(E, 1) * NH);
        unsigned* dRowMin = ctx->ws[S_ROWMIN].as<unsigned>((size_t)P);
        prof.begin(ROME_PHASE_CROSS_GEMM);
        ROME_CUDA(cudaMemsetAsync(dRowMin, 0xFF, sizeof(unsigned) * P, st));
        if (E > 0) {
            fine_diff2_kernel<128, 8, 4><<<E, 128, 0, st>>>(ntr, g.Kp, g.Kq, dFe, dPairId, dA, dB, dW2, dQ, dS, dXi2,
                                                          dDiff2, dRowMin, dSx);
            ROME_CHECK_LAUNCH();
        }
        if (E > 0) prof.launched(ROME_PHASE_CROSS_GEMM);
        prof.add_flops(ROME_PHASE_CROSS_GEMM, 4.0 * (double)E * NH * g.Kact);
        prof.end(ROME_PHASE_CROSS_GEMM);

        // posterior over the ragged rows
        PostLayout Lf{Tf, NOTR, NOR, npsi, ntr, K};
        Lf.ndir = ndir;
        Lf.ent = dEnt;
        Lf.ent_stride = stride;
        Lf.roff = dOffP;
        Lf.epr = NH;
        Lf.list_zeros = 1;
        double* dW = nullptr;
        if (out->fine_weight) dW = ctx->ws[S_WCHK].as<double>((size_t)std::max(E, 1) * NH);
        int* dCounter = ctx->ws[S_LISTCNT].as<int>((size_t)Jf + 4);
        int listcap = std::max(1024, P * 64), nsig = 0;
        SigEntry* dList = nullptr;
        prof.begin(ROME_PHASE_POSTERIOR);
        prof.add_bytes(ROME_PHASE_POSTERIOR, 4.0 * (double)E * NH);  // diff2 rows read once
        for (;;) {
            dList = ctx->ws[S_SIGLIST].as<SigEntry>((size_t)listcap * 2);
            SelectResult sr = ccm ? run_select_cc(st, P, Xf, Lf, dDiff2, dPart, dPartI, dW, dList, dCounter, listcap,
                                                  dSeg)
                                  : run_select(ctx, st, 0, P, Xf, Lf, dDiff2, dPdir, dPoff, in->adaptive_fraction,
                                               dPart, dPartI, nullptr, dW, dList, dCounter, listcap, dSeg, dRowMin);
            prof.launched(ROME_PHASE_POSTERIOR, sr.launches);
            nsig = sr.nlist;
            if (sr.nlist <= listcap) break;
            listcap = sr.nlist;
        }
        if (nsig > 0) {
            fine_list_dense_kernel<<<(nsig + 255) / 256, 256, 0, st>>>(nsig, NOR, NOTR, Tf, stride, dFe, dOffP, dList);
            ROME_CHECK_LAUNCH();
            prof.launched(ROME_PHASE_POSTERIOR);
        }
        prof.end(ROME_PHASE_POSTERIOR);

        ROME_CUDA(cudaMemcpyAsync(hpart.data(), dPart, sizeof(double) * P * 8, cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaMemcpyAsync(hparti.data(), dPartI, sizeof(int) * P * 8, cudaMemcpyDeviceToHost, st));
        std::vector<int4> hfe(std::max(E, 1));
        if (E > 0) ROME_CUDA(cudaMemcpyAsync(hfe.data(), dFe, sizeof(int4) * E, cudaMemcpyDeviceToHost, st));
        std::vector<float> hd;
        std::vector<double> hw;
        if (out->fine_count || out->fine_index || out->fine_diff2 || out->fine_weight) {
            hd.resize((size_t)std::max(E, 1) * NH);
            ROME_CUDA(cudaMemcpyAsync(hd.data(), dDiff2, sizeof(float) * hd.size(), cudaMemcpyDeviceToHost, st));
            if (dW) {
                hw.resize((size_t)std::max(E, 1) * NH);
                ROME_CUDA(cudaMemcpyAsync(hw.data(), dW, sizeof(double) * hw.size(), cudaMemcpyDeviceToHost, st));
            }
        }
        ROME_CUDA(cudaStreamSynchronize(st));
        if (!hd.empty()) {
            long q = 0;
            for (int i = 0; i < P; i++) {
                const int n = hcnt[i] * NH;
                if (out->fine_count) out->fine_count[i] = n;
                for (int e = 0; e < n; e++, q++) {
                    if (q >= out->fine_capacity) fail(ROME_ERR_ARG, "fine_capacity %ld too small", out->fine_capacity);
                    const int4 en = hfe[hoffp[i] + e / NH];
                    const long jc = uj[en.z];
                    if (out->fine_index) out->fine_index[q] = ((jc * ntr + en.w) * NH) + e % NH;
                    const size_t at = (size_t)hoffp[i] * NH + e;
                    if (out->fine_diff2) out->fine_diff2[q] = (double)hd[at];
                    if (out->fine_weight) out->fine_weight[q] = hw.empty() ? 0.0 : hw[at];
                }
            }
        }
        for (int i = 0; i < P; i++) {
            const double mn = hpart[i * 8 + 0], sw = hpart[i * 8 + 1], sig = hpart[i * 8 + 2], mx = hpart[i * 8 + 4];
            const int best = hparti[i * 8 + 0];
            h_min[i] = mn;
            h_sum[i] = sw;
            h_sig[i] = sig;
            if (out->pass_min_diff2[1]) out->pass_min_diff2[1][i] = mn;
            if (out->pass_sum_weight[1]) out->pass_sum_weight[1][i] = sw;
            if (out->pass_significant_weight[1]) out->pass_significant_weight[1][i] = sig;
            // convertSquaredDifferencesToWeights metadata (map3d_optimizer.cpp:1787-1804)
            const int r = best / NH, h = best % NH, o = h / NOTR, t = h % NOTR;
            if (hcnt[i] == 0 || r >= hcnt[i]) continue;
            const int4 en = hfe[hoffp[i] + r];
            const int jc = uj[en.z], cd = jc / npsi, dp = jc % (ndir * npsi);
            const double* a = in->angles[1] + ((size_t)dp * NOR + o) * 3;
            if (out->pmax) out->pmax[i] = mx / sw;
            if (out->cls) out->cls[i] = cd / ndir + 1;
            if (out->rot) out->rot[i] = a[0];
            if (out->tilt) out->tilt[i] = a[1];
            if (out->psi) out->psi[i] = a[2];
            if (out->xoff) out->xoff[i] = in->old_offsetx[i] + in->over_trans_x[1][en.w * NOTR + t];
            if (out->yoff) out->yoff[i] = in->old_offsety[i] + in->over_trans_y[1][en.w * NOTR + t];
        }

        // ---- updateOtherParams ----
        double* dWsn = ctx->ws[S_WSN].as<double>((size_t)G * oriF + P);
        double* dNormCorr = dWsn + (size_t)G * oriF;
        const int nwk = K + KD + 1 + G;
        double* dWk = ctx->ws[S_WSUMK].as<double>((size_t)nwk);
        ROME_CUDA(cudaMemsetAsync(dWsn, 0, sizeof(double) * ((size_t)G * oriF + P), st));
        ROME_CUDA(cudaMemsetAsync(dWk, 0, sizeof(double) * nwk, st));
        const int NT = 256, PIX = 8;
        const int nsplit = (g.F + NT * PIX - 1) / (NT * PIX);
        prof.begin(ROME_PHASE_WSUM);
        ROME_REQUIRE(P <= 65535, "pool of %d particles: at most 65,535", P);
        // the longest list segment sets the number of entry chunks (grid z) of the wsum kernel
        std::vector<int> hseg((size_t)2 * P);
        ROME_CUDA(cudaMemcpyAsync(hseg.data(), dSeg, sizeof(int) * 2 * P, cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaStreamSynchronize(st));
        int maxseg = 1;
        for (int i = 0; i < P; i++) maxseg = std::max(maxseg, hseg[(size_t)2 * i + 1]);
        const int WCH = 256;
        const int nzch = std::min(65535, (maxseg + WCH - 1) / WCH);
        const int wchunk = (maxseg + nzch - 1) / nzch;
        if (scl)
            wsum3d_list_kernel<NT, PIX, true><<<dim3(nsplit, P, nzch), NT, 0, st>>>(
                Tf, K, ndir, g.F, g.csF, cur, oriF, dList, dSeg, dJf + Jf, dFimg, dLctf, apply_ctf ? 1 : 0, dProj,
                dActIdx, g.Kact, dShift, dPh, dMresF, dGroup, dOld, dTr, dPriorX, dPriorY, dWsn, dNormCorr, dWk, wchunk,
                ssum);
        else
            wsum3d_list_kernel<NT, PIX, false><<<dim3(nsplit, P, nzch), NT, 0, st>>>(
                Tf, K, ndir, g.F, g.csF, cur, oriF, dList, dSeg, dJf + Jf, dFimg, dLctf, apply_ctf ? 1 : 0, dProj,
                dActIdx, g.Kact, dShift, dPh, dMresF, dGroup, dOld, dTr, dPriorX, dPriorY, dWsn, dNormCorr, dWk, wchunk,
                ssum);
        ROME_CHECK_LAUNCH();
        prof.launched(ROME_PHASE_WSUM);
        prof.end(ROME_PHASE_WSUM);

        // ---- backProjection ----
        std::vector<int> hoff_bp;  // list offsets per fine orientation (profiling: slices back-projected)
        {
            double2* dFnm = ctx->ws[S_FNOMASK].as<double2>((size_t)P * g.F);
            double* dMctf2 = dMinv;  // becomes ctf^2 * Minvsigma2 in place
            prof.begin(ROME_PHASE_BACKPROJECT);
            bp_prep_kernel<<<P, 256, 0, st>>>(P, g.F, dFnr, dFni, dLctf, dMinv, dSig2, dGroup, oriF, in->sigma2_fudge,
                                              in->do_map, in->do_ctf_correction, dFnm, dMctf2, nullptr, dScale);
            ROME_CHECK_LAUNCH();
            int* dJcnt = dCounter + 2;
            int* dJoff = ctx->ws[S_REC_SMALL].as<int>((size_t)2 * Jf + 2);
            int* dFill = dJoff + Jf + 1;
            SigEntry* dSorted = dList + listcap;
            ROME_CUDA(cudaMemsetAsync(dJcnt, 0, sizeof(int) * Jf, st));
            ROME_CUDA(cudaMemsetAsync(dFill, 0, sizeof(int) * Jf, st));
            if (nsig > 0) {
                count_by_j_kernel<<<(nsig + 255) / 256, 256, 0, st>>>(nsig, Tf, dList, dJcnt);
                ROME_CHECK_LAUNCH();
            }
            exclusive_scan_kernel<<<1, 1024, 0, st>>>(Jf, dJcnt, dJoff);
            ROME_CHECK_LAUNCH();
            if (nsig > 0) {
                scatter_by_j_kernel<<<(nsig + 255) / 256, 256, 0, st>>>(nsig, Tf, dList, dJoff, dFill, dSorted);
                ROME_CHECK_LAUNCH();
            }
            for (int j0 = 0; j0 < Jf; j0 += 65535) {  // grid y limit
                bp3d_list_kernel<NT, PIX><<<dim3(nsplit, std::min(Jf - j0, 65535)), NT, 0, st>>>(
                    Tf, g.F, g.csF, cur, dSorted, dJoff, dJf, dFnm, dMctf2, dShift, dPh, dRotF, ctx->r_max,
                    ctx->pad_size, ctx->pad_size / 2 + 1, ctx->bp_data, ctx->bp_weight, ctx->vox, j0);
                ROME_CHECK_LAUNCH();
            }
            prof.launched(ROME_PHASE_BACKPROJECT, 5);
            prof.end(ROME_PHASE_BACKPROJECT);
            if (ctx->profile) {
                hoff_bp.resize((size_t)Jf + 1);
                ROME_CUDA(cudaMemcpyAsync(hoff_bp.data(), dJoff, sizeof(int) * (Jf + 1), cudaMemcpyDeviceToHost, st));
            }
        }

        // ---- outputs ----
        std::vector<double> hwsn((size_t)G * oriF + P), hwk(nwk);
        ROME_CUDA(cudaMemcpyAsync(hwsn.data(), dWsn, sizeof(double) * hwsn.size(), cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaMemcpyAsync(hwk.data(), dWk, sizeof(double) * hwk.size(), cudaMemcpyDeviceToHost, st));
        if (scl && out->wsum_scale_correction_XA)
            ROME_CUDA(cudaMemcpyAsync(out->wsum_scale_correction_XA, ssum.xa, sizeof(double) * P * oriF,
                                      cudaMemcpyDeviceToHost, st));
        if (scl && out->wsum_scale_correction_AA)
            ROME_CUDA(cudaMemcpyAsync(out->wsum_scale_correction_AA, ssum.aa, sizeof(double) * P * oriF,
                                      cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaStreamSynchronize(st));
        prof.collect();
        if (!hoff_bp.empty()) {
            // algorithmic bytes of the back-projection: the prepared image and ctf^2 Minvsigma2 of every
            // significant hypothesis (24 B per active pixel) and 24 FP64 updates (192 B) per active pixel of
            // every back-projected slice (fine orientation with significant hypotheses)
            long nslice = 0;
            for (int j = 0; j + 1 < (int)hoff_bp.size(); j++) nslice += hoff_bp[j + 1] > hoff_bp[j];
            prof.add_bytes(ROME_PHASE_BACKPROJECT, (double)g.Kact * (24.0 * nsig + 192.0 * nslice));
        }
        for (size_t q = 0; q < (size_t)G * oriF; q++) out->wsum_sigma2_noise[q] += hwsn[q];
        for (int i = 0; i < P; i++) {
            if (out->wsum_norm_correction) out->wsum_norm_correction[i] = hwsn[(size_t)G * oriF + i];
            if (out->min_diff2) out->min_diff2[i] = h_min[i];
            if (out->sum_weight) out->sum_weight[i] = h_sum[i];
            if (out->significant_weight) out->significant_weight[i] = h_sig[i];
            if (out->nr_sign) out->nr_sign[i] = h_nsig[i];
        }
        for (int k = 0; k < K; k++) out->wsum_pdf_class[k] += hwk[k];
        for (int q = 0; q < KD; q++) out->wsum_pdf_direction[q] += hwk[K + q];
        out->wsum_sigma2_offset[0] += hwk[K + KD];
        for (int q = 0; q < G; q++) out->wsum_sumw_group[q] += hwk[K + KD + 1 + q];
        for (int i = 0; i < P; i++)
            if (h_sum[i] == 0) fail(ROME_ERR_NUMERIC, "exp_sum_weight[%d] == 0", i);
    });
}

extern "C" int rome_gpu_backproject_images(RomeGpuCtx* ctx, int iclass, int n, int size, const double* Fimg_real,
                                           const double* Fimg_imag, const double* Fctf, const double* poses,
                                           int inputs_on_device) {
    if (!ctx) return ROME_ERR_ARG;
    return guarded(ctx, [&] {
        if (!ctx->bp_data || ctx->ref_dim != 3) fail(ROME_ERR_STATE, "3D back-projectors not set (rome_gpu_set_projectors)");
        ROME_REQUIRE(iclass >= 0 && iclass < ctx->nr_classes, "iclass %d out of range", iclass);
        ROME_REQUIRE(n >= 0 && Fimg_real && Fimg_imag && poses, "bad back-projection args");
        ROME_REQUIRE(size == ctx->ori_size, "image size %d differs from the back-projector's %d", size,
                     ctx->ori_size);
        if (n == 0) return;
        ROME_CUDA(cudaSetDevice(ctx->device));
        arena_reset(ctx);
        cudaStream_t st = ctx->stream;
        const int csF = size / 2 + 1, F = size * csF;
        const int r_max = std::min(ctx->r_max, size / 2);
        std::vector<Rot3> hrot(n);
        std::vector<double2> hsh(n);
        std::vector<double> key(n);
        const double d2r = 3.14159265358979323846 / 180.;
        for (int i = 0; i < n; i++) {
            const double* a = poses + 5 * (size_t)i;
            for (int q = 0; q < 5; q++)
                ROME_REQUIRE(std::isfinite(a[q]), "pose %d field %d is not finite", i, q);
            hrot[i] = rot3_inv(a[0], a[1], a[2], ctx->padding);
            hsh[i] = make_double2(a[3] / (-size), a[4] / (-size));
            // the slice's plane is set by its normal, the projection direction
            // (sin tilt cos rot, sin tilt sin rot, cos tilt), up to sign
            // (Friedel); order images along serpentine bands of the polar angle
            // of the upper-hemisphere normal so concurrent blocks share voxels
            double nx = sin(a[1] * d2r) * cos(a[0] * d2r), ny = sin(a[1] * d2r) * sin(a[0] * d2r);
            double nz = cos(a[1] * d2r);
            if (nz < 0) {
                nx = -nx;
                ny = -ny;
                nz = -nz;
            }
            const double theta = acos(std::min(1.0, nz)) / d2r, phi = atan2(ny, nx);
            const int band = std::min(29, (int)(theta / 3.0));
            key[i] = band * 16.0 + ((band & 1) ? -phi : phi);
        }
        std::vector<int> ord(n);
        for (int i = 0; i < n; i++) ord[i] = i;
        std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return key[x] < key[y]; });
        Rot3* dRot = upload3(ctx, S_ROTM, hrot.data(), hrot.size());
        double2* dSh = upload3(ctx, S_SHIFT, hsh.data(), hsh.size());
        int* dOrd = upload3(ctx, S_PARTI, ord.data(), ord.size());
        const double *dRe = Fimg_real, *dIm = Fimg_imag, *dCtf = Fctf;
        if (!inputs_on_device) {
            double* buf = ctx->ws[S_FNOMASK].as<double>((size_t)2 * n * F);
            ROME_CUDA(cudaMemcpyAsync(buf, Fimg_real, sizeof(double) * n * F, cudaMemcpyHostToDevice, st));
            ROME_CUDA(cudaMemcpyAsync(buf + (size_t)n * F, Fimg_imag, sizeof(double) * n * F, cudaMemcpyHostToDevice,
                                      st));
            dRe = buf;
            dIm = buf + (size_t)n * F;
            if (Fctf) {
                double* c = ctx->ws[S_CTF].as<double>((size_t)n * F);
                ROME_CUDA(cudaMemcpyAsync(c, Fctf, sizeof(double) * n * F, cudaMemcpyHostToDevice, st));
                dCtf = c;
            }
        }
        const int NT = 256, PIX = 4;
        const int nsplit = (F + NT * PIX - 1) / (NT * PIX);
        Profiler prof(ctx);
        prof.begin(ROME_PHASE_BACKPROJECT);
        for (int i0 = 0; i0 < n; i0 += 65535) {  // grid y limit
            const int m = std::min(n - i0, 65535);
            bp_images_kernel<NT, PIX><<<dim3(nsplit, m), NT, 0, st>>>(
                F, csF, size, dOrd + i0, dRe, dIm, dCtf, dSh, ctx->d_shift_tab, ctx->shift_sampling, dRot, r_max,
                ctx->pad_size, ctx->pad_size / 2 + 1, ctx->bp_data + (long)iclass * ctx->vox,
                ctx->bp_weight + (long)iclass * ctx->vox);
            ROME_CHECK_LAUNCH();
            prof.launched(ROME_PHASE_BACKPROJECT);
        }
        prof.end(ROME_PHASE_BACKPROJECT);
        prof.add_bytes(ROME_PHASE_BACKPROJECT, (double)n * F * (Fctf ? 24.0 : 16.0));  // spectra (+ CTF) read once
        ROME_CUDA(cudaStreamSynchronize(st));
        prof.collect();
    });
}
