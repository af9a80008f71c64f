// MAP2D E-step for one pool of particles on sm_100a.
//
// Replaces Map2dOptimizer_old::expectationSomeParticles
// (src/map2d_optimizer.cpp:802-854) minus storeWeightedSums.  Per pass:
//   prep      windowed image / CTF / Minvsigma2    (exp_model.cpp:935-1104)
//   project   rotate2D of every class x psi         (reconstruct.cpp:823-958)
//   shift     table-based phase shift + A operand   (image.h:1478-1575)
//   diff2     cross term as a dense contraction, fused epilogue
//             diff2 = (N_ij - 2 C_(it)j + S_it + highres_Xi2_i) / 2
//                                                  (map2d_optimizer.cpp:907-1074)
//   posterior FP64 weights, sum, argmax, significance selection
//                                                  (map2d_optimizer.cpp:1077-1311)
// then updateOtherParams (wsum kernel, :1417-1663) and backProjection
// (slice accumulation + backrotate2D scatter, :1666-1873,
// reconstruct.cpp:1353-1500).
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>
#include <algorithm>
#include <mutex>
#include <string>

#include "common.cuh"
#include "estep_kernels.cuh"
#include "gemm_simt.cuh"
#include "gemm_tc.cuh"
#include "restricted_kernels.cuh"
#include "restricted_tc.cuh"
#include "select_kernels.cuh"

using namespace rome;

namespace rome {
namespace {

struct PassGeom {
    int cs, F, csF;          // image size of the pass, half-plane pixels, row length
    int nor, notr, T, nrot;  // over-rotations, over-translations, T = ntr*notr, nrot = npsi*nor
    int J;                   // orientations K*nrot
    long X;                  // hypotheses per particle J*T
    int Kact, Kp;            // active pixels, padded GEMM depth (2*Kact rounded to 64)
    int Kq;                  // padded depth of the norm GEMM (Kact rounded to 16)
    int my_r_max;
};

template <typename T>
T* upload(RomeGpuCtx* ctx, Slot s, const T* host, size_t n) {
    T* d = ctx->ws[s].as<T>(n);
    stage_copy(ctx, d, host, n);
    return d;
}

// Euler_angles2matrix(0, 0, psi) (src/math.cpp:86-115); the projector uses
// the transpose times the padding factor (src/reconstruct.cpp:860-870).
void rot2d_inv(double psi_deg, int padding, double out[4]) {
    const double rome_pi = 3.14159265358979323846;
    double alpha = 0 * rome_pi / 180., beta = 0 * rome_pi / 180., gamma = psi_deg * rome_pi / 180.;
    double ca = cos(alpha), cb = cos(beta), cg = cos(gamma);
    double sa = sin(alpha), sb = sin(beta), sg = sin(gamma);
    double cc = cb * ca, cs = cb * sa;
    double A00 = cg * cc - sg * sa, A01 = cg * cs + sg * ca;
    double A10 = -sg * cc - cg * sa, A11 = -sg * cs + cg * ca;
    out[0] = A00 * (double)padding;  // Ainv[0][0] = A[0][0]
    out[1] = A10 * (double)padding;  // Ainv[0][1] = A[1][0]
    out[2] = A01 * (double)padding;  // Ainv[1][0] = A[0][1]
    out[3] = A11 * (double)padding;  // Ainv[1][1] = A[1][1]
}

}  // namespace
}  // namespace rome

// ---------------------------------------------------------------------------
extern "C" int rome_gpu_map2d_estep_pool(RomeGpuCtx* ctx, const RomeMap2dPool* in, RomeMap2dPoolOut* out) {
    if (!ctx || !in || !out) return ROME_ERR_ARG;
    return guarded(ctx, [&] {
        if (!ctx->proj || ctx->ref_dim != 2) fail(ROME_ERR_STATE, "2D projectors not set (rome_gpu_set_projectors)");
        ROME_CUDA(cudaSetDevice(ctx->device));
        arena_reset(ctx);
        const int P = in->nr_images, K = in->nr_classes, ori = in->ori_size, cur = in->current_size;
        const int npsi = in->nr_psi, ntr = in->nr_trans, G = in->nr_groups, oriF = ori / 2 + 1;
        ROME_REQUIRE(P > 0 && K == ctx->nr_classes && ori == ctx->ori_size, "pool/projector mismatch");
        ROME_REQUIRE(cur > 0 && cur <= ori && cur % 2 == 0, "bad current_size %d", cur);
        ROME_REQUIRE(in->adaptive_oversampling >= 0 && in->adaptive_oversampling <= 1,
                     "adaptive_oversampling %d not supported (0 or 1)", in->adaptive_oversampling);
        ROME_REQUIRE(in->iclass_min >= 0 && in->iclass_max < K && in->iclass_min <= in->iclass_max, "bad class range");
        ROME_REQUIRE(ctx->r_max == std::min(cur / 2, ori / 2),
                     "projector r_max %d does not match current_size %d", ctx->r_max, cur);
        ROME_REQUIRE(in->Fimg_real && in->Fimg_imag && in->Fimg_nomask_real && in->Fimg_nomask_imag && in->Fctf,
                     "missing particle images");
        ROME_REQUIRE(npsi > 0 && ntr > 0 && G > 0, "empty sampling");
        ROME_CUDA(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        const int npass = in->adaptive_oversampling > 0 ? 2 : 1;
        const int curF2 = cur * (cur / 2 + 1);
        const long ncoarse = (long)K * npsi * ntr;
        const bool apply_ctf = in->do_ctf_correction && in->refs_are_ctf_corrected;
        Profiler prof(ctx);

        // ---- particle data at the fine size ----
        const int* dRows = nullptr;  // input row of each particle (subset of a staged pool)
        if (in->particle_rows) {
            ROME_REQUIRE(in->inputs_on_device, "particle_rows needs inputs_on_device");
            for (int i = 0; i < P; i++) ROME_REQUIRE(in->particle_rows[i] >= 0, "negative particle row");
            dRows = upload(ctx, S_ROWS, in->particle_rows, (size_t)P);
        }
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
        double* dSig2 = upload(ctx, S_SIG2, in->sigma2_noise, (size_t)G * oriF);
        int* dGroup = upload(ctx, S_GROUP, in->group, (size_t)P);
        double* dXi2 = upload(ctx, S_XI2, in->highres_Xi2, (size_t)P);
        // per-class model values: pdf_direction, prior offsets
        std::vector<double> hcls((size_t)3 * K);
        for (int k = 0; k < K; k++) {
            hcls[k] = in->pdf_direction[k];
            hcls[K + k] = in->prior_offsetx_class[k];
            hcls[2 * K + k] = in->prior_offsety_class[k];
        }
        double* dCls = upload(ctx, S_PDIR, hcls.data(), hcls.size());
        double* dPdir = dCls;
        std::vector<double2> hoff(P);
        for (int i = 0; i < P; i++) hoff[i] = make_double2(in->old_offsetx[i], in->old_offsety[i]);
        double2* dOld = upload(ctx, S_OLDOFF, hoff.data(), hoff.size());
        std::vector<double2> htc(ntr);
        for (int t = 0; t < ntr; t++) htc[t] = make_double2(in->trans_x[t], in->trans_y[t]);
        double2* dTrC = upload(ctx, S_TMP1, htc.data(), htc.size());
        // offset prior per particle, class and coarse translation
        double* dPoff = ctx->ws[S_POFF].as<double>((size_t)P * K * ntr);
        prof.begin(ROME_PHASE_PREP);
        pdf_offset_kernel<<<P, 128, 0, st>>>(P, K, ntr, dOld, dTrC, dCls + K, dCls + 2 * K, in->sigma2_offset, dPoff);
        prof.launched(ROME_PHASE_PREP);
        prof.end(ROME_PHASE_PREP);
        std::vector<int> hclass_ok(K);
        for (int k = 0; k < K; k++)
            hclass_ok[k] = (k >= in->iclass_min && k <= in->iclass_max && in->pdf_class[k] > 0. &&
                            in->pdf_direction[k] > 0.);

        double* dPart = ctx->ws[S_PART].as<double>((size_t)P * 8);  // min, sum, sig, thr, maxw, dcut
        int* dPartI = ctx->ws[S_PARTI].as<int>((size_t)P * 8);     // best e, nr_sign, overflow, b_low
        char* dMcoarse = ctx->ws[S_MCOARSE].as<char>((size_t)P * ncoarse);
        char* dRotSig = ctx->ws[S_ROTSIG].as<char>((size_t)K * npsi);

        std::vector<double> h_min(P), h_sum(P), h_sig(P), h_nsig(P);
        PassGeom g{};
        double2* dFimg = nullptr;
        double* dLctf = nullptr;
        double* dMinv = nullptr;
        double2* dProj = nullptr;
        float* dDiff2 = nullptr;
        int* dActIdx = nullptr;
        int* dAct = nullptr;
        double4* dRot = nullptr;
        double2* dShift = nullptr;
        double2* dPh = nullptr;
        int* dJvalid = nullptr;
        // significant-hypothesis list (filled by the selection of each pass)
        int* dCounter = ctx->ws[S_LISTCNT].as<int>((size_t)2 * K * npsi * 2 * 4 + 4);
        int* dSeg = ctx->ws[S_SEG].as<int>((size_t)2 * P);
        int listcap = std::max(1024, P * 64), nsigtot = 0;
        SigEntry* dList = nullptr;

        // optional restricted search (learned proposals): validated on the host
        const bool restricted = in->proposals != nullptr;
        const int nprop = restricted ? in->nr_proposals : 0;
        int* dProp = nullptr;
        if (restricted) {
            ROME_REQUIRE(npass == 1, "proposals need adaptive_oversampling 0");
            ROME_REQUIRE(nprop > 0 && nprop <= K * npsi, "nr_proposals %d out of range (1..%d)", nprop, K * npsi);
            for (int i = 0; i < P; i++)
                for (int q = 0; q < nprop; q++) {
                    const int j = in->proposals[(size_t)i * nprop + q];
                    ROME_REQUIRE(j >= 0 && j < K * npsi, "proposal %d of particle %d out of range", j, i);
                    ROME_REQUIRE(q == 0 || j > in->proposals[(size_t)i * nprop + q - 1],
                                 "proposals of particle %d not ascending and distinct", i);
                }
            dProp = upload(ctx, S_PROP, in->proposals, (size_t)P * nprop);
        }

        for (int ipass = 0; ipass < npass; ipass++) {
            const int cs = (ipass == 0 && in->adaptive_oversampling > 0) ? in->coarse_size : cur;
            const int over = ipass == 0 ? 0 : in->adaptive_oversampling;
            ROME_REQUIRE(cs > 0 && cs <= cur && cs % 2 == 0, "bad coarse_size %d", cs);
            g.cs = cs;
            g.csF = cs / 2 + 1;
            g.F = cs * g.csF;
            g.nor = 1 << over;
            g.notr = 1 << (2 * over);
            g.T = ntr * g.notr;
            g.nrot = npsi * g.nor;
            g.J = K * g.nrot;
            g.X = (long)g.J * g.T;
            g.my_r_max = std::min(ctx->r_max, cs / 2);
            ROME_REQUIRE(in->over_psi[ipass] && in->over_trans_x[ipass] && in->over_trans_y[ipass],
                         "missing sampling tables for pass %d", ipass);
            const int* Mresol = ipass == 0 ? in->Mresol_coarse : in->Mresol_fine;
            ROME_REQUIRE(Mresol, "missing Mresol for pass %d", ipass);

            // active pixels: the support of rotate2D, r^2 <= my_r_max^2 (reconstruct.cpp:866-891)
            std::vector<int> act, actidx(g.F, -1);
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
            dAct = upload(ctx, S_ACT, act.data(), act.size());
            dActIdx = upload(ctx, S_ACTIDX, actidx.data(), actidx.size());
            int* dClassOk = ctx->ws[S_JVALID].as<int>((size_t)K + g.J);
            stage_copy(ctx, dClassOk, hclass_ok.data(), (size_t)K);
            dJvalid = dClassOk + K;
            int* dMres = upload(ctx, S_MRES, Mresol, (size_t)g.F);

            // rotation matrices and translations of this pass
            std::vector<double4> hrot(g.J);
            for (int k = 0; k < K; k++)
                for (int r = 0; r < g.nrot; r++) {
                    double m[4];
                    rot2d_inv(in->over_psi[ipass][r], ctx->padding, m);
                    hrot[(size_t)k * g.nrot + r] = make_double4(m[0], m[1], m[2], m[3]);
                }
            dRot = upload(ctx, S_ROTM, hrot.data(), hrot.size());
            std::vector<double2> hsh(g.T);
            for (int t = 0; t < g.T; t++)
                hsh[t] = make_double2((double)in->over_trans_x[ipass][t] / (-ori),
                                      (double)in->over_trans_y[ipass][t] / (-ori));
            dShift = upload(ctx, S_SHIFT, hsh.data(), hsh.size());
            dPh = ctx->ws[S_PHASE].as<double2>((size_t)g.T * g.F);
            prof.begin(ROME_PHASE_SHIFT);
            phase_table_kernel<<<(unsigned)(((long)g.T * g.F + 255) / 256), 256, 0, st>>>(
                g.T, g.F, g.csF, cs, dShift, ctx->d_shift_tab, ctx->shift_sampling, dPh);
            prof.launched(ROME_PHASE_SHIFT);
            prof.end(ROME_PHASE_SHIFT);

            // ---- prep: window to cs, local CTF, Minvsigma2 ----
            dFimg = ctx->ws[S_FIMG].as<double2>((size_t)P * g.F);
            dLctf = ctx->ws[S_CTF].as<double>((size_t)P * g.F);
            dMinv = ctx->ws[S_MINV].as<double>((size_t)P * g.F);
            // the restricted tensor-core search takes its per-particle operands from the same pass
            const bool rtc_pass = restricted && ctx->precision != ROME_PREC_FP32 && g.T <= 256;
            RestrictedOut ro;
            if (rtc_pass) {
                const int Kh = g.Kp / 2;
                char* buf = (char*)ctx->ws[S_A].get((size_t)P * Kh * (sizeof(float2) + sizeof(float)));
                ro.xw = (float2*)buf;
                ro.w2 = (float*)(buf + (size_t)P * Kh * sizeof(float2));
                ro.S = ctx->ws[S_S].as<float>((size_t)P * g.T);
                ro.actidx = dActIdx;
                ro.Kact = g.Kact;
                ro.Kh = Kh;
                ro.apply_ctf = apply_ctf ? 1 : 0;
            }
            prof.begin(ROME_PHASE_PREP);
            prep_particles_kernel<<<P, 256, 0, st>>>(P, cur, cs, dFr, dFi, dCtf, dMres, dSig2, dGroup, oriF,
                                                      in->sigma2_fudge, dFimg, dLctf, dMinv, dRows, ro);
            prof.launched(ROME_PHASE_PREP);
            prof.end(ROME_PHASE_PREP);

            // ---- orientation validity and projections (getReferenceAllOrientations) ----
            const bool tc = ctx->precision != ROME_PREC_FP32;
            dProj = ctx->ws[S_PROJ].as<double2>((size_t)g.J * g.Kact);
            float* dQ = ctx->ws[S_Q].as<float>((size_t)g.J * g.Kq);
            void* dB = ctx->ws[S_B].get((size_t)g.J * g.Kp * 4);
            prof.begin(ROME_PHASE_PROJECT);
            {
                const int nkp = K * npsi;
                rot_sig_kernel<<<(nkp + 255) / 256, 256, 0, st>>>(nkp, P, ntr, ncoarse, ipass > 0 ? dMcoarse : nullptr,
                                                                   dRotSig);
                prof.launched(ROME_PHASE_PROJECT);
                jvalid_kernel<<<(g.J + 255) / 256, 256, 0, st>>>(g.J, g.nrot, g.nor, dClassOk, dRotSig, dJvalid);
                prof.launched(ROME_PHASE_PROJECT);
            }
            // the projections depend only on the model and the pass's sampling, not on the
            // particles: a pass-0 call with the same inputs as the previous one reuses them
            std::string key;
            if (ipass == 0) {
                auto put = [&key](const void* p, size_t n) { key.append((const char*)p, n); };
                const long hdr[12] = {ctx->proj_version, ctx->ref_dim, cs, g.my_r_max, K, npsi, g.nor, g.J, g.Kact,
                                      g.Kp, ctx->precision, ctx->padding};
                put(hdr, sizeof(hdr));
                put(hclass_ok.data(), sizeof(int) * hclass_ok.size());
                put(in->over_psi[0], sizeof(double) * (size_t)npsi * g.nor);
            }
            if (key.empty() || key != ctx->proj_key) {
                project2d_kernel<<<g.J, 256, 0, st>>>(g.J, g.Kact, g.Kp, g.Kq, cs, g.csF, g.my_r_max,
                                                      ctx->pad_size, ctx->pad_size / 2 + 1, g.nrot, ctx->proj,
                                                      ctx->vox, dRot, dAct, dJvalid, dProj, dQ, dB, ctx->precision);
                prof.launched(ROME_PHASE_PROJECT);
                ctx->proj_key = key;  // empty after a later pass: its projections replace pass 0's
            }
            prof.end(ROME_PHASE_PROJECT);

            // ---- shifted images -> A operand, S term ----
            const long M = (long)P * g.T;
            // restricted search on the tensor cores: no shifted images, the
            // translations enter through a [32][Kp] phase operand instead
            const bool rtc = restricted && tc && g.T <= 256;
            const int Kh = g.Kp / 2;
            void* dA = nullptr;
            float2* dXw = nullptr;
            float* dW2h = nullptr;
            void* dSh = nullptr;
            float* dS = ctx->ws[S_S].as<float>((size_t)M);
            float* dW2 = nullptr;
            prof.begin(ROME_PHASE_SHIFT);
            unsigned short* dPidx = ctx->ws[S_PIDX].as<unsigned short>((size_t)g.T * g.Kact);
            phase_index_kernel<<<(unsigned)(((long)g.T * g.Kact + 255) / 256), 256, 0, st>>>(
                g.T, g.Kact, g.csF, cs, dAct, dShift, ctx->shift_sampling, dPidx);
            prof.launched(ROME_PHASE_SHIFT);
            if (rtc) {
                // xw, w2 and S were written by prep_particles_kernel (ro)
                dXw = ro.xw;
                dW2h = ro.w2;
                dSh = ctx->ws[S_NORM].get((size_t)2 * restricted_tile_tn(g.T) * g.Kp * 2);
                restricted_shift_operand(st, g.T, g.Kact, g.Kp, dPidx, ctx->d_shift_tab, ctx->precision, dSh);
                prof.launched(ROME_PHASE_SHIFT);
            } else {
                dA = ctx->ws[S_A].get((size_t)M * g.Kp * 4);
                dW2 = ctx->ws[S_W2].as<float>((size_t)P * g.Kq);
                shift_operand2_kernel<256><<<P, 256, 0, st>>>(P, g.T, g.F, g.Kact, g.Kp, dFimg, dLctf, dMinv,
                                                               apply_ctf ? 1 : 0, dAct, dPidx, ctx->d_shift_tab, dA,
                                                               dS, ctx->precision);
                prof.launched(ROME_PHASE_SHIFT);
                w2_kernel<<<P, 256, 0, st>>>(P, g.Kact, g.Kq, dAct, dLctf, dMinv, g.F, apply_ctf ? 1 : 0, dW2);
                prof.launched(ROME_PHASE_SHIFT);
            }
            prof.end(ROME_PHASE_SHIFT);

            unsigned* dRowMin = ctx->ws[S_ROWMIN].as<unsigned>((size_t)P);
            ROME_CUDA(cudaMemsetAsync(dRowMin, 0xFF, sizeof(unsigned) * P, st));
            long Xrow = g.X;  // hypotheses per particle row
            if (!restricted) {
                // ---- norm term N[i][j] = sum_n Minv c^2 |P_j|^2 (FP32 CUDA cores) ----
                float* dNorm = ctx->ws[S_NORM].as<float>((size_t)P * g.J);
                prof.begin(ROME_PHASE_NORM_GEMM);
                if (!tc) {
                    sgemm_tn(st, P, g.J, g.Kq, dW2, g.Kq, dQ, g.Kq, StoreEpi{dNorm, g.J});
                    prof.launched(ROME_PHASE_NORM_GEMM);
                } else {
                    // split-BF16 on the tensor cores in every tensor-core mode: the
                    // norm term is all positive, so its hi/lo rounding averages out
                    const int Kq64 = ((g.Kact + 63) / 64) * 64;
                    void* dW2b = ctx->ws[S_W2B].get((size_t)P * Kq64 * 4);
                    void* dQb = ctx->ws[S_QB].get((size_t)g.J * Kq64 * 4);
                    split_bf16(st, dW2, P, g.Kact, g.Kq, Kq64, dW2b);
                    split_bf16(st, dQ, g.J, g.Kact, g.Kq, Kq64, dQb);
                    tc_store_gemm(st, P, g.J, Kq64, dW2b, dQb, dNorm, g.J, ctx->d_err);
                    prof.launched(ROME_PHASE_NORM_GEMM, 3);
                }
                prof.add_flops(ROME_PHASE_NORM_GEMM, 2.0 * P * g.J * g.Kact);
                prof.end(ROME_PHASE_NORM_GEMM);

                // ---- cross term + fused diff2 epilogue ----
                dDiff2 = ctx->ws[S_DIFF2].as<float>((size_t)P * g.X);
                Diff2Epi epi{dDiff2, dNorm, dS, dXi2, dJvalid, g.T, g.J, g.X, g.notr, g.nor, ntr, ncoarse,
                             ipass > 0 ? dMcoarse : nullptr, dRowMin};
                prof.begin(ROME_PHASE_CROSS_GEMM);
                if (!tc) {
                    sgemm_tn(st, (int)M, g.J, g.Kp, (const float*)dA, g.Kp, (const float*)dB, g.Kp, epi);
                } else {
                    tc_diff2_gemm(st, (int)M, g.J, g.Kp, dA, dB, ctx->precision, epi, ctx->d_err);
                }
                prof.launched(ROME_PHASE_CROSS_GEMM);
                // algorithmic work: 4 flops per active complex coefficient per (image, translation, orientation)
                prof.add_flops(ROME_PHASE_CROSS_GEMM, 4.0 * (double)M * g.J * g.Kact);
                prof.end(ROME_PHASE_CROSS_GEMM);
            } else {
                // ---- restricted search: only the proposed orientations ----
                Xrow = (long)nprop * g.T;
                dDiff2 = ctx->ws[S_DIFF2].as<float>((size_t)P * Xrow);
                dim3 grid((nprop + RS_QQ - 1) / RS_QQ, (g.T + RS_TQ - 1) / RS_TQ, P);
                prof.begin(ROME_PHASE_RESTRICTED);
                if (rtc) {
                    restricted_tc_diff2(st, ctx->precision, P, nprop, g.T, g.Kp, dProp, dJvalid, dXw, dW2h, dB, g.J,
                                        dSh, dS, dXi2, Xrow, dDiff2, dRowMin, ctx->d_err);
                } else {
                    // CUDA cores over the shifted images (FP32 mode, or more than 256 translations)
                    if (ctx->precision == ROME_PREC_FP32)
                        restricted_diff2_kernel<ROME_PREC_FP32><<<grid, RS_THREADS, 0, st>>>(
                            g.T, g.Kp, g.Kq, nprop, M, g.J, dProp, dJvalid, dA, dB, dW2, dQ, dS, dXi2, Xrow, dDiff2,
                            dRowMin);
                    else if (ctx->precision == ROME_PREC_BF16)
                        restricted_diff2_kernel<ROME_PREC_BF16><<<grid, RS_THREADS, 0, st>>>(
                            g.T, g.Kp, g.Kq, nprop, M, g.J, dProp, dJvalid, dA, dB, dW2, dQ, dS, dXi2, Xrow, dDiff2,
                            dRowMin);
                    else
                        restricted_diff2_kernel<ROME_PREC_BF16X3><<<grid, RS_THREADS, 0, st>>>(
                            g.T, g.Kp, g.Kq, nprop, M, g.J, dProp, dJvalid, dA, dB, dW2, dQ, dS, dXi2, Xrow, dDiff2,
                            dRowMin);
                    ROME_CHECK_LAUNCH();
                }
                prof.launched(ROME_PHASE_RESTRICTED);
                prof.add_flops(ROME_PHASE_RESTRICTED, 4.0 * (double)P * Xrow * g.Kact);
                prof.end(ROME_PHASE_RESTRICTED);
            }

            // ---- posterior: min, FP64 weights, sum, argmax, significance ----
            double* dW = nullptr;
            if (out->weight[ipass] && !restricted) dW = ctx->ws[S_WCHK].as<double>((size_t)P * g.X);
            PostLayout Lp{g.T, g.notr, g.nor, npsi, ntr, K};
            if (restricted) {
                int2* dEntR = ctx->ws[S_FENT].as<int2>((size_t)P * nprop);
                restricted_entries_kernel<<<(unsigned)(((long)P * nprop + 255) / 256), 256, 0, st>>>(
                    (long)P * nprop, g.nrot, dProp, dEntR);
                ROME_CHECK_LAUNCH();
                Lp.ent = dEntR;
                Lp.ent_stride = nprop;
                Lp.epr = g.T;
            }
            prof.begin(ROME_PHASE_POSTERIOR);
            for (;;) {
                dList = ctx->ws[S_SIGLIST].as<SigEntry>((size_t)listcap * 2);
                SelectResult sr = run_select(ctx, st, 0, P, Xrow, Lp, dDiff2, dPdir, dPoff, in->adaptive_fraction,
                                             dPart, dPartI, nullptr, dW, dList, dCounter, listcap, dSeg, dRowMin);
                prof.launched(ROME_PHASE_POSTERIOR, sr.launches);
                nsigtot = sr.nlist;
                if (sr.nlist <= listcap) break;
                listcap = sr.nlist;  // every segment fits on the second run
            }
            if (restricted && nsigtot > 0) {
                restricted_list_dense_kernel<<<(nsigtot + 255) / 256, 256, 0, st>>>(nsigtot, g.T, nprop, dProp, dList);
                ROME_CHECK_LAUNCH();
                prof.launched(ROME_PHASE_POSTERIOR);
            }
            if (ipass == npass - 1 && out->post_class_psi) {
                double* dMarg = ctx->ws[S_TMP2].as<double>((size_t)P * K * npsi);
                ROME_CUDA(cudaMemsetAsync(dMarg, 0, sizeof(double) * P * K * npsi, st));
                if (nsigtot > 0) {
                    post_marginal_kernel<<<(nsigtot + 255) / 256, 256, 0, st>>>(nsigtot, g.T, g.nor, K * npsi, dList,
                                                                               dMarg);
                    ROME_CHECK_LAUNCH();
                }
                ROME_CUDA(cudaMemcpyAsync(out->post_class_psi, dMarg, sizeof(double) * P * K * npsi,
                                          cudaMemcpyDeviceToHost, st));
            }
            if (ipass == 0 && (npass > 1 || out->Mcoarse_significant)) {
                ROME_CUDA(cudaMemsetAsync(dMcoarse, 0, (size_t)P * ncoarse, st));
                if (nsigtot > 0) {
                    mcoarse_from_list_kernel<<<(nsigtot + 255) / 256, 256, 0, st>>>(nsigtot, g.X, dList, dMcoarse);
                    prof.launched(ROME_PHASE_POSTERIOR);
                }
            }
            prof.end(ROME_PHASE_POSTERIOR);

            if (tc) tc_check_error(st, ctx->d_err);

            // ---- checkpoints and per-particle results of this pass ----
            std::vector<double> hpart((size_t)P * 8);
            std::vector<int> hparti((size_t)P * 8);
            ROME_CUDA(cudaMemcpyAsync(hpart.data(), dPart, sizeof(double) * P * 8, cudaMemcpyDeviceToHost, st));
            ROME_CUDA(cudaMemcpyAsync(hparti.data(), dPartI, sizeof(int) * P * 8, cudaMemcpyDeviceToHost, st));
            if (out->diff2[ipass] && !restricted) {
                std::vector<float> hd((size_t)P * g.X);
                ROME_CUDA(cudaMemcpyAsync(hd.data(), dDiff2, sizeof(float) * hd.size(), cudaMemcpyDeviceToHost, st));
                ROME_CUDA(cudaStreamSynchronize(st));
                for (size_t q = 0; q < hd.size(); q++)
                    out->diff2[ipass][q] = hd[q] < INFINITY ? (double)hd[q] : (double)INT_MIN;
            }
            if (out->weight[ipass] && dW)
                ROME_CUDA(cudaMemcpyAsync(out->weight[ipass], dW, sizeof(double) * P * g.X, cudaMemcpyDeviceToHost,
                                          st));
            if (ipass == 0 && out->Mcoarse_significant)
                ROME_CUDA(cudaMemcpyAsync(out->Mcoarse_significant, dMcoarse, (size_t)P * ncoarse,
                                          cudaMemcpyDeviceToHost, st));
            ROME_CUDA(cudaStreamSynchronize(st));
            for (int i = 0; i < P; i++) {
                double mn = hpart[i * 8 + 0], sw = hpart[i * 8 + 1], sig = hpart[i * 8 + 2], mx = hpart[i * 8 + 4];
                int best = hparti[i * 8 + 0], nsig = hparti[i * 8 + 1];
                if (ipass == 0 && nsig == 0)
                    fail(ROME_ERR_NUMERIC, "my_nr_significant_coarse_samples == 0 for particle %d", i);
                h_min[i] = mn;
                h_sum[i] = sw;
                h_sig[i] = sig;
                if (ipass == 0) h_nsig[i] = nsig;
                // convertSquaredDifferencesToWeights metadata (map2d_optimizer.cpp:1199-1216)
                long e = best;
                int j = (int)(e / g.T), t = (int)(e % g.T);
                if (restricted) j = in->proposals[(size_t)i * nprop + j];  // row position -> orientation
                int r = j % g.nrot, k = j / g.nrot;
                int itr = t / g.notr, iotr = t % g.notr;
                if (out->pmax) out->pmax[i] = mx / sw;
                if (out->cls) out->cls[i] = k + 1;
                if (out->psi) {
                    double psi = in->over_psi[ipass][r];
                    if (psi > 180.) psi -= 360.;
                    if (psi < -180.) psi += 360.;
                    out->psi[i] = psi;
                }
                if (out->xoff) out->xoff[i] = in->old_offsetx[i] + in->over_trans_x[ipass][itr * g.notr + iotr];
                if (out->yoff) out->yoff[i] = in->old_offsety[i] + in->over_trans_y[ipass][itr * g.notr + iotr];
            }
        }

        // ---- updateOtherParams (last pass, current_size) ----
        const int lp = npass - 1;
        std::vector<double2> htr(g.T);
        for (int t = 0; t < g.T; t++) htr[t] = make_double2(in->over_trans_x[lp][t], in->over_trans_y[lp][t]);
        double2* dTr = upload(ctx, S_TRANS, htr.data(), htr.size());
        int* dMresF = upload(ctx, S_MRES, in->Mresol_fine, (size_t)g.F);
        // accumulators: wsum_sigma2_noise [G][oriF], norm_corr [P];
        // class sums [0] pdf_class [1] pdf_direction [2] prior x [3] prior y [4] sigma2_offset, then groups
        double* dWsn = ctx->ws[S_WSN].as<double>((size_t)G * oriF + P);
        double* dNormCorr = dWsn + (size_t)G * oriF;
        double* dWk = ctx->ws[S_WSUMK].as<double>((size_t)5 * K + G + 1);
        ROME_CUDA(cudaMemsetAsync(dWsn, 0, sizeof(double) * ((size_t)G * oriF + P), st));
        ROME_CUDA(cudaMemsetAsync(dWk, 0, sizeof(double) * ((size_t)5 * K + G + 1), st));
        // significant hypotheses of the last pass are in dList (particle segments)
        const int cap = listcap;
        prof.begin(ROME_PHASE_WSUM);
        {
            const int NT = 256, PIX = 4;
            int nsplit = (g.F + NT * PIX - 1) / (NT * PIX);
            ROME_REQUIRE(P <= 65535, "pool of %d particles: at most 65,535", P);
            wsum_list_kernel<NT, PIX><<<dim3(nsplit, P), NT, 0, st>>>(
                g.T, g.nrot, K, g.F, g.csF, cur, oriF, dList, dSeg, dFimg, dLctf, apply_ctf ? 1 : 0, dProj, dActIdx,
                g.Kact, dShift, dPh, dMresF, dGroup, dOld, dTr, dCls + K,
                dCls + 2 * K, dWsn, dNormCorr, dWk);
            prof.launched(ROME_PHASE_WSUM);
        }
        prof.end(ROME_PHASE_WSUM);

        // ---- backProjection ----
        std::vector<int> hoff_bp;  // list offsets per orientation (profiling: slices back-projected)
        {
            double2* dFnm = ctx->ws[S_FNOMASK].as<double2>((size_t)P * g.F);
            double* dMctf2 = dMinv;  // reused in place: becomes ctf^2 * Minvsigma2
            prof.begin(ROME_PHASE_BACKPROJECT);
            bp_prep_kernel<<<P, 256, 0, st>>>(P, g.F, dFnr, dFni, dLctf, dMinv, dSig2, dGroup, oriF,
                                              in->sigma2_fudge, in->do_map, in->do_ctf_correction, dFnm, dMctf2,
                                              dRows);
            prof.launched(ROME_PHASE_BACKPROJECT);
            // group the significant list by orientation (counting sort)
            int* dCnt = dCounter + 2;
            int* dOff = ctx->ws[S_OFFJ].as<int>((size_t)2 * g.J + 2);
            int* dFill = dOff + g.J + 1;
            SigEntry* dSorted = dList + cap;
            ROME_CUDA(cudaMemsetAsync(dCnt, 0, sizeof(int) * g.J, st));
            ROME_CUDA(cudaMemsetAsync(dFill, 0, sizeof(int) * g.J, st));
            if (nsigtot > 0) {
                count_by_j_kernel<<<(nsigtot + 255) / 256, 256, 0, st>>>(nsigtot, g.T, dList, dCnt);
                prof.launched(ROME_PHASE_BACKPROJECT);
            }
            exclusive_scan_kernel<<<1, 1024, 0, st>>>(g.J, dCnt, dOff);
            prof.launched(ROME_PHASE_BACKPROJECT);
            if (nsigtot > 0) {
                scatter_by_j_kernel<<<(nsigtot + 255) / 256, 256, 0, st>>>(nsigtot, g.T, dList, dOff, dFill, dSorted);
                prof.launched(ROME_PHASE_BACKPROJECT);
            }
            const int NT = 256, PIX = 4;
            int nsplit = (g.F + NT * PIX - 1) / (NT * PIX);
            for (int j0 = 0; j0 < g.J; j0 += 65535)  // grid y limit
                bp_list_kernel<NT, PIX><<<dim3(nsplit, std::min(g.J - j0, 65535)), NT, 0, st>>>(
                    g.T, g.nrot, g.F, g.csF, cur, dSorted, dOff, dFnm, dMctf2, dShift, dPh, dRot, ctx->r_max,
                    ctx->pad_size, ctx->pad_size / 2 + 1, ctx->bp_data, ctx->bp_weight, ctx->vox, j0);
            prof.launched(ROME_PHASE_BACKPROJECT);
            prof.end(ROME_PHASE_BACKPROJECT);
            if (ctx->profile) {
                hoff_bp.resize((size_t)g.J + 1);
                ROME_CUDA(cudaMemcpyAsync(hoff_bp.data(), dOff, sizeof(int) * (g.J + 1), cudaMemcpyDeviceToHost, st));
            }
        }

        // ---- outputs ----
        std::vector<double> hwsn((size_t)G * oriF + P), hwk((size_t)5 * K + G + 1);
        ROME_CUDA(cudaMemcpyAsync(hwsn.data(), dWsn, sizeof(double) * hwsn.size(), cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaMemcpyAsync(hwk.data(), dWk, sizeof(double) * hwk.size(), cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaStreamSynchronize(st));
        prof.collect();
        if (!hoff_bp.empty()) {
            // algorithmic bytes of the back-projection: the prepared image and ctf^2 Minvsigma2 of every
            // significant hypothesis (24 B per active pixel) and 12 FP64 updates (96 B) per active pixel of
            // every back-projected slice (orientation with significant hypotheses)
            long nslice = 0;
            for (int j = 0; j + 1 < (int)hoff_bp.size(); j++) nslice += hoff_bp[j + 1] > hoff_bp[j];
            prof.add_bytes(ROME_PHASE_BACKPROJECT, (double)g.Kact * (24.0 * nsigtot + 96.0 * nslice));
        }
        for (size_t q = 0; q < (size_t)G * oriF; q++) out->wsum_sigma2_noise[q] += hwsn[q];
        for (int i = 0; i < P; i++) {
            if (out->wsum_norm_correction) out->wsum_norm_correction[i] = hwsn[(size_t)G * oriF + i];
            if (out->min_diff2) out->min_diff2[i] = h_min[i];
            if (out->sum_weight) out->sum_weight[i] = h_sum[i];
            if (out->significant_weight) out->significant_weight[i] = h_sig[i];
            if (out->nr_sign) out->nr_sign[i] = h_nsig[i];
        }
        for (int k = 0; k < K; k++) {
            out->wsum_pdf_class[k] += hwk[0 * K + k];
            out->wsum_pdf_direction[k] += hwk[1 * K + k];
            out->wsum_prior_offsetx_class[k] += hwk[2 * K + k];
            out->wsum_prior_offsety_class[k] += hwk[3 * K + k];
        }
        for (int q = 0; q < G; q++) out->wsum_sumw_group[q] += hwk[5 * K + q];
        for (int k = 0; k < K; k++) out->wsum_sigma2_offset[0] += hwk[4 * K + k];
        for (int i = 0; i < P; i++)
            if (h_sum[i] == 0) fail(ROME_ERR_NUMERIC, "exp_sum_weight[%d] == 0", i);
    });
}

extern "C" int rome_gpu_select_significant(RomeGpuCtx* ctx, int n, long len, const double* weights,
                                           const double* sum_weight, double adaptive_fraction,
                                           double* significant_weight, double* nr_significant) {
    if (!ctx) return ROME_ERR_ARG;
    return guarded(ctx, [&] {
        ROME_REQUIRE(n > 0 && len > 0 && weights && sum_weight && significant_weight && nr_significant,
                     "bad arguments");
        ROME_CUDA(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        double* dW = ctx->ws[S_WCHK].as<double>((size_t)n * len);
        ROME_CUDA(cudaMemcpyAsync(dW, weights, sizeof(double) * n * len, cudaMemcpyHostToDevice, st));
        double* dPart = ctx->ws[S_PART].as<double>((size_t)n * 8);
        int* dPartI = ctx->ws[S_PARTI].as<int>((size_t)n * 8);
        std::vector<double> hp((size_t)n * 8, 0.0);
        for (int i = 0; i < n; i++) hp[(size_t)i * 8 + 1] = sum_weight[i];
        ROME_CUDA(cudaMemcpyAsync(dPart, hp.data(), sizeof(double) * n * 8, cudaMemcpyHostToDevice, st));
        run_select(ctx, st, 1, n, len, PostLayout{1, 1, 1, 1, 1, 1}, nullptr, nullptr, nullptr, adaptive_fraction,
                   dPart, dPartI, dW, nullptr, nullptr, nullptr, 0, nullptr);
        std::vector<double> hpart((size_t)n * 8);
        std::vector<int> hparti((size_t)n * 8);
        ROME_CUDA(cudaMemcpyAsync(hpart.data(), dPart, sizeof(double) * n * 8, cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaMemcpyAsync(hparti.data(), dPartI, sizeof(int) * n * 8, cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaStreamSynchronize(st));
        for (int i = 0; i < n; i++) {
            significant_weight[i] = hpart[(size_t)i * 8 + 2];
            nr_significant[i] = hparti[(size_t)i * 8 + 1];
        }
    });
}

// ---------------------------------------------------------------------------
// Significance selection without device allocation.
//
// rome_gpu_select_significant_static runs the same kernels as
// rome_gpu_select_significant, but every device buffer it touches is carved
// from one fixed array compiled into this library (g_select_static below)
// instead of the context's grow-on-demand workspace.  It is meant for callers
// that must not allocate device memory during the call: a host that has
// handed all free HBM to its own pool allocator, a caller running inside a
// memory budget it cannot exceed, or code that must not trigger the implicit
// device synchronisation a cudaMalloc/cudaFree can cause.
//
// Limits: n <= ROME_SELECT_STATIC_MAX_IMAGES and n * len <=
// ROME_SELECT_STATIC_MAX_WEIGHTS; larger requests return ROME_ERR_ARG and
// touch nothing.  The array is 8 MiB of weights + 8 MiB of sort scratch for
// rows whose candidate set does not fit in shared memory + per-row scalars.
//
// The first call on each device looks the array's device address up
// (cudaGetSymbolAddress, which may load the module on that device); make
// that first call before any stream capture on the device.  Under lazy
// module loading that first call is where the driver reserves the array and
// the module's code, so it is a warm-up: later calls allocate nothing.  The
// call is synchronous (results are in the caller's host arrays when it
// returns).  All calls on one
// device share the array, so two calls overlapping in time would race on it:
// the entry point holds a process-wide lock and returns only after its
// stream work has finished, which serialises calls from different host
// threads.
namespace rome {
namespace {

constexpr size_t kStaticAlign = 256;
constexpr size_t align_up(size_t v) { return (v + kStaticAlign - 1) / kStaticAlign * kStaticAlign; }

constexpr size_t kOffW = 0;  // caller weights [n][len] double
constexpr size_t kOffFB = kOffW + align_up(sizeof(double) * ROME_SELECT_STATIC_MAX_WEIGHTS);  // fallback sort slots
constexpr size_t kOffPart = kOffFB + align_up(sizeof(double) * ROME_SELECT_STATIC_MAX_WEIGHTS);
constexpr size_t kOffPartI = kOffPart + align_up(sizeof(double) * 8 * ROME_SELECT_STATIC_MAX_IMAGES);
constexpr size_t kOffList = kOffPartI + align_up(sizeof(int) * 8 * ROME_SELECT_STATIC_MAX_IMAGES);
constexpr size_t kOffCount = kOffList + align_up(sizeof(int) * ROME_SELECT_STATIC_MAX_IMAGES);
constexpr size_t kOffIO = kOffCount + kStaticAlign;  // sum_weight in, [sig | nsig] out
constexpr size_t kStaticBytes = kOffIO + align_up(sizeof(double) * 2 * ROME_SELECT_STATIC_MAX_IMAGES);

static __device__ __align__(256) unsigned char g_select_static[kStaticBytes];

constexpr int kMaxDevices = 64;
std::mutex g_static_lock;
unsigned char* g_static_base[kMaxDevices] = {};

// per-row scalars start from zero, except the caller's sum of weights
__global__ void static_prep_kernel(int n, const double* __restrict__ sumw, double* __restrict__ part,
                                   int* __restrict__ parti) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = 0; k < 8; k++) {
        part[(long)i * 8 + k] = k == 1 ? sumw[i] : 0.0;
        parti[(long)i * 8 + k] = 0;
    }
}

// rows whose candidates overflowed shared memory, compacted in one block
__global__ void static_overflow_kernel(int n, const int* __restrict__ parti, int* __restrict__ list,
                                       int* __restrict__ count) {
    __shared__ int cnt;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (parti[(long)i * 8 + 2]) list[atomicAdd(&cnt, 1)] = i;
    __syncthreads();
    if (threadIdx.x == 0) *count = cnt;
}

__global__ void static_finish_kernel(int n, const double* __restrict__ part, const int* __restrict__ parti,
                                     double* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = part[(long)i * 8 + 2];
    out[n + i] = (double)parti[(long)i * 8 + 1];
}

}  // namespace
}  // namespace rome

extern "C" int rome_gpu_select_significant_static(RomeGpuCtx* ctx, int n, long len, const double* weights,
                                                  const double* sum_weight, double adaptive_fraction,
                                                  double* significant_weight, double* nr_significant) {
    if (!ctx) return ROME_ERR_ARG;
    return guarded(ctx, [&] {
        ROME_REQUIRE(n > 0 && len > 0 && weights && sum_weight && significant_weight && nr_significant,
                     "bad arguments");
        ROME_REQUIRE(n <= ROME_SELECT_STATIC_MAX_IMAGES,
                     "select_significant_static: %d images exceed the static limit of %d", n,
                     ROME_SELECT_STATIC_MAX_IMAGES);
        ROME_REQUIRE(len <= (long)ROME_SELECT_STATIC_MAX_WEIGHTS / n,
                     "select_significant_static: %d x %ld weights exceed the static limit of %d", n, len,
                     ROME_SELECT_STATIC_MAX_WEIGHTS);
        ROME_REQUIRE(ctx->device >= 0 && ctx->device < kMaxDevices, "device %d out of range", ctx->device);
        std::lock_guard<std::mutex> lock(g_static_lock);
        ROME_CUDA(cudaSetDevice(ctx->device));
        if (!g_static_base[ctx->device]) {
            void* p = nullptr;
            ROME_CUDA(cudaGetSymbolAddress(&p, g_select_static));
            g_static_base[ctx->device] = (unsigned char*)p;
        }
        unsigned char* base = g_static_base[ctx->device];
        double* dW = (double*)(base + kOffW);
        double* dFB = (double*)(base + kOffFB);
        double* dPart = (double*)(base + kOffPart);
        int* dPartI = (int*)(base + kOffPartI);
        int* dList = (int*)(base + kOffList);
        int* dCount = (int*)(base + kOffCount);
        double* dIO = (double*)(base + kOffIO);
        cudaStream_t st = ctx->stream;

        ROME_CUDA(cudaMemcpyAsync(dW, weights, sizeof(double) * n * len, cudaMemcpyHostToDevice, st));
        ROME_CUDA(cudaMemcpyAsync(dIO, sum_weight, sizeof(double) * n, cudaMemcpyHostToDevice, st));
        static_prep_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, dIO, dPart, dPartI);
        ROME_CHECK_LAUNCH();
        const size_t smem = (sizeof(double) + sizeof(int)) * SEL2_CAP;
        ROME_CUDA(cudaFuncSetAttribute(post_select2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const PostLayout L{1, 1, 1, 1, 1, 1};
        post_select2_kernel<<<n, SEL2_THREADS, smem, st>>>(1, len, L, nullptr, nullptr, nullptr, adaptive_fraction,
                                                           dPart, dPartI, dW, nullptr, nullptr, nullptr, 0, nullptr,
                                                           nullptr);
        ROME_CHECK_LAUNCH();
        static_overflow_kernel<<<1, 256, 0, st>>>(n, dPartI, dList, dCount);
        ROME_CHECK_LAUNCH();
        int nover = 0;
        ROME_CUDA(cudaMemcpyAsync(&nover, dCount, sizeof(int), cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaStreamSynchronize(st));
        int launches = 3;
        if (nover > 0) {
            long n2 = 1;
            while (n2 < len) n2 <<= 1;  // len <= the weight limit, so one slot always fits
            const int slots = (int)std::min<long>(nover, (long)ROME_SELECT_STATIC_MAX_WEIGHTS / n2);
            for (int b = 0; b < nover; b += slots) {
                const int nb = std::min(slots, nover - b);
                select_fallback2_kernel<<<nb, SEL2_THREADS, 0, st>>>(1, len, L, nullptr, nullptr, nullptr, dW,
                                                                    dList + b, n2, dFB, dPart, dPartI);
                ROME_CHECK_LAUNCH();
                launches++;
            }
        }
        static_finish_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, dPart, dPartI, dIO);
        ROME_CHECK_LAUNCH();
        launches++;
        ROME_CUDA(cudaMemcpyAsync(significant_weight, dIO, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaMemcpyAsync(nr_significant, dIO + n, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaStreamSynchronize(st));
        ctx->phase_launches[ROME_PHASE_POSTERIOR] += launches;
        ctx->total_launches += launches;
    });
}
