/*
 * CPU restatement of the ROME MAP2D E-step (test infrastructure only; the
 * parity checker for the GPU path, never linked by the product).
 *
 * Every function follows a reference routine, cited at its definition, in
 * FP64 and in the reference's loop order.  Built with -ffp-contract=off so
 * no multiply-add is fused, matching the reference build in this directory.
 */
#include "estep_oracle.h"

#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_PI 3.14159265358979323846 /* src/macros.h:69 */
#define ORACLE_EQUAL_ACCURACY 1e-6       /* src/macros.h:73-80 (FP64 build) */

/* ---- Euler_angles2matrix, src/math.cpp:86-115 ---- */
void oracle_euler_matrix(double alpha, double beta, double gamma, double A[9]) {
    const double rome_pi = 3.14159265358979323846; /* src/math.h:38 */
    alpha = alpha * rome_pi / 180.;
    beta = beta * rome_pi / 180.;
    gamma = gamma * rome_pi / 180.;
    double ca = cos(alpha), cb = cos(beta), cg = cos(gamma);
    double sa = sin(alpha), sb = sin(beta), sg = sin(gamma);
    double cc = cb * ca, cs = cb * sa, sc = sb * ca, ss = sb * sa;
    A[0] = cg * cc - sg * sa;
    A[1] = cg * cs + sg * ca;
    A[2] = -cg * sb;
    A[3] = -sg * cc - cg * sa;
    A[4] = -sg * cs + cg * ca;
    A[5] = sg * sb;
    A[6] = sc;
    A[7] = ss;
    A[8] = cb;
}

/* ---- shiftImageInFourierTransform, src/image.h:1478-1575 ---- */
static double g_tab_sin[5000], g_tab_cos[5000];
static int g_tab_ready = 0;

static void shift_tables(void) {
    if (g_tab_ready) return;
    double sampling = 2 * ORACLE_PI / (double)5000;
    for (int i = 0; i < 5000; i++) {
        double xx = (double)i * sampling;
        g_tab_sin[i] = sin(xx);
        g_tab_cos[i] = cos(xx);
    }
    g_tab_ready = 1;
}

static void shift_one(double x, double y, double xshift, double yshift, double c, double d, double* outr,
                      double* outi) {
    const double sampling = 2 * ORACLE_PI / (double)5000;
    double dotp = 2 * ORACLE_PI * (x * xshift + y * yshift);
    double a = g_tab_cos[((int)(fabs(dotp) / sampling)) % 5000];
    double b = g_tab_sin[((int)(fabs(dotp) / sampling)) % 5000];
    b = (dotp < 0) ? -b : b;
    double ac = a * c, bd = b * d, ab_cd = (a + b) * (c + d);
    *outr = ac - bd;
    *outi = ab_cd - ac - bd;
}

void oracle_shift_image(const double* fin_real, const double* fin_imag, double* fout_real, double* fout_imag,
                        int size, double shift_x, double shift_y, int ori_size) {
    shift_tables();
    int Fs = size / 2 + 1;
    double xshift = (double)shift_x / (-ori_size);
    double yshift = (double)shift_y / (-ori_size);
    if (fabs(xshift) < ORACLE_EQUAL_ACCURACY && fabs(yshift) < ORACLE_EQUAL_ACCURACY) {
        memcpy(fout_real, fin_real, sizeof(double) * size * Fs);
        memcpy(fout_imag, fin_imag, sizeof(double) * size * Fs);
        return;
    }
    for (int i = 0; i < size; i++) {
        double y = (i < Fs) ? i : i - size;
        for (int j = 0; j < Fs; j++) {
            int n = i * Fs + j;
            shift_one((double)j, y, xshift, yshift, fin_real[n], fin_imag[n], &fout_real[n], &fout_imag[n]);
        }
    }
}

/* windowFourierTransform / windowTransform (src/image.h:419-568), downsizing branch or copy */
static void window_ft(const double* in, int in_size, double* out, int out_size) {
    int inF = in_size / 2 + 1, outF = out_size / 2 + 1;
    if (in_size == out_size) {
        memcpy(out, in, sizeof(double) * out_size * outF);
        return;
    }
    for (int i = 0; i < out_size; i++) {
        int ip = (i < outF) ? i : i - out_size;
        int in_i = ip < 0 ? ip + in_size : ip;
        int out_i = ip < 0 ? ip + out_size : ip;
        for (int j = 0; j < outF; j++) out[out_i * outF + j] = in[in_i * inF + j];
    }
}

/* ---- MyProjector::rotate2D, src/reconstruct.cpp:823-958 (trilinear branch) ---- */
void oracle_rotate2d(const double* data, int pad_size, int r_max, int padding_factor, double psi_deg, int f2d_size,
                     double* f2d_real, double* f2d_imag) {
    double A[9], Ainv[9];
    oracle_euler_matrix(0, 0, psi_deg, A);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Ainv[i * 3 + j] = A[j * 3 + i] * (double)padding_factor;
    int padF = pad_size / 2 + 1;
    int my_r_max = r_max < f2d_size / 2 ? r_max : f2d_size / 2;
    int max_r2 = my_r_max * my_r_max;
    int Fs = f2d_size / 2 + 1;
    int shift = -(int)((float)pad_size / 2.0);
    for (int i = 0; i < f2d_size * Fs; i++) f2d_real[i] = f2d_imag[i] = 0;
    for (int i = 0; i < f2d_size; i++) {
        int y;
        if (i <= my_r_max) y = i;
        else if (i >= f2d_size - my_r_max) y = i - f2d_size;
        else continue;
        int y2 = y * y;
        for (int x = 0; x <= my_r_max; x++) {
            int r2 = x * x + y2;
            if (r2 > max_r2) continue;
            double xp = Ainv[0] * x + Ainv[1] * y;
            double yp = Ainv[3] * x + Ainv[4] * y;
            int neg = 0;
            if (xp < 0) {
                xp = -xp;
                yp = -yp;
                neg = 1;
            }
            int x0 = (int)floor(xp);
            double fx = xp - x0;
            int y0 = (int)floor(yp);
            double fy = yp - y0;
            y0 -= shift;
            int y1 = y0 + 1;
            const double* d00 = data + ((long)y0 * padF + x0) * 2;
            const double* d10 = data + ((long)y1 * padF + x0) * 2;
            double dx0r = d00[0] + (d00[2] - d00[0]) * fx;
            double dx0i = d00[1] + (d00[3] - d00[1]) * fx;
            double dx1r = d10[0] + (d10[2] - d10[0]) * fx;
            double dx1i = d10[1] + (d10[3] - d10[1]) * fx;
            double vr = dx0r + (dx1r - dx0r) * fy;
            double vi = dx0i + (dx1i - dx0i) * fy;
            f2d_real[i * Fs + x] = vr;
            f2d_imag[i * Fs + x] = neg ? -1.0 * vi : vi;
        }
    }
}

/* ---- MyBackProjector::backrotate2D, src/reconstruct.cpp:1353-1500 (trilinear branch) ---- */
void oracle_backrotate2d(const double* f2d_real, const double* f2d_imag, const double* Mweight, int f2d_size,
                         double psi_deg, int pad_size, int r_max, int padding_factor, double* bp_data,
                         double* bp_weight) {
    double A[9], Ainv[9];
    oracle_euler_matrix(0, 0, psi_deg, A);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Ainv[i * 3 + j] = A[j * 3 + i] * (double)padding_factor;
    int padF = pad_size / 2 + 1;
    int Fs = f2d_size / 2 + 1;
    int shift = -(int)((float)pad_size / 2.0);
    int max_r2 = r_max * r_max;
    for (int i = 0; i < f2d_size; i++) {
        int y, first_x;
        if (i <= r_max) {
            y = i;
            first_x = 0;
        } else if (i >= f2d_size - r_max) {
            y = i - f2d_size;
            first_x = 1;
        } else
            continue;
        int y2 = y * y;
        for (int x = first_x; x <= r_max; x++) {
            int r2 = x * x + y2;
            if (r2 > max_r2) continue;
            double vr = f2d_real[i * Fs + x], vi = f2d_imag[i * Fs + x];
            double w = Mweight ? Mweight[i * Fs + x] : 1.;
            if (!(w > 0.)) continue;
            double xp = Ainv[0] * x + Ainv[1] * y;
            double yp = Ainv[3] * x + Ainv[4] * y;
            int neg = 0;
            if (xp < 0) {
                xp = -xp;
                yp = -yp;
                neg = 1;
            }
            int x0 = (int)floor(xp);
            double fx = xp - x0;
            int y0 = (int)floor(yp);
            double fy = yp - y0;
            y0 -= shift;
            int y1 = y0 + 1;
            double mfx = 1. - fx, mfy = 1. - fy;
            double dd00 = mfy * mfx, dd01 = mfy * fx, dd10 = fy * mfx, dd11 = fy * fx;
            if (neg) vi = -1 * vi;
            double* t00 = bp_data + ((long)y0 * padF + x0) * 2;
            double* t10 = bp_data + ((long)y1 * padF + x0) * 2;
            t00[0] += dd00 * vr;
            t00[1] += dd00 * vi;
            t00[2] += dd01 * vr;
            t00[3] += dd01 * vi;
            t10[0] += dd10 * vr;
            t10[1] += dd10 * vi;
            t10[2] += dd11 * vr;
            t10[3] += dd11 * vi;
            double* w00 = bp_weight + (long)y0 * padF + x0;
            double* w10 = bp_weight + (long)y1 * padF + x0;
            w00[0] += dd00 * w;
            w00[1] += dd01 * w;
            w10[0] += dd10 * w;
            w10[1] += dd11 * w;
        }
    }
}

/* ---- findAllSignificantPoints selection, src/map2d_optimizer.cpp:1233-1263 ---- */
static int cmp_double(const void* a, const void* b) {
    double x = *(const double*)a, y = *(const double*)b;
    return (x > y) - (x < y);
}

void oracle_select_significant(long len, const double* w, double sum_weight, double adaptive_fraction,
                               double* significant_weight, double* nr_significant) {
    double* sorted = (double*)malloc(sizeof(double) * (len > 0 ? len : 1));
    long cnt = 0;
    for (long i = 0; i < len; i++)
        if (w[i] > 0.) sorted[cnt++] = w[i];
    qsort(sorted, (size_t)cnt, sizeof(double), cmp_double);
    double frac = 0., sig = 0.;
    long nsig = 0;
    for (long i = cnt - 1; i >= 0; i--) {
        nsig++;
        sig = sorted[i];
        frac += sig;
        if (frac > adaptive_fraction * sum_weight) break;
    }
    free(sorted);
    *significant_weight = sig;
    *nr_significant = (double)nsig;
}

/* MLModel::calculatePdfOffset, src/ml_model.h:231-242 */
static double pdf_offset(double ox, double oy, double px, double py, double sigma2_offset) {
    const double rome_pi = 3.14159265358979323846;
    double tdiff2 = (ox - px) * (ox - px) + (oy - py) * (oy - py);
    if (sigma2_offset < 0.0001) return (tdiff2 > 0.) ? 0. : 1.;
    return exp(tdiff2 / (-2. * sigma2_offset)) / (2. * rome_pi * sigma2_offset);
}

/* ---- the pool E-step, src/map2d_optimizer.cpp:802-854 ---- */
int oracle_map2d_estep_pool(const RomeMap2dPool* in, RomeMap2dPoolOut* out, int pad_size, int r_max,
                            int padding_factor, const double* proj_data, double* bp_data, double* bp_weight) {
    const int P = in->nr_images, K = in->nr_classes, ori = in->ori_size, cur = in->current_size;
    const int npsi = in->nr_psi, ntr = in->nr_trans, oriF = ori / 2 + 1;
    const int curF2 = cur * (cur / 2 + 1);
    const int npass = in->adaptive_oversampling > 0 ? 2 : 1;
    const int padF = pad_size / 2 + 1;
    const long vox = (long)pad_size * padF;
    int status = ROME_OK;

    /* Mcoarse_significant [P][K*npsi*ntr] and Rot_significant [K][npsi] */
    long ncoarse = (long)K * npsi * ntr;
    char* Mcoarse = (char*)calloc((size_t)P * ncoarse, 1);
    char* Rot_sig = (char*)calloc((size_t)K * npsi, 1);
    double *Minvsigma2 = NULL, *lctf = NULL, *shr = NULL, *shi = NULL, *Fref_r = NULL, *Fref_i = NULL, *Mweight = NULL;
    double* min_diff2 = (double*)malloc(sizeof(double) * P);
    double* sum_weight = (double*)malloc(sizeof(double) * P);
    double* sig_weight = (double*)malloc(sizeof(double) * P);
    int nor = 1, notr = 1, cs = cur;
    long xsize = 0;

    for (int ipass = 0; ipass < npass; ipass++) {
        cs = (ipass == 0 && in->adaptive_oversampling > 0) ? in->coarse_size : cur;
        int over = ipass == 0 ? 0 : in->adaptive_oversampling;
        nor = 1 << over;
        notr = 1 << (2 * over);
        int F = cs * (cs / 2 + 1);
        int T = ntr * notr;
        int nrot = npsi * nor;
        xsize = (long)K * nrot * T;
        const int* Mresol = ipass == 0 ? in->Mresol_coarse : in->Mresol_fine;
        const double* opsi = in->over_psi[ipass];
        const double* otx = in->over_trans_x[ipass];
        const double* oty = in->over_trans_y[ipass];

        free(Minvsigma2); free(lctf); free(shr); free(shi); free(Fref_r); free(Fref_i); free(Mweight);
        Minvsigma2 = (double*)malloc(sizeof(double) * P * F);
        lctf = (double*)malloc(sizeof(double) * P * F);
        shr = (double*)malloc(sizeof(double) * (long)P * T * F);
        shi = (double*)malloc(sizeof(double) * (long)P * T * F);
        Fref_r = (double*)calloc((size_t)K * nrot * F, sizeof(double));
        Fref_i = (double*)calloc((size_t)K * nrot * F, sizeof(double));
        Mweight = (double*)malloc(sizeof(double) * P * xsize);

        /* preShiftedImagesCtfsAndInvSigma2s, src/exp_model.cpp:935-1104 */
        double* wr = (double*)malloc(sizeof(double) * F);
        double* wi = (double*)malloc(sizeof(double) * F);
        for (int i = 0; i < P; i++) {
            window_ft(in->Fimg_real + (long)i * curF2, cur, wr, cs);
            window_ft(in->Fimg_imag + (long)i * curF2, cur, wi, cs);
            window_ft(in->Fctf + (long)i * curF2, cur, lctf + (long)i * F, cs);
            for (int t = 0; t < T; t++) {
                int itr = t / notr, iotr = t % notr;
                oracle_shift_image(wr, wi, shr + ((long)i * T + t) * F, shi + ((long)i * T + t) * F, cs,
                                   otx[itr * notr + iotr], oty[itr * notr + iotr], ori);
            }
            const double* s2 = in->sigma2_noise + (long)in->group[i] * oriF;
            for (int n = 0; n < F; n++) {
                int ires = Mresol[n];
                Minvsigma2[(long)i * F + n] = ires > 0 ? 1. / (in->sigma2_fudge * s2[ires]) : 0;
            }
        }
        free(wr);
        free(wi);

        /* getReferenceAllOrientations, src/map2d_optimizer.cpp:856-904 */
        for (int k = in->iclass_min; k <= in->iclass_max; k++)
            for (int ipsi = 0; ipsi < npsi; ipsi++) {
                if (in->pdf_class[k] <= 0.) continue;
                if (ipass == 0) Rot_sig[k * npsi + ipsi] = 1;
                else {
                    int any = 0;
                    long h0 = ((long)k * npsi + ipsi) * ntr;
                    for (int i = 0; i < P && !any; i++)
                        for (int h = 0; h < ntr; h++)
                            if (Mcoarse[(long)i * ncoarse + h0 + h]) { any = 1; break; }
                    Rot_sig[k * npsi + ipsi] = (char)any;
                }
            }
        for (int k = in->iclass_min; k <= in->iclass_max; k++)
            for (int ipsi = 0; ipsi < npsi; ipsi++)
                for (int ior = 0; ior < nor; ior++) {
                    if (!Rot_sig[k * npsi + ipsi] || in->pdf_direction[k] <= 0. || in->pdf_class[k] <= 0.) continue;
                    long r = (long)k * nrot + ipsi * nor + ior;
                    oracle_rotate2d(proj_data + (long)k * vox * 2, pad_size, r_max, padding_factor,
                                    opsi[ipsi * nor + ior], cs, Fref_r + r * F, Fref_i + r * F);
                }

        /* getAllSquaredDifferences, src/map2d_optimizer.cpp:907-1074 */
        for (long q = 0; q < (long)P * xsize; q++) Mweight[q] = (double)INT_MIN;
        int apply_ctf = in->do_ctf_correction && in->refs_are_ctf_corrected;
        double* frc_r = (double*)malloc(sizeof(double) * F);
        double* frc_i = (double*)malloc(sizeof(double) * F);
        for (int i = 0; i < P; i++) {
            double mind = DBL_MAX;
            const double* M = Minvsigma2 + (long)i * F;
            for (int k = in->iclass_min; k <= in->iclass_max; k++)
                for (int ipsi = 0; ipsi < npsi; ipsi++)
                    for (int ior = 0; ior < nor; ior++) {
                        if (!Rot_sig[k * npsi + ipsi] || in->pdf_direction[k] <= 0. || in->pdf_class[k] <= 0.)
                            continue;
                        long r = (long)k * nrot + ipsi * nor + ior;
                        const double* fr = Fref_r + r * F;
                        const double* fi = Fref_i + r * F;
                        for (int n = 0; n < F; n++) {
                            double c = apply_ctf ? lctf[(long)i * F + n] : 1.;
                            frc_r[n] = apply_ctf ? fr[n] * c : fr[n];
                            frc_i[n] = apply_ctf ? fi[n] * c : fi[n];
                        }
                        for (int itr = 0; itr < ntr; itr++)
                            for (int iotr = 0; iotr < notr; iotr++) {
                                if (ipass != 0 && !Mcoarse[(long)i * ncoarse + ((long)k * npsi + ipsi) * ntr + itr])
                                    continue;
                                int t = itr * notr + iotr;
                                const double* xr = shr + ((long)i * T + t) * F;
                                const double* xi = shi + ((long)i * T + t) * F;
                                double d2 = 0;
                                for (int n = 0; n < F; n++) {
                                    double dr = frc_r[n] - xr[n], di = frc_i[n] - xi[n];
                                    d2 += (dr * dr + di * di) * M[n];
                                }
                                d2 = (d2 + in->highres_Xi2[i]) / 2;
                                Mweight[(long)i * xsize + r * T + t] = d2;
                                if (d2 < mind) mind = d2;
                            }
                    }
            min_diff2[i] = mind;
        }
        free(frc_r);
        free(frc_i);
        if (out->diff2[ipass]) memcpy(out->diff2[ipass], Mweight, sizeof(double) * P * xsize);

        /* convertSquaredDifferencesToWeights, src/map2d_optimizer.cpp:1077-1224 */
        for (int i = 0; i < P; i++) {
            double sumw = 0., maxw = DBL_MIN;
            int bk = 0, bpsi = 0, bior = 0, btr = 0, botr = 0;
            for (int k = in->iclass_min; k <= in->iclass_max; k++)
                for (int ipsi = 0; ipsi < npsi; ipsi++)
                    for (int itr = 0; itr < ntr; itr++)
                        for (int ior = 0; ior < nor; ior++)
                            for (int iotr = 0; iotr < notr; iotr++) {
                                long r = (long)k * nrot + ipsi * nor + ior;
                                long idx = (long)i * xsize + r * T + itr * notr + iotr;
                                if (Mweight[idx] < 0.) {
                                    Mweight[idx] = 0.;
                                    continue;
                                }
                                double ox = in->trans_x[itr] + in->old_offsetx[i];
                                double oy = in->trans_y[itr] + in->old_offsety[i];
                                double po = pdf_offset(ox, oy, in->prior_offsetx_class[k], in->prior_offsety_class[k],
                                                       in->sigma2_offset);
                                double w = in->pdf_direction[k] * po;
                                double d = Mweight[idx] - min_diff2[i];
                                if (d > 700.) w = 0.;
                                else w *= exp(-d);
                                Mweight[idx] = w;
                                sumw += w;
                                if (w > maxw) {
                                    maxw = w;
                                    bk = k; bpsi = ipsi; bior = ior; btr = itr; botr = iotr;
                                }
                            }
            sum_weight[i] = sumw;
            if (out->pmax) out->pmax[i] = maxw / sumw;
            if (out->cls) out->cls[i] = bk + 1;
            if (out->psi) {
                double psi = opsi[bpsi * nor + bior];
                if (psi > 180.) psi -= 360.;
                if (psi < -180.) psi += 360.;
                out->psi[i] = psi;
            }
            if (out->xoff) out->xoff[i] = in->old_offsetx[i] + otx[btr * notr + botr];
            if (out->yoff) out->yoff[i] = in->old_offsety[i] + oty[btr * notr + botr];
        }
        if (out->weight[ipass]) memcpy(out->weight[ipass], Mweight, sizeof(double) * P * xsize);

        /* findAllSignificantPoints, src/map2d_optimizer.cpp:1226-1311 */
        for (int i = 0; i < P; i++) {
            double sw, ns;
            oracle_select_significant(xsize, Mweight + (long)i * xsize, sum_weight[i], in->adaptive_fraction, &sw, &ns);
            if (ipass == 0 && ns == 0) status = ROME_ERR_NUMERIC;
            if (ipass == 0) {
                if (out->nr_sign) out->nr_sign[i] = ns;
                for (long h = 0; h < xsize; h++) Mcoarse[(long)i * ncoarse + h] = Mweight[(long)i * xsize + h] >= sw;
            }
            sig_weight[i] = sw;
        }
        if (ipass == 0 && out->Mcoarse_significant) memcpy(out->Mcoarse_significant, Mcoarse, (size_t)P * ncoarse);
    }

    /* updateOtherParams, src/map2d_optimizer.cpp:1417-1663 (last pass, current_size) */
    {
        int F = cur * (cur / 2 + 1), T = ntr * notr, nrot = npsi * nor;
        int apply_ctf = in->do_ctf_correction && in->refs_are_ctf_corrected;
        const double* otx = in->over_trans_x[npass - 1];
        const double* oty = in->over_trans_y[npass - 1];
        double* wsn = (double*)calloc((size_t)P * F, sizeof(double));
        for (int i = 0; i < P; i++) {
            double norm_corr = 0.;
            for (int k = in->iclass_min; k <= in->iclass_max; k++)
                for (int ipsi = 0; ipsi < npsi; ipsi++)
                    for (int ior = 0; ior < nor; ior++) {
                        if (!Rot_sig[k * npsi + ipsi]) continue;
                        long r = (long)k * nrot + ipsi * nor + ior;
                        for (int t = 0; t < T; t++) {
                            double w = Mweight[(long)i * xsize + r * T + t];
                            if (!(w >= sig_weight[i])) continue;
                            w /= sum_weight[i];
                            double sum_wdiff2 = 0.;
                            for (int n = 0; n < F; n++) {
                                int ires = in->Mresol_fine[n];
                                if (ires > -1) {
                                    double c = apply_ctf ? lctf[(long)i * F + n] : 1.;
                                    double pr = apply_ctf ? Fref_r[r * F + n] * c : Fref_r[r * F + n];
                                    double pi = apply_ctf ? Fref_i[r * F + n] * c : Fref_i[r * F + n];
                                    double dr = pr - shr[((long)i * T + t) * F + n];
                                    double di = pi - shi[((long)i * T + t) * F + n];
                                    double wd = w * (dr * dr + di * di);
                                    wsn[(long)i * F + n] += wd;
                                    sum_wdiff2 += wd;
                                }
                            }
                            norm_corr += sum_wdiff2;
                        }
                    }
            if (out->wsum_norm_correction) out->wsum_norm_correction[i] = norm_corr;
        }
        for (int i = 0; i < P; i++) {
            double* dst = out->wsum_sigma2_noise + (long)in->group[i] * oriF;
            for (int n = 0; n < F; n++) {
                int ires = in->Mresol_fine[n];
                if (ires > -1) dst[ires] += wsn[(long)i * F + n];
            }
        }
        free(wsn);
        for (int i = 0; i < P; i++)
            for (int k = in->iclass_min; k <= in->iclass_max; k++)
                for (int ipsi = 0; ipsi < npsi; ipsi++)
                    for (int ior = 0; ior < nor; ior++)
                        for (int itr = 0; itr < ntr; itr++)
                            for (int iotr = 0; iotr < notr; iotr++) {
                                if (!Rot_sig[k * npsi + ipsi]) continue;
                                long r = (long)k * nrot + ipsi * nor + ior;
                                double w = Mweight[(long)i * xsize + r * T + itr * notr + iotr];
                                if (!(w >= sig_weight[i])) continue;
                                w /= sum_weight[i];
                                double tx = otx[itr * notr + iotr], ty = oty[itr * notr + iotr];
                                out->wsum_sumw_group[in->group[i]] += w;
                                out->wsum_pdf_class[k] += w;
                                out->wsum_pdf_direction[k] += w;
                                out->wsum_prior_offsetx_class[k] += w * (in->old_offsetx[i] + tx);
                                out->wsum_prior_offsety_class[k] += w * (in->old_offsety[i] + ty);
                                double ox = in->prior_offsetx_class[k] - in->old_offsetx[i] - tx;
                                double oy = in->prior_offsety_class[k] - in->old_offsety[i] - ty;
                                out->wsum_sigma2_offset[0] += w * (ox * ox + oy * oy);
                            }
    }

    /* backProjection, src/map2d_optimizer.cpp:1666-1873 */
    {
        int F = cur * (cur / 2 + 1), T = ntr * notr, nrot = npsi * nor;
        const double* otx = in->over_trans_x[npass - 1];
        const double* oty = in->over_trans_y[npass - 1];
        double* mctf = (double*)malloc(sizeof(double) * P * F);   /* ctf * Minvsigma2 */
        double* mctf2 = (double*)malloc(sizeof(double) * P * F);  /* ctf^2 * Minvsigma2 */
        double* nr = (double*)malloc(sizeof(double) * F);
        double* ni = (double*)malloc(sizeof(double) * F);
        for (int i = 0; i < P; i++) {
            double* M = Minvsigma2 + (long)i * F;
            M[0] = 1. / (in->sigma2_fudge * in->sigma2_noise[(long)in->group[i] * oriF + 0]);
            for (int n = 0; n < F; n++) {
                double m = in->do_map ? M[n] : 1.0;
                double c = in->do_ctf_correction ? lctf[(long)i * F + n] : 1.0;
                double mc = c * m;
                mctf[(long)i * F + n] = mc;
                mctf2[(long)i * F + n] = c * mc;
            }
            /* pregetShiftedImagesNomask on the nomask image times ctf*Minvsigma2 */
            for (int n = 0; n < F; n++) {
                nr[n] = in->Fimg_nomask_real[(long)i * curF2 + n] * mctf[(long)i * F + n];
                ni[n] = in->Fimg_nomask_imag[(long)i * curF2 + n] * mctf[(long)i * F + n];
            }
            for (int t = 0; t < T; t++) {
                int itr = t / notr, iotr = t % notr;
                oracle_shift_image(nr, ni, shr + ((long)i * T + t) * F, shi + ((long)i * T + t) * F, cur,
                                   otx[itr * notr + iotr], oty[itr * notr + iotr], ori);
            }
        }
        double* sl_r = (double*)malloc(sizeof(double) * F);
        double* sl_i = (double*)malloc(sizeof(double) * F);
        double* sl_w = (double*)malloc(sizeof(double) * F);
        for (int k = in->iclass_min; k <= in->iclass_max; k++)
            for (int ipsi = 0; ipsi < npsi; ipsi++)
                for (int ior = 0; ior < nor; ior++) {
                    if (!Rot_sig[k * npsi + ipsi]) continue;
                    long r = (long)k * nrot + ipsi * nor + ior;
                    memset(sl_r, 0, sizeof(double) * F);
                    memset(sl_i, 0, sizeof(double) * F);
                    memset(sl_w, 0, sizeof(double) * F);
                    for (int i = 0; i < P; i++)
                        for (int t = 0; t < T; t++) {
                            double w = Mweight[(long)i * xsize + r * T + t];
                            if (!(w >= sig_weight[i])) continue;
                            w /= sum_weight[i];
                            const double* xr = shr + ((long)i * T + t) * F;
                            const double* xi = shi + ((long)i * T + t) * F;
                            for (int n = 0; n < F; n++) {
                                sl_r[n] += xr[n] * w;
                                sl_i[n] += xi[n] * w;
                                sl_w[n] += mctf2[(long)i * F + n] * w;
                            }
                        }
                    oracle_backrotate2d(sl_r, sl_i, sl_w, cur, in->over_psi[npass - 1][ipsi * nor + ior], pad_size,
                                        r_max, padding_factor, bp_data + (long)k * vox * 2, bp_weight + (long)k * vox);
                }
        free(sl_r); free(sl_i); free(sl_w); free(mctf); free(mctf2); free(nr); free(ni);
    }

    for (int i = 0; i < P; i++) {
        if (out->min_diff2) out->min_diff2[i] = min_diff2[i];
        if (out->sum_weight) out->sum_weight[i] = sum_weight[i];
        if (out->significant_weight) out->significant_weight[i] = sig_weight[i];
        if (sum_weight[i] == 0) status = ROME_ERR_NUMERIC;
    }
    free(Minvsigma2); free(lctf); free(shr); free(shi); free(Fref_r); free(Fref_i); free(Mweight);
    free(min_diff2); free(sum_weight); free(sig_weight); free(Mcoarse); free(Rot_sig);
    return status;
}
