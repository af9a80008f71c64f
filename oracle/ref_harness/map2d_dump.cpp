// Reference harness for MAP2D (test infrastructure; links the reference's
// own objects from oracle/_ref/libromeref.a).
//
// It drives Map2dOptimizer_old exactly like apps/rome_map2d.cpp:27-139, runs
// the reference iterations 1..dump_iter-1 unchanged through iterate()
// (src/map2d_optimizer.cpp:456-565), and then performs iteration dump_iter
// step by step, calling the reference's own E-step functions in the order
// expectationSomeParticles() uses (src/map2d_optimizer.cpp:802-854).  After
// each step of the first pool it writes the arrays the GPU path must
// reproduce (named like the reference's DataStream checkpoints,
// src/debug.h).  Finally it dumps the M-step inputs (backprojector,
// wsums) and outputs (Irefs, tau2, sigma2, data_vs_prior) of
// maximization() (src/map2d_optimizer.cpp:1876-1981).
#include "map2d_optimizer.h"
#include "option.h"

#include <sys/stat.h>

#include <vector>

#include "dump.h"

using namespace Map2dOptimizer_old;

namespace {

template <typename V>
std::vector<double> flat2(V& arr, int n0, int n1) {
    std::vector<double> out((size_t)n0 * n1);
    for (int i = 0; i < n0; i++) {
        auto p = arr[i].wptr(n1);
        for (int j = 0; j < n1; j++) out[(size_t)i * n1 + j] = p[j];
    }
    return out;
}

void dump_model_sums(Dumper& d, const std::string& pre) {
    int K = nr_classes, G = mlModel.nr_groups, oF = mlModel.ori_Fsize;
    std::vector<double> s2n((size_t)G * oF);
    for (int g = 0; g < G; g++) {
        auto p = mlModel.wsum_sigma2_noise[g].wptr(oF);
        for (int n = 0; n < oF; n++) s2n[(size_t)g * oF + n] = p[n];
    }
    d.f64(pre + "wsum_sigma2_noise", s2n.data(), {G, oF});
    d.f64(pre + "wsum_pdf_class", mlModel.wsum_pdf_class.wptrAll(), {K});
    std::vector<double> pdir(K);
    for (int k = 0; k < K; k++) pdir[k] = mlModel.wsum_pdf_direction[k][0];
    d.f64(pre + "wsum_pdf_direction", pdir.data(), {K});
    d.f64(pre + "wsum_prior_offsetx_class", mlModel.wsum_prior_offsetx_class.wptrAll(), {K});
    d.f64(pre + "wsum_prior_offsety_class", mlModel.wsum_prior_offsety_class.wptrAll(), {K});
    d.scalar(pre + "wsum_sigma2_offset", mlModel.wsum_sigma2_offset);
    d.f64(pre + "wsum_sumw_group", mlModel.wsum_sumw_group.wptrAll(), {G});
    d.scalar(pre + "wsum_LL", mlModel.wsum_LL);
    d.scalar(pre + "wsum_ave_Pmax", mlModel.wsum_ave_Pmax);
    d.scalar(pre + "wsum_avg_norm_correction", mlModel.wsum_avg_norm_correction);
}

void dump_backprojectors(Dumper& d, const std::string& pre) {
    int K = nr_classes;
    int pad = mapModel.backprojector[0].pad_size, padF = mapModel.backprojector[0].pad_Fsize;
    size_t vox = (size_t)pad * padF;
    std::vector<double> data(K * vox * 2), weight(K * vox);
    for (int k = 0; k < K; k++) {
        auto dp = (double*)mapModel.backprojector[k].data.wptr();
        auto wp = mapModel.backprojector[k].weight.wptr();
        for (size_t i = 0; i < vox * 2; i++) data[k * vox * 2 + i] = dp[i];
        for (size_t i = 0; i < vox; i++) weight[k * vox + i] = wp[i];
    }
    d.f64(pre + "bp_data", data.data(), {K, pad, padF, 2});
    d.f64(pre + "bp_weight", weight.data(), {K, pad, padF});
}

void dump_pass_inputs(Dumper& d, int ipass) {
    std::string pre = "pass" + std::to_string(ipass) + "_";
    int npsi = exp_nr_psi, nor = exp_nr_over_rot, ntr = exp_nr_trans, notr = exp_nr_over_trans;
    std::vector<double> psi((size_t)npsi * nor), tx((size_t)ntr * notr), ty((size_t)ntr * notr);
    for (int i = 0; i < npsi; i++)
        for (int j = 0; j < nor; j++) psi[(size_t)i * nor + j] = samplingGrid.exp_over_psi[i][j];
    for (int i = 0; i < ntr; i++)
        for (int j = 0; j < notr; j++) {
            tx[(size_t)i * notr + j] = samplingGrid.exp_over_trans_x[i][j];
            ty[(size_t)i * notr + j] = samplingGrid.exp_over_trans_y[i][j];
        }
    d.f64(pre + "over_psi", psi.data(), {npsi, nor});
    d.f64(pre + "over_trans_x", tx.data(), {ntr, notr});
    d.f64(pre + "over_trans_y", ty.data(), {ntr, notr});
    d.iscalar(pre + "current_size", exp_current_size);
    int F = exp_current_size * (exp_current_size / 2 + 1);
    auto ms = flat2(exp_local_Minvsigma2s, exp_nr_images, F);
    d.f64(pre + "Minvsigma2", ms.data(), {exp_nr_images, F});
    auto ctf = flat2(exp_local_Fctfs, exp_nr_images, F);
    d.f64(pre + "local_Fctf", ctf.data(), {exp_nr_images, F});
    std::vector<double> sr((size_t)exp_nr_images * ntr * notr * F), si(sr.size());
    for (int i = 0; i < exp_nr_images; i++)
        for (int t = 0; t < ntr * notr; t++) {
            auto pr = exp_Fimgs_shifted_real.wptr(i, t, F);
            auto pi = exp_Fimgs_shifted_imag.wptr(i, t, F);
            for (int n = 0; n < F; n++) {
                sr[((size_t)i * ntr * notr + t) * F + n] = pr[n];
                si[((size_t)i * ntr * notr + t) * F + n] = pi[n];
            }
        }
    d.f64(pre + "Fimg_shifted_real", sr.data(), {exp_nr_images, ntr * notr, F});
    d.f64(pre + "Fimg_shifted_imag", si.data(), {exp_nr_images, ntr * notr, F});
}

}  // namespace

int main(int argc, char* argv[]) {
    Option option;
    option.addOption("-i", "Input STAR file");
    option.addOption("-dump_dir", "Directory for the dumped arrays");
    option.addOption("-K", "Number of classes");
    option.addOption("-iter", "Iteration to dump (>= 2)");
    option.addOption("-angpix", "Pixel size (A)");
    option.addOption("-tau2_fudge", "Regularisation parameter");
    option.addOption("-oversampling", "Adaptive oversampling order");
    option.addOption("-particle_diameter", "Particle diameter", "-1");
    option.addOption("-pool", "Pool size", "50");
    option.addOption("-random_seed", "Random seed", "33");
    option.addOption("-offset_step", "Offset step (pixels)", "2");
    option.addOption("-offset_range", "Offset range (pixels)", "10");
    option.addOption("-psi_step", "Psi step (degrees)", "10");
    option.addOption("-ctf", "CTF correction", "0");
    option.addOption("-norm", "Norm correction", "0");
    option.addOption("-zero_mask", "Zero mask", "0");
    option.addOption("-dump_pools", "Number of pools dumped step by step", "1");
    option.readCommandLine(argc, argv);

    std::string dump_dir = option.getStrOption("-dump_dir");
    mkdir(dump_dir.c_str(), 0755);
    Dumper d(dump_dir);

    star_fn = pathRemoveSuffix(option.getStrOption("-i")) + ".star";
    mrcs_dir = pathGetDir(star_fn);
    write_path = "NULL";
    write_fn = "NULL";
    nr_classes = option.getIntOption("-K");
    nr_pool = option.getIntOption("-pool");
    pixel_size = option.getFloatOption("-angpix");
    int dump_iter = option.getIntOption("-iter");
    random_seed = option.getIntOption("-random_seed");
    offset_step = option.getIntOption("-offset_step");
    offset_range = option.getIntOption("-offset_range");
    psi_step = option.getIntOption("-psi_step");
    tau2_fudge_factor = option.getFloatOption("-tau2_fudge");
    particle_diameter = option.getFloatOption("-particle_diameter");
    adaptive_oversampling = option.getIntOption("-oversampling");
    do_ctf_correction = option.getBoolOption("-ctf");
    only_flip_phases = false;
    ctf_phase_flipped = false;
    refs_are_ctf_corrected = false;
    intact_ctf_first_peak = false;
    do_norm_correction = option.getBoolOption("-norm");
    do_zero_mask = option.getBoolOption("-zero_mask");
    do_solvent = false;
    data_stream_in_fn = "NULL";
    data_stream_out_fn = "NULL";
    iter = 0;
    guidance_fn = "NULL";
    ref_fn = "NULL";
    int dump_pools = option.getIntOption("-dump_pools");
    if (dump_iter < 2) {
        std::cerr << "-iter must be >= 2" << std::endl;
        return 2;
    }

    setupMap2dOptimizer();
    readImages();
    Map2dOptimizer_old::prepare();

    // iterations 1 .. dump_iter-1: the reference driver, unchanged
    nr_iter = dump_iter - 1;
    Map2dOptimizer_old::iterate();
    nr_iter = dump_iter;
    iter = dump_iter;

    // ---- iteration dump_iter, step by step ----
    double ang = sampler2d.getAngularSampling();
    mapModel.updateImageSizeAndResolutionPointers(Npix_per_shell, Mresol_coarse, Mresol_fine, coarse_size, current_size,
                                                  adaptive_oversampling, ang, mlModel.ave_Pmax);
    prepareExpData();

    int K = nr_classes, G = mlModel.nr_groups, oF = mlModel.ori_Fsize;
    d.iscalar("ori_size", ori_size);
    d.iscalar("current_size", current_size);
    d.iscalar("coarse_size", coarse_size);
    d.iscalar("nr_classes", K);
    d.iscalar("nr_groups", G);
    d.iscalar("adaptive_oversampling", adaptive_oversampling);
    d.iscalar("do_ctf_correction", do_ctf_correction);
    d.iscalar("refs_are_ctf_corrected", refs_are_ctf_corrected);
    d.iscalar("do_norm_correction", do_norm_correction);
    d.iscalar("do_map", do_map);
    d.scalar("sigma2_fudge", sigma2_fudge);
    d.scalar("adaptive_fraction", adaptive_fraction);
    d.scalar("pixel_size", pixel_size);
    d.scalar("tau2_fudge_factor", tau2_fudge_factor);
    d.iscalar("gridding_nr_iter", gridding_nr_iter);
    d.iscalar("minres_map", mapModel.minres_map);
    d.iscalar("random_seed", random_seed);
    d.scalar("random_perturbation", sampler2d.random_perturbation);
    d.scalar("offset_step", sampler2d.offset_step);
    d.scalar("offset_range", sampler2d.offset_range);
    d.scalar("psi_step", sampler2d.psi_step);
    {
        int ntr = (int)sampler2d.NrTrans(0);
        std::vector<double> tx(ntr), ty(ntr);
        for (int t = 0; t < ntr; t++) sampler2d.getTranslation(t, tx[t], ty[t]);
        d.f64("trans_x", tx.data(), {ntr});
        d.f64("trans_y", ty.data(), {ntr});
    }
    d.i32("Npix_per_shell", Npix_per_shell.wptrAll(), {oF});
    d.i32("Mresol_fine", Mresol_fine.wptrAll(), {current_size * (current_size / 2 + 1)});
    d.i32("Mresol_coarse", Mresol_coarse.wptrAll(), {coarse_size * (coarse_size / 2 + 1)});
    // model state the E-step reads
    std::vector<double> s2((size_t)G * oF);
    for (int g = 0; g < G; g++)
        for (int n = 0; n < oF; n++) s2[(size_t)g * oF + n] = mlModel.sigma2_noise[g][n];
    d.f64("sigma2_noise", s2.data(), {G, oF});
    d.f64("pdf_class", mlModel.pdf_class.wptrAll(), {K});
    std::vector<double> pdir(K);
    for (int k = 0; k < K; k++) pdir[k] = mlModel.pdf_direction[k][0];
    d.f64("pdf_direction", pdir.data(), {K});
    d.f64("prior_offsetx_class", mlModel.prior_offsetx_class.wptrAll(), {K});
    d.f64("prior_offsety_class", mlModel.prior_offsety_class.wptrAll(), {K});
    d.scalar("sigma2_offset", mlModel.sigma2_offset);
    d.scalar("avg_norm_correction", mlModel.avg_norm_correction);
    // class references and their Fourier-space projector maps
    {
        int pad = mapModel.projector[0].pad_size, padF = mapModel.projector[0].pad_Fsize;
        size_t vox = (size_t)pad * padF;
        std::vector<double> pdata(K * vox * 2), irefs((size_t)K * ori_size * ori_size);
        for (int k = 0; k < K; k++) {
            auto p = (double*)mapModel.projector[k].data.wptr();
            for (size_t i = 0; i < vox * 2; i++) pdata[k * vox * 2 + i] = p[i];
            auto r = mapModel.Irefs[k].wptr();
            for (int i = 0; i < ori_size * ori_size; i++) irefs[(size_t)k * ori_size * ori_size + i] = r[i];
        }
        d.f64("projector_data", pdata.data(), {K, pad, padF, 2});
        d.iscalar("projector_r_max", mapModel.projector[0].r_max);
        d.iscalar("projector_pad_size", pad);
        d.iscalar("projector_padding_factor", mapModel.projector[0].padding_factor);
        d.f64("Irefs_before", irefs.data(), {K, ori_size, ori_size});
        std::vector<double> tau2((size_t)K * oF), dvp((size_t)K * oF);
        for (int k = 0; k < K; k++)
            for (int n = 0; n < oF; n++) {
                tau2[(size_t)k * oF + n] = mlModel.tau2_class[k][n];
                dvp[(size_t)k * oF + n] = mlModel.data_vs_prior_class[k][n];
            }
        d.f64("tau2_class_before", tau2.data(), {K, oF});
        d.f64("data_vs_prior_before", dvp.data(), {K, oF});
    }

    // ---- expectation() with the first pools dumped stage by stage ----
    int nr_done = 0, pool_index = 0;
    while (nr_done < nr_local_images) {
        int first = first_local_image + nr_done;
        int last = std::min(first_local_image + nr_local_images - 1, first + nr_pool - 1);
        exp_first_image = first;
        exp_last_image = last;
        exp_nr_images = last - first + 1;
        exp_iclass_min = 0;
        exp_iclass_max = nr_classes - 1;
        for (int i = 0; i < exp_nr_images; i++) {
            auto dst = exp_imgs[i].wptr(ori_size * ori_size);
            auto src = images[(first - first_local_image) + i].wptrAll();
            for (int j = 0; j < ori_size * ori_size; j++) dst[j] = src[j];
            exp_metadata[i] = metadata[i + first];
        }
        particleModel.prepare(exp_imgs, exp_metadata, exp_first_image, exp_nr_images);
        particleModel.setFourierTransforms(exp_power_imgs, exp_highres_Xi2_imgs, exp_old_offsetx, exp_old_offsety, mlModel,
                                           do_ctf_correction);
        if (pool_index < dump_pools) {
            std::string pp = "pool" + std::to_string(pool_index) + "_";
            int P = exp_nr_images, Ff = current_size * (current_size / 2 + 1);
            d.iscalar(pp + "nr_images", P);
            d.iscalar(pp + "first_image", first);
            auto a = flat2(particleModel.Fimages_mask_fine_real, P, Ff);
            d.f64(pp + "Fimg_real", a.data(), {P, Ff});
            a = flat2(particleModel.Fimages_mask_fine_imag, P, Ff);
            d.f64(pp + "Fimg_imag", a.data(), {P, Ff});
            a = flat2(particleModel.Fimages_nomask_real, P, Ff);
            d.f64(pp + "Fimg_nomask_real", a.data(), {P, Ff});
            a = flat2(particleModel.Fimages_nomask_imag, P, Ff);
            d.f64(pp + "Fimg_nomask_imag", a.data(), {P, Ff});
            a = flat2(particleModel.Fctfs, P, Ff);
            d.f64(pp + "Fctf", a.data(), {P, Ff});
            a = flat2(exp_power_imgs, P, oF);
            d.f64(pp + "power_imgs", a.data(), {P, oF});
            d.f64(pp + "highres_Xi2", exp_highres_Xi2_imgs.wptrAll(), {P});
            d.f64(pp + "old_offsetx", exp_old_offsetx.wptrAll(), {P});
            d.f64(pp + "old_offsety", exp_old_offsety.wptrAll(), {P});
            std::vector<int> grp(P);
            std::vector<double> norm(P);
            for (int i = 0; i < P; i++) {
                grp[i] = exp_metadata[i].GROUP_NO - 1;
                norm[i] = exp_metadata[i].NORM;
            }
            d.i32(pp + "group", grp.data(), {P});
            d.f64(pp + "norm_in", norm.data(), {P});
            // inputs of the image preparation (ParticleModel::setFourierTransforms,
            // src/exp_model.h:397-640): the pool's images as read, the metadata it uses
            {
                const int o2 = ori_size * ori_size;
                std::vector<double> raw((size_t)P * o2);
                for (int i = 0; i < P; i++) {
                    auto src = images[(first - first_local_image) + i].wptrAll();
                    for (int j = 0; j < o2; j++) raw[(size_t)i * o2 + j] = src[j];
                }
                d.f64(pp + "raw_images", raw.data(), {P, ori_size, ori_size});
                std::vector<double> meta((size_t)P * 10);
                for (int i = 0; i < P; i++) {
                    const auto& m = exp_metadata[i];
                    const double v[10] = {m.NORM,          m.XOFF,          m.YOFF,   m.CTF_DEFOCUS_U, m.CTF_DEFOCUS_V,
                                          m.CTF_DEFOCUS_ANGLE, m.CTF_VOLTAGE, m.CTF_CS, m.CTF_Q0,        m.CTF_BFAC};
                    for (int q = 0; q < 10; q++) meta[(size_t)i * 10 + q] = v[q];
                }
                d.f64(pp + "prep_metadata", meta.data(), {P, 10});
                if (pool_index == 0) {
                    d.scalar("prep_avg_norm_correction", mlModel.avg_norm_correction);
                    d.scalar("prep_pixel_size", particleModel.pixel_size);
                    d.scalar("prep_particle_diameter", particleModel.particle_diameter);
                    d.iscalar("prep_width_mask_edge", particleModel.width_mask_edge);
                    d.scalar("prep_sigma2_fudge", particleModel.sigma2_fudge);
                    d.iscalar("prep_random_seed", particleModel.random_seed);
                    d.iscalar("prep_do_norm_correction", particleModel.do_norm_correction);
                    d.iscalar("prep_do_zero_mask", particleModel.do_zero_mask);
                    d.iscalar("prep_only_flip_phases", particleModel.only_flip_phases);
                    d.iscalar("prep_ctf_phase_flipped", particleModel.ctf_phase_flipped);
                    d.iscalar("prep_intact_ctf_first_peak", particleModel.intact_ctf_first_peak);
                }
            }

            // the stages of expectationSomeParticles()
            int npass = adaptive_oversampling > 0 ? 2 : 1;
            for (exp_ipass = 0; exp_ipass < npass; exp_ipass++) {
                std::string ps = pp + "pass" + std::to_string(exp_ipass) + "_";
                exp_current_size = (exp_ipass == 0 && adaptive_oversampling > 0) ? coarse_size : current_size;
                exp_current_oversampling = (exp_ipass == 0) ? 0 : adaptive_oversampling;
                samplingGrid.computeGrid2D(sampler2d, exp_current_oversampling);
                exp_nr_over_rot = samplingGrid.exp_nr_over_rot();
                exp_nr_over_trans = samplingGrid.exp_nr_over_trans();
                particleModel.preShiftedImagesCtfsAndInvSigma2s(
                    exp_Fimgs_shifted_real, exp_Fimgs_shifted_imag, exp_local_Minvsigma2s, exp_local_sqrtXi2,
                    exp_local_Fctfs, exp_current_size, false, exp_ipass == 0, samplingGrid, mlModel, Mresol_coarse,
                    Mresol_fine);
                if (pool_index == 0) dump_pass_inputs(d, exp_ipass);
                getReferenceAllOrientations();
                {
                    int Fc = exp_current_size * (exp_current_size / 2 + 1);
                    int nrot = exp_nr_psi * exp_nr_over_rot;
                    std::vector<double> rr((size_t)K * nrot * Fc), ri(rr.size());
                    for (int k = 0; k < K; k++)
                        for (int r = 0; r < nrot; r++) {
                            auto pr = exp_Frefs_Rot_real.wptr(k, r, Fc);
                            auto pi = exp_Frefs_Rot_imag.wptr(k, r, Fc);
                            for (int n = 0; n < Fc; n++) {
                                rr[((size_t)k * nrot + r) * Fc + n] = pr[n];
                                ri[((size_t)k * nrot + r) * Fc + n] = pi[n];
                            }
                        }
                    d.f64(ps + "Fref_real", rr.data(), {K, nrot, Fc});
                    d.f64(ps + "Fref_imag", ri.data(), {K, nrot, Fc});
                    std::vector<char> rs((size_t)K * exp_nr_psi);
                    for (int k = 0; k < K; k++)
                        for (int r = 0; r < exp_nr_psi; r++) rs[(size_t)k * exp_nr_psi + r] = exp_Rot_significant[k][r];
                    d.i8(ps + "Rot_significant", rs.data(), {K, exp_nr_psi});
                }
                getAllSquaredDifferences();
                d.f64(ps + "diff2", exp_Mweight, {P, exp_Mweight_xsize});
                d.f64(ps + "min_diff2", exp_min_diff2.wptrAll(), {P});
                convertSquaredDifferencesToWeights();
                d.f64(ps + "weight", exp_Mweight, {P, exp_Mweight_xsize});
                d.f64(ps + "sum_weight", exp_sum_weight.wptrAll(), {P});
                findAllSignificantPoints();
                d.f64(ps + "significant_weight", exp_significant_weight.wptrAll(), {P});
                std::vector<double> pm(P), psi(P), xo(P), yo(P), ns(P);
                std::vector<int> cl(P);
                for (int i = 0; i < P; i++) {
                    pm[i] = exp_metadata[i].PMAX;
                    psi[i] = exp_metadata[i].PSI;
                    xo[i] = exp_metadata[i].XOFF;
                    yo[i] = exp_metadata[i].YOFF;
                    ns[i] = exp_metadata[i].NR_SIGN;
                    cl[i] = exp_metadata[i].CLASS;
                }
                d.f64(ps + "pmax", pm.data(), {P});
                d.f64(ps + "psi", psi.data(), {P});
                d.f64(ps + "xoff", xo.data(), {P});
                d.f64(ps + "yoff", yo.data(), {P});
                d.f64(ps + "nr_sign", ns.data(), {P});
                d.i32(ps + "class", cl.data(), {P});
                if (exp_ipass == 0) {
                    int nc = (int)exp_Mcoarse_significant[0].size();
                    std::vector<char> mc((size_t)P * nc);
                    for (int i = 0; i < P; i++)
                        for (int j = 0; j < nc; j++) mc[(size_t)i * nc + j] = exp_Mcoarse_significant[i][j];
                    d.i8(ps + "Mcoarse_significant", mc.data(), {P, nc});
                }
            }
            exp_current_size = current_size;
            updateOtherParams();
            d.f64(pp + "wsum_norm_correction", exp_wsum_norm_correction.wptrAll(), {P});
            dump_model_sums(d, pp + "after_update_");
            backProjection();
            if (pool_index == 0) dump_backprojectors(d, pp + "after_bp_");
            storeWeightedSums();
            std::vector<double> dll(P), nrm(P);
            for (int i = 0; i < P; i++) {
                dll[i] = exp_metadata[i].DLL;
                nrm[i] = exp_metadata[i].NORM;
            }
            d.f64(pp + "dLL", dll.data(), {P});
            d.f64(pp + "norm_out", nrm.data(), {P});
            dump_model_sums(d, pp + "after_store_");
        } else {
            expectationSomeParticles();
        }
        hiddenVarMonitor.monitorHiddenVariableChanges(sampler2d, metadata, first, &exp_metadata[0], exp_nr_images);
        for (int i = 0; i < exp_nr_images; i++) metadata[i + first] = exp_metadata[i];
        nr_done += last - first + 1;
        pool_index++;
    }

    // ---- M-step inputs and outputs ----
    dump_model_sums(d, "iter_");
    dump_backprojectors(d, "iter_");
    maximization();
    {
        std::vector<double> irefs((size_t)K * ori_size * ori_size), tau2((size_t)K * oF), sig((size_t)K * oF),
            dvp((size_t)K * oF);
        for (int k = 0; k < K; k++) {
            auto r = mapModel.Irefs[k].wptr();
            for (int i = 0; i < ori_size * ori_size; i++) irefs[(size_t)k * ori_size * ori_size + i] = r[i];
            for (int n = 0; n < oF; n++) {
                tau2[(size_t)k * oF + n] = mlModel.tau2_class[k][n];
                sig[(size_t)k * oF + n] = mlModel.sigma2_class[k][n];
                dvp[(size_t)k * oF + n] = mlModel.data_vs_prior_class[k][n];
            }
        }
        d.f64("Irefs_after", irefs.data(), {K, ori_size, ori_size});
        d.f64("tau2_class_after", tau2.data(), {K, oF});
        d.f64("sigma2_class_after", sig.data(), {K, oF});
        d.f64("data_vs_prior_after", dvp.data(), {K, oF});
        d.f64("pdf_class_after", mlModel.pdf_class.wptrAll(), {K});
        // the rest of the model as maximizationOtherParameters (map2d_optimizer.cpp:1984-2045) left it
        d.f64("sigma2_noise_after", flat2(mlModel.sigma2_noise, G, oF).data(), {G, oF});
        std::vector<double> pdir(K);
        for (int k = 0; k < K; k++) pdir[k] = mlModel.pdf_direction[k][0];
        d.f64("pdf_direction_after", pdir.data(), {K});
        d.f64("prior_offsetx_class_after", mlModel.prior_offsetx_class.wptrAll(), {K});
        d.f64("prior_offsety_class_after", mlModel.prior_offsety_class.wptrAll(), {K});
        d.scalar("sigma2_offset_after", mlModel.sigma2_offset);
        d.scalar("avg_norm_correction_after", mlModel.avg_norm_correction);
        d.scalar("LL_after", mlModel.LL);
        d.scalar("ave_Pmax_after", mlModel.ave_Pmax);
        d.iscalar("refs_are_ctf_corrected_after", refs_are_ctf_corrected);
    }
    std::cout << "map2d_dump: done" << std::endl;
    return 0;
}
