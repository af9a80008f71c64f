// Reference harness for MAP3D (test infrastructure; links the reference's
// own objects from oracle/_ref/libromeref.a).
//
// It drives Map3dOptimizer_old like apps/rome_map3d.cpp:27-139, runs the
// reference iterations 1..dump_iter-1 unchanged through iterate()
// (src/map3d_optimizer.cpp:519-612), and then performs iteration dump_iter
// step by step, calling the reference's own E-step functions in the order
// expectationSomeParticles() uses (src/map3d_optimizer.cpp:883-953).  For
// the first pool it writes every stage's inputs and outputs: the sampling
// tables the pass used (samplingGrid.setOrientation, exp_over_trans_x/y),
// shifted images, Minvsigma2, CTF, the sparse diff2 / weight lists of
// Exp_Mweight_old, metadata, Mcoarse/Rot significance, the wsums after
// updateOtherParams, the backprojectors after backProjection, and finally
// the M-step inputs/outputs of maximization()
// (src/map3d_optimizer.cpp:2507-2617).
#include "map3d_optimizer.h"
#include "option.h"

#include <sys/stat.h>

#include <vector>

#include "dump.h"

// defined in src/map3d_optimizer.cpp:46,71-72 but not declared in its header
namespace Map3dOptimizer_old {
extern Images images;
extern Exp_Mweight_old exp_Mweight_coarse;
extern Exp_Mweight_old exp_Mweight_fine;
}  // namespace Map3dOptimizer_old

using namespace Map3dOptimizer_old;

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
    int K = nr_classes, G = mlModel.nr_groups, oF = mlModel.ori_Fsize, ND = exp_nr_dir;
    std::vector<double> s2n((size_t)G * oF);
    for (int g = 0; g < G; g++) {
        auto p = mlModel.wsum_sigma2_noise[g].wptr(oF);
        for (int n = 0; n < oF; n++) s2n[(size_t)g * oF + n] = p[n];
    }
    d.f64(pre + "wsum_sigma2_noise", s2n.data(), {G, oF});
    d.f64(pre + "wsum_pdf_class", mlModel.wsum_pdf_class.wptrAll(), {K});
    std::vector<double> pdir((size_t)K * ND);
    for (int k = 0; k < K; k++) {
        auto p = mlModel.wsum_pdf_direction[k].wptr(ND);
        for (int j = 0; j < ND; j++) pdir[(size_t)k * ND + j] = p[j];
    }
    d.f64(pre + "wsum_pdf_direction", pdir.data(), {K, ND});
    d.scalar(pre + "wsum_sigma2_offset", mlModel.wsum_sigma2_offset);
    d.f64(pre + "wsum_sumw_group", mlModel.wsum_sumw_group.wptrAll(), {G});
    d.scalar(pre + "wsum_LL", mlModel.wsum_LL);
    d.scalar(pre + "wsum_ave_Pmax", mlModel.wsum_ave_Pmax);
    d.scalar(pre + "wsum_avg_norm_correction", mlModel.wsum_avg_norm_correction);
    if (do_scale_correction) {
        std::vector<double> xa((size_t)G * oF), aa((size_t)G * oF);
        for (int g = 0; g < G; g++) {
            auto px = mlModel.wsum_signal_product_spectra[g].wptr(oF);
            auto pa = mlModel.wsum_reference_power_spectra[g].wptr(oF);
            for (int n = 0; n < oF; n++) {
                xa[(size_t)g * oF + n] = px[n];
                aa[(size_t)g * oF + n] = pa[n];
            }
        }
        d.f64(pre + "wsum_signal_product_spectra", xa.data(), {G, oF});
        d.f64(pre + "wsum_reference_power_spectra", aa.data(), {G, oF});
    }
}

void dump_backprojectors(Dumper& d, const std::string& pre) {
    int K = nr_classes;
    int pad = mapModel.backprojector[0].pad_size, padF = mapModel.backprojector[0].pad_Fsize;
    size_t vox = (size_t)pad * pad * padF;
    std::vector<double> data(K * vox * 2), weight(K * vox);
    for (int k = 0; k < K; k++) {
        auto dp = (double*)mapModel.backprojector[k].data.wptr();
        auto wp = mapModel.backprojector[k].weight.wptr();
        for (size_t i = 0; i < vox * 2; i++) data[k * vox * 2 + i] = dp[i];
        for (size_t i = 0; i < vox; i++) weight[k * vox + i] = wp[i];
    }
    d.f64(pre + "bp_data", data.data(), {K, pad, pad, padF, 2});
    d.f64(pre + "bp_weight", weight.data(), {K, pad, pad, padF});
}

// the sampling tables of the current pass and its per-particle inputs
bool g_light = false;

void dump_pass_inputs(Dumper& d, const std::string& pre) {
    int nd = exp_nr_dir, npsi = exp_nr_psi, nor = exp_nr_over_rot, ntr = exp_nr_trans, notr = exp_nr_over_trans;
    std::vector<double> ang((size_t)nd * npsi * nor * 3);
    for (int i = 0; i < nd; i++)
        for (int p = 0; p < npsi; p++) {
            FDOUBLE *r, *t, *s;
            samplingGrid.setOrientation(sampler3d, exp_current_oversampling, i, p, r, t, s);
            for (int o = 0; o < nor; o++) {
                size_t b = (((size_t)i * npsi + p) * nor + o) * 3;
                ang[b] = r[o];
                ang[b + 1] = t[o];
                ang[b + 2] = s[o];
            }
        }
    d.f64(pre + "angles", ang.data(), {nd, npsi, nor, 3});
    std::vector<double> tx((size_t)ntr * notr), ty((size_t)ntr * notr);
    for (int i = 0; i < ntr; i++)
        for (int j = 0; j < notr; j++) {
            tx[(size_t)i * notr + j] = samplingGrid.exp_over_trans_x[i][j];
            ty[(size_t)i * notr + j] = samplingGrid.exp_over_trans_y[i][j];
        }
    d.f64(pre + "over_trans_x", tx.data(), {ntr, notr});
    d.f64(pre + "over_trans_y", ty.data(), {ntr, notr});
    d.iscalar(pre + "current_size", exp_current_size);
    int F = exp_current_size * (exp_current_size / 2 + 1);
    auto ms = flat2(exp_local_Minvsigma2s, exp_nr_images, F);
    d.f64(pre + "Minvsigma2", ms.data(), {exp_nr_images, F});
    auto ctf = flat2(exp_local_Fctfs, exp_nr_images, F);
    d.f64(pre + "local_Fctf", ctf.data(), {exp_nr_images, F});
    d.f64(pre + "local_sqrtXi2", exp_local_sqrtXi2.wptrAll(), {exp_nr_images});
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
    if (!g_light) {
        d.f64(pre + "Fimg_shifted_real", sr.data(), {exp_nr_images, ntr * notr, F});
        d.f64(pre + "Fimg_shifted_imag", si.data(), {exp_nr_images, ntr * notr, F});
    }
}

// Exp_Mweight_old as flat lists: count[P][K][ndir][npsi], then (ihidden, value)
// concatenated in that loop order (the order every reference consumer walks)
void dump_mweight(Dumper& d, const std::string& pre, Exp_Mweight_old& mw) {
    int P = exp_nr_images, K = nr_classes, nd = exp_nr_dir, np = exp_nr_psi;
    std::vector<int> cnt((size_t)P * K * nd * np), ih;
    std::vector<double> val;
    size_t c = 0;
    for (int i = 0; i < P; i++)
        for (int k = 0; k < K; k++)
            for (int j = 0; j < nd; j++)
                for (int p = 0; p < np; p++) {
                    auto& v = mw.wptr_sparse(i, k, j, p);
                    cnt[c++] = (int)v.size();
                    for (auto& e : v) {
                        ih.push_back(e.first);
                        val.push_back(e.second);
                    }
                }
    d.i32(pre + "count", cnt.data(), {P, K, nd, np});
    int n = (int)ih.size();
    d.i32(pre + "ihidden", ih.data(), {n});
    d.f64(pre + "value", val.data(), {n});
}

void dump_metadata(Dumper& d, const std::string& pre) {
    int P = exp_nr_images;
    std::vector<double> pm(P), rot(P), tilt(P), psi(P), xo(P), yo(P), ns(P);
    std::vector<int> cl(P);
    for (int i = 0; i < P; i++) {
        pm[i] = exp_metadata[i].PMAX;
        rot[i] = exp_metadata[i].ROT;
        tilt[i] = exp_metadata[i].TILT;
        psi[i] = exp_metadata[i].PSI;
        xo[i] = exp_metadata[i].XOFF;
        yo[i] = exp_metadata[i].YOFF;
        ns[i] = exp_metadata[i].NR_SIGN;
        cl[i] = exp_metadata[i].CLASS;
    }
    d.f64(pre + "pmax", pm.data(), {P});
    d.f64(pre + "rot", rot.data(), {P});
    d.f64(pre + "tilt", tilt.data(), {P});
    d.f64(pre + "psi", psi.data(), {P});
    d.f64(pre + "xoff", xo.data(), {P});
    d.f64(pre + "yoff", yo.data(), {P});
    d.f64(pre + "nr_sign", ns.data(), {P});
    d.i32(pre + "class", cl.data(), {P});
}

}  // namespace

int main(int argc, char* argv[]) {
    Option option;
    option.addOption("-i", "Input STAR file");
    option.addOption("-ref", "Reference volume (MRC)");
    option.addOption("-dump_dir", "Directory for the dumped arrays");
    option.addOption("-K", "Number of classes");
    option.addOption("-iter", "Iteration to dump (>= 2)");
    option.addOption("-angpix", "Pixel size (A)");
    option.addOption("-ini_high", "Initial low-pass resolution (A)");
    option.addOption("-tau2_fudge", "Regularisation parameter");
    option.addOption("-oversampling", "Adaptive oversampling order (>= 1)");
    option.addOption("-healpix_order", "HEALPix order");
    option.addOption("-particle_diameter", "Particle diameter", "-1");
    option.addOption("-pool", "Pool size", "50");
    option.addOption("-random_seed", "Random seed", "33");
    option.addOption("-offset_step", "Offset step (pixels)", "2");
    option.addOption("-offset_range", "Offset range (pixels)", "10");
    option.addOption("-ctf", "CTF correction", "0");
    option.addOption("-norm", "Norm correction", "0");
    option.addOption("-scale", "Scale correction", "0");
    option.addOption("-firstiter_cc", "CC in the first iteration", "0");
    option.addOption("-always_cc", "CC in every iteration", "0");
    option.addOption("-dump_pools", "Number of pools dumped step by step", "1");
    option.addOption("-uniform_directions", "Reset pdf_direction to uniform before the dumped iteration", "0");
    option.addOption("-full_size", "Run the dumped iteration at the full image size (current resolution = Nyquist)", "0");
    option.addOption("-light", "Skip the per-translation shifted images and the input maps (large at 128^2)", "0");
    option.addOption("-skip_mstep", "Stop after dumping the M-step inputs (no maximization)", "0");
    option.readCommandLine(argc, argv);

    std::string dump_dir = option.getStrOption("-dump_dir");
    mkdir(dump_dir.c_str(), 0755);
    Dumper d(dump_dir);

    star_fn = pathRemoveSuffix(option.getStrOption("-i")) + ".star";
    write_path = "NULL";
    write_fn = "NULL";
    ref_fn = option.getStrOption("-ref");
    nr_classes = option.getIntOption("-K");
    nr_pool = option.getIntOption("-pool");
    pixel_size = option.getFloatOption("-angpix");
    int dump_iter = option.getIntOption("-iter");
    random_seed = option.getIntOption("-random_seed");
    offset_step = option.getIntOption("-offset_step");
    offset_range = option.getIntOption("-offset_range");
    do_ctf_correction = option.getBoolOption("-ctf");
    only_flip_phases = false;
    ctf_phase_flipped = false;
    refs_are_ctf_corrected = false;
    intact_ctf_first_peak = false;
    ini_high = option.getFloatOption("-ini_high");
    adaptive_oversampling = option.getIntOption("-oversampling");
    sampler3d_healpix_order = option.getIntOption("-healpix_order");
    tau2_fudge_factor = option.getFloatOption("-tau2_fudge");
    sampler3d_fn_sym = "C1";
    particle_diameter = option.getFloatOption("-particle_diameter");
    do_firstiter_cc = option.getBoolOption("-firstiter_cc");
    do_always_cc = option.getBoolOption("-always_cc");
    do_scale_correction = option.getBoolOption("-scale");
    do_norm_correction = option.getBoolOption("-norm");
    do_zero_mask = false;
    do_solvent = false;
    do_map = true;
    mask_fn = "NULL";
    data_stream_in_fn = "NULL";
    data_stream_out_fn = "NULL";
    continue_fn = "NULL";
    guidance_fn = "NULL";
    iter = 0;
    int dump_pools = option.getIntOption("-dump_pools");
    g_light = option.getBoolOption("-light");
    if (dump_iter < 2 || adaptive_oversampling < 1) {
        std::cerr << "-iter must be >= 2 and -oversampling >= 1" << std::endl;
        return 2;
    }

    Map3dOptimizer_old::setupMLoptimizer();
    Map3dOptimizer_old::prepare();

    // iterations 1 .. dump_iter-1: the reference driver, unchanged
    nr_iter = dump_iter - 1;
    Map3dOptimizer_old::iterate();
    nr_iter = dump_iter;
    iter = dump_iter;

    // A handful of particles leaves most directions with zero prior after one
    // iteration; optionally start the dumped iteration from the uniform
    // prior MLModel::initialize sets (src/ml_model.cpp:58) so that every
    // direction is searched.
    if (option.getBoolOption("-uniform_directions"))
        for (int k = 0; k < nr_classes; k++)
            for (int j = 0; j < sampler3d.NrDir(); j++)
                mlModel.pdf_direction[k][j] = 1. / ((double)nr_classes * sampler3d.NrDir());

    // Optionally run the dumped iteration at the full image size, the size
    // a converged refinement reaches (current_size = ori_size, projectors
    // padded to 2*(2*ori/2+1)+1), whatever resolution the short run reached.
    if (option.getBoolOption("-full_size")) mapModel.current_resolution = 1. / (2. * pixel_size);

    // ---- iteration dump_iter, step by step (iterate() body) ----
    double ang = sampler3d.getAngularSampling();
    mapModel.updateImageSizeAndResolutionPointers(Npix_per_shell, Mresol_coarse, Mresol_fine, coarse_size, current_size,
                                                  adaptive_oversampling, ang, mlModel.ave_Pmax);
    prepareExpData();

    int K = nr_classes, G = mlModel.nr_groups, oF = mlModel.ori_Fsize, ND = exp_nr_dir;
    d.iscalar("ori_size", ori_size);
    d.iscalar("current_size", current_size);
    d.iscalar("coarse_size", coarse_size);
    d.iscalar("nr_classes", K);
    d.iscalar("nr_groups", G);
    d.iscalar("nr_dir", ND);
    d.iscalar("nr_psi", exp_nr_psi);
    d.iscalar("nr_trans", exp_nr_trans);
    d.iscalar("healpix_order", sampler3d_healpix_order);
    d.iscalar("adaptive_oversampling", adaptive_oversampling);
    d.iscalar("do_ctf_correction", do_ctf_correction);
    d.iscalar("refs_are_ctf_corrected", refs_are_ctf_corrected);
    d.iscalar("do_scale_correction", do_scale_correction);
    d.iscalar("do_norm_correction", do_norm_correction);
    d.iscalar("do_map", do_map);
    d.iscalar("do_cross_correlation", (iter == 1 && do_firstiter_cc) || do_always_cc);
    d.scalar("sigma2_fudge", sigma2_fudge);
    d.scalar("adaptive_fraction", adaptive_fraction);
    d.scalar("pixel_size", pixel_size);
    d.scalar("tau2_fudge_factor", tau2_fudge_factor);
    d.iscalar("gridding_nr_iter", gridding_nr_iter);
    d.iscalar("minres_map", mapModel.minres_map);
    d.iscalar("random_seed", random_seed);
    d.scalar("random_perturbation", sampler3d.random_perturbation);
    {
        int ntr = exp_nr_trans;
        std::vector<double> tx(ntr), ty(ntr);
        for (int t = 0; t < ntr; t++) sampler3d.getTranslation(t, tx[t], ty[t]);
        d.f64("trans_x", tx.data(), {ntr});
        d.f64("trans_y", ty.data(), {ntr});
    }
    d.i32("Npix_per_shell", Npix_per_shell.wptrAll(), {oF});
    d.i32("Mresol_fine", Mresol_fine.wptrAll(), {current_size * (current_size / 2 + 1)});
    d.i32("Mresol_coarse", Mresol_coarse.wptrAll(), {coarse_size * (coarse_size / 2 + 1)});
    std::vector<double> s2((size_t)G * oF);
    for (int g = 0; g < G; g++)
        for (int n = 0; n < oF; n++) s2[(size_t)g * oF + n] = mlModel.sigma2_noise[g][n];
    d.f64("sigma2_noise", s2.data(), {G, oF});
    d.f64("pdf_class", mlModel.pdf_class.wptrAll(), {K});
    {
        std::vector<double> pdir((size_t)K * ND);
        for (int k = 0; k < K; k++)
            for (int j = 0; j < ND; j++) pdir[(size_t)k * ND + j] = mlModel.pdf_direction[k][j];
        d.f64("pdf_direction", pdir.data(), {K, ND});
    }
    d.f64("prior_offsetx_class", mlModel.prior_offsetx_class.wptrAll(), {K});
    d.f64("prior_offsety_class", mlModel.prior_offsety_class.wptrAll(), {K});
    d.f64("scale_correction", mlModel.scale_correction.wptrAll(), {G});
    d.scalar("sigma2_offset", mlModel.sigma2_offset);
    d.scalar("avg_norm_correction", mlModel.avg_norm_correction);
    {
        int pad = mapModel.projector[0].pad_size, padF = mapModel.projector[0].pad_Fsize;
        size_t vox = (size_t)pad * pad * padF;
        size_t ov = (size_t)ori_size * ori_size * ori_size;
        std::vector<double> pdata(K * vox * 2), irefs(K * ov);
        for (int k = 0; k < K; k++) {
            auto p = (double*)mapModel.projector[k].data.wptr();
            for (size_t i = 0; i < vox * 2; i++) pdata[k * vox * 2 + i] = p[i];
            auto r = mapModel.Irefs[k].wptr();
            for (size_t i = 0; i < ov; i++) irefs[k * ov + i] = r[i];
        }
        d.f64("projector_data", pdata.data(), {K, pad, pad, padF, 2});
        d.iscalar("projector_r_max", mapModel.projector[0].r_max);
        d.iscalar("projector_pad_size", pad);
        d.iscalar("projector_padding_factor", mapModel.projector[0].padding_factor);
        if (!g_light) d.f64("Irefs_before", irefs.data(), {K, ori_size, ori_size, ori_size});
        std::vector<double> tau2((size_t)K * oF), dvp((size_t)K * oF);
        for (int k = 0; k < K; k++)
            for (int n = 0; n < oF; n++) {
                tau2[(size_t)k * oF + n] = mlModel.tau2_class[k][n];
                dvp[(size_t)k * oF + n] = mlModel.data_vs_prior_class[k][n];
            }
        d.f64("tau2_class_before", tau2.data(), {K, oF});
        d.f64("data_vs_prior_before", dvp.data(), {K, oF});
    }

    // ---- expectation() (src/map3d_optimizer.cpp:788-881) with the first pools staged ----
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
            exp_metadata[i] = metadata[i + first];
            auto dst = exp_imgs[i].wptr(ori_size * ori_size);
            auto src = images[first + i - first_local_image].rptrAll();
            for (int j = 0; j < ori_size * ori_size; j++) dst[j] = src[j];
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

            for (exp_ipass = 0; exp_ipass < 2; exp_ipass++) {
                std::string ps = pp + "pass" + std::to_string(exp_ipass) + "_";
                bool coarse = exp_ipass == 0;
                exp_current_size = coarse ? coarse_size : current_size;
                exp_current_oversampling = coarse ? 0 : adaptive_oversampling;
                samplingGrid.computeGrid3D(sampler3d, exp_current_oversampling);
                exp_nr_over_rot = samplingGrid.exp_nr_over_rot();
                exp_nr_over_trans = samplingGrid.exp_nr_over_trans();
                bool cc = (iter == 1 && do_firstiter_cc) || do_always_cc;
                particleModel.preShiftedImagesCtfsAndInvSigma2s(
                    exp_Fimgs_shifted_real, exp_Fimgs_shifted_imag, exp_local_Minvsigma2s, exp_local_sqrtXi2,
                    exp_local_Fctfs, exp_current_size, cc, coarse, samplingGrid, mlModel, Mresol_coarse, Mresol_fine);
                if (pool_index == 0) dump_pass_inputs(d, ps);
                getReferenceAllOrientations();
                {
                    std::vector<char> rs((size_t)K * ND * exp_nr_psi);
                    for (int k = 0; k < K; k++)
                        for (int r = 0; r < ND * exp_nr_psi; r++)
                            rs[(size_t)k * ND * exp_nr_psi + r] = exp_Rot_significant[k][r];
                    d.i8(ps + "Rot_significant", rs.data(), {K, ND, exp_nr_psi});
                }
                Exp_Mweight_old& mw = coarse ? exp_Mweight_coarse : exp_Mweight_fine;
                getAllSquaredDifferences(coarse);
                dump_mweight(d, ps + "diff2_", mw);
                d.f64(ps + "min_diff2", exp_min_diff2.wptrAll(), {P});
                convertSquaredDifferencesToWeights(mw);
                dump_mweight(d, ps + "weight_", mw);
                d.f64(ps + "sum_weight", exp_sum_weight.wptrAll(), {P});
                findAllSignificantPoints(mw);
                d.f64(ps + "significant_weight", exp_significant_weight.wptrAll(), {P});
                dump_metadata(d, ps);
                if (coarse) {
                    int nc = (int)exp_Mcoarse_significant[0].size();
                    std::vector<char> mc((size_t)P * nc);
                    for (int i = 0; i < P; i++)
                        for (int j = 0; j < nc; j++) mc[(size_t)i * nc + j] = exp_Mcoarse_significant[i][j];
                    d.i8(ps + "Mcoarse_significant", mc.data(), {P, nc});
                }
            }
            updateOtherParams();
            d.f64(pp + "wsum_norm_correction", exp_wsum_norm_correction.wptrAll(), {P});
            if (do_scale_correction) {
                // per-particle scale-correction spectra of updateOtherParams (before storeWeightedSums divides them)
                auto xa = flat2(exp_wsum_scale_correction_XA, P, oF);
                d.f64(pp + "wsum_scale_correction_XA", xa.data(), {P, oF});
                auto aa = flat2(exp_wsum_scale_correction_AA, P, oF);
                d.f64(pp + "wsum_scale_correction_AA", aa.data(), {P, oF});
            }
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
        hiddenVarMonitor.monitorHiddenVariableChanges(sampler3d, metadata, first, &exp_metadata[0], exp_nr_images);
        for (int i = 0; i < exp_nr_images; i++) metadata[i + first] = exp_metadata[i];
        nr_done += last - first + 1;
        pool_index++;
    }

    // ---- M-step inputs and outputs ----
    dump_model_sums(d, "iter_");
    dump_backprojectors(d, "iter_");
    if (option.getBoolOption("-skip_mstep")) {
        std::cout << "map3d_dump: done (M-step skipped)" << std::endl;
        return 0;
    }
    maximization();
    {
        size_t ov = (size_t)ori_size * ori_size * ori_size;
        std::vector<double> irefs(K * ov), tau2((size_t)K * oF), sig((size_t)K * oF), dvp((size_t)K * oF);
        for (int k = 0; k < K; k++) {
            auto r = mapModel.Irefs[k].wptr();
            for (size_t i = 0; i < ov; i++) irefs[k * ov + i] = r[i];
            for (int n = 0; n < oF; n++) {
                tau2[(size_t)k * oF + n] = mlModel.tau2_class[k][n];
                sig[(size_t)k * oF + n] = mlModel.sigma2_class[k][n];
                dvp[(size_t)k * oF + n] = mlModel.data_vs_prior_class[k][n];
            }
        }
        d.f64("Irefs_after", irefs.data(), {K, ori_size, ori_size, ori_size});
        d.f64("tau2_class_after", tau2.data(), {K, oF});
        d.f64("sigma2_class_after", sig.data(), {K, oF});
        d.f64("data_vs_prior_after", dvp.data(), {K, oF});
        d.f64("pdf_class_after", mlModel.pdf_class.wptrAll(), {K});
        // the rest of the model as maximizationOtherParameters (map3d_optimizer.cpp:2620-2798) left it
        const int nd = mlModel.nr_directions;
        d.f64("sigma2_noise_after", flat2(mlModel.sigma2_noise, G, oF).data(), {G, oF});
        d.f64("pdf_direction_after", flat2(mlModel.pdf_direction, K, nd).data(), {K, nd});
        d.scalar("sigma2_offset_after", mlModel.sigma2_offset);
        d.scalar("avg_norm_correction_after", mlModel.avg_norm_correction);
        d.f64("scale_correction_after", mlModel.scale_correction.wptrAll(), {G});
        d.scalar("LL_after", mlModel.LL);
        d.scalar("ave_Pmax_after", mlModel.ave_Pmax);
        d.i32("nr_particles_group", mlModel.nr_particles_group.wptrAll(), {G});
        d.iscalar("refs_are_ctf_corrected_after", refs_are_ctf_corrected);
    }
    std::cout << "map3d_dump: done" << std::endl;
    return 0;
}
