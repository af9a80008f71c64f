// Drop-in check of the MAP2D C ABI from C++ (test infrastructure; links the
// reference's own objects from oracle/_ref/libromeref.a and
// rome_b200/librome_b200.so).
//
// It drives Map2dOptimizer_old like apps/rome_map2d.cpp:27-139, runs the
// reference iterations 1..iter-1 unchanged, and for the first pool of
// iteration `iter` fills RomeMap2dPool from the reference's own state the
// way a patched expectationSomeParticles() (src/map2d_optimizer.cpp:802-854)
// would, calls rome_gpu_map2d_estep_pool, then runs the reference's own
// E-step functions on the same pool and compares: per-particle
// exp_min_diff2, exp_sum_weight, exp_significant_weight, PMAX and pose, the
// wsums of updateOtherParams and the back-projectors of backProjection.
// Prints one line "DROPIN key=value ..." and exits 0 when the library agrees
// within the FP32 mode's tolerances (diff2 1e-5 relative, FP64 sums and
// back-projectors 1e-3 relative, every pose but one near tie identical).
#include "map2d_optimizer.h"
#include "option.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "rome_gpu.h"

using namespace Map2dOptimizer_old;

namespace {

// VectorOfArray2d rows are separate allocations: a C caller gathers them into [n0][n1]
template <typename V>
std::vector<double> flat2(V& arr, int n0, int n1) {
    std::vector<double> out((size_t)n0 * n1);
    for (int i = 0; i < n0; i++) {
        auto p = arr[i].wptr(n1);
        for (int j = 0; j < n1; j++) out[(size_t)i * n1 + j] = p[j];
    }
    return out;
}

double max_rel(const double* a, const double* b, size_t n) {
    double m = 0.0;
    for (size_t i = 0; i < n; i++) m = std::max(m, std::fabs(a[i] - b[i]) / std::max(std::fabs(b[i]), 1e-300));
    return m;
}

// max |a - b| / max |b|
double rel_to_max(const double* a, const double* b, size_t n) {
    double d = 0.0, s = 0.0;
    for (size_t i = 0; i < n; i++) {
        d = std::max(d, std::fabs(a[i] - b[i]));
        s = std::max(s, std::fabs(b[i]));
    }
    return s > 0 ? d / s : d;
}

// the sampling tables of a pass as the reference's E-step computes them
struct PassTables {
    std::vector<double> psi, otx, oty;
};

PassTables pass_tables(int oversampling) {
    samplingGrid.computeGrid2D(sampler2d, oversampling);
    const int npsi = exp_nr_psi, nor = samplingGrid.exp_nr_over_rot();
    const int ntr = exp_nr_trans, notr = samplingGrid.exp_nr_over_trans();
    PassTables t;
    t.psi.resize((size_t)npsi * nor);
    for (int i = 0; i < npsi; i++)
        for (int j = 0; j < nor; j++) t.psi[(size_t)i * nor + j] = samplingGrid.exp_over_psi[i][j];
    t.otx.resize((size_t)ntr * notr);
    t.oty.resize(t.otx.size());
    for (int i = 0; i < ntr; i++)
        for (int j = 0; j < notr; j++) {
            t.otx[(size_t)i * notr + j] = samplingGrid.exp_over_trans_x[i][j];
            t.oty[(size_t)i * notr + j] = samplingGrid.exp_over_trans_y[i][j];
        }
    return t;
}

#define CHECK_ROME(call)                                                                         \
    do {                                                                                         \
        int rc_ = (call);                                                                        \
        if (rc_ != ROME_OK) {                                                                    \
            std::fprintf(stderr, "%s failed (%d): %s\n", #call, rc_, rome_gpu_last_error(g));    \
            return 3;                                                                            \
        }                                                                                        \
    } while (0)

}  // namespace

int main(int argc, char* argv[]) {
    Option option;
    option.addOption("-i", "Input STAR file");
    option.addOption("-K", "Number of classes");
    option.addOption("-iter", "Iteration whose first pool is compared (>= 2)");
    option.addOption("-angpix", "Pixel size (A)");
    option.addOption("-tau2_fudge", "Regularisation parameter");
    option.addOption("-oversampling", "Adaptive oversampling order (0 or 1)");
    option.addOption("-particle_diameter", "Particle diameter", "-1");
    option.addOption("-pool", "Pool size", "50");
    option.addOption("-random_seed", "Random seed", "33");
    option.addOption("-offset_step", "Offset step (pixels)", "2");
    option.addOption("-offset_range", "Offset range (pixels)", "10");
    option.addOption("-psi_step", "Psi step (degrees)", "10");
    option.addOption("-ctf", "CTF correction", "0");
    if (argc < 3) {
        option.printHelp();
        return 2;
    }
    option.readCommandLine(argc, argv);

    star_fn = pathRemoveSuffix(option.getStrOption("-i")) + ".star";
    mrcs_dir = pathGetDir(star_fn);
    write_path = "NULL";
    write_fn = "NULL";
    nr_classes = option.getIntOption("-K");
    nr_pool = option.getIntOption("-pool");
    pixel_size = option.getFloatOption("-angpix");
    const int cmp_iter = option.getIntOption("-iter");
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
    do_norm_correction = false;
    do_zero_mask = false;
    do_solvent = false;
    data_stream_in_fn = "NULL";
    data_stream_out_fn = "NULL";
    iter = 0;
    guidance_fn = "NULL";
    ref_fn = "NULL";
    if (cmp_iter < 2 || adaptive_oversampling < 0 || adaptive_oversampling > 1) {
        std::fprintf(stderr, "-iter must be >= 2 and -oversampling 0 or 1\n");
        return 2;
    }

    setupMap2dOptimizer();
    readImages();
    Map2dOptimizer_old::prepare();
    nr_iter = cmp_iter - 1;
    Map2dOptimizer_old::iterate();
    nr_iter = cmp_iter;
    iter = cmp_iter;

    // ---- iteration cmp_iter, first pool (the body of iterate() and expectation()) ----
    double ang = sampler2d.getAngularSampling();
    mapModel.updateImageSizeAndResolutionPointers(Npix_per_shell, Mresol_coarse, Mresol_fine, coarse_size, current_size,
                                                  adaptive_oversampling, ang, mlModel.ave_Pmax);
    prepareExpData();
    const int K = nr_classes, G = mlModel.nr_groups, oF = mlModel.ori_Fsize;
    const int first = first_local_image, last = std::min(first_local_image + nr_local_images - 1, first + nr_pool - 1);
    exp_first_image = first;
    exp_last_image = last;
    exp_nr_images = last - first + 1;
    exp_iclass_min = 0;
    exp_iclass_max = nr_classes - 1;
    const int P = exp_nr_images, Ff = current_size * (current_size / 2 + 1);
    for (int i = 0; i < P; i++) {
        auto dst = exp_imgs[i].wptr(ori_size * ori_size);
        auto src = images[(first - first_local_image) + i].wptrAll();
        for (int j = 0; j < ori_size * ori_size; j++) dst[j] = src[j];
        exp_metadata[i] = metadata[i + first];
    }
    particleModel.prepare(exp_imgs, exp_metadata, exp_first_image, exp_nr_images);
    particleModel.setFourierTransforms(exp_power_imgs, exp_highres_Xi2_imgs, exp_old_offsetx, exp_old_offsety, mlModel,
                                       do_ctf_correction);

    // ---- the library: the patched expectationSomeParticles() ----
    RomeGpuCtx* g = nullptr;
    RomeGpuConfig cfg = {};
    cfg.precision = ROME_PREC_FP32;
    if (rome_gpu_create(0, &cfg, &g) != ROME_OK) {
        std::fprintf(stderr, "rome_gpu_create failed\n");
        return 3;
    }
    {
        const int pad = mapModel.projector[0].pad_size, padF = mapModel.projector[0].pad_Fsize;
        const size_t vox = (size_t)pad * padF;
        std::vector<double> proj((size_t)K * vox * 2);
        for (int k = 0; k < K; k++) {
            auto p = (const double*)mapModel.projector[k].data.wptr();
            std::copy(p, p + vox * 2, proj.begin() + (size_t)k * vox * 2);
        }
        CHECK_ROME(rome_gpu_set_projectors(g, 2, K, ori_size, pad, mapModel.projector[0].r_max,
                                           mapModel.projector[0].padding_factor, proj.data()));
    }
    const PassTables t0 = pass_tables(0);
    const PassTables t1 = adaptive_oversampling > 0 ? pass_tables(adaptive_oversampling) : t0;
    std::vector<double> trx(exp_nr_trans), try_(exp_nr_trans);
    for (int t = 0; t < exp_nr_trans; t++) sampler2d.getTranslation(t, trx[t], try_[t]);
    std::vector<double> fr = flat2(particleModel.Fimages_mask_fine_real, P, Ff);
    std::vector<double> fi = flat2(particleModel.Fimages_mask_fine_imag, P, Ff);
    std::vector<double> fnr = flat2(particleModel.Fimages_nomask_real, P, Ff);
    std::vector<double> fni = flat2(particleModel.Fimages_nomask_imag, P, Ff);
    std::vector<double> fctf = flat2(particleModel.Fctfs, P, Ff);
    std::vector<int> grp(P);
    for (int i = 0; i < P; i++) grp[i] = exp_metadata[i].GROUP_NO - 1;
    std::vector<double> s2((size_t)G * oF), pdir(K);
    for (int q = 0; q < G; q++)
        for (int n = 0; n < oF; n++) s2[(size_t)q * oF + n] = mlModel.sigma2_noise[q][n];
    for (int k = 0; k < K; k++) pdir[k] = mlModel.pdf_direction[k][0];

    RomeMap2dPool in = {};
    in.nr_images = P;
    in.ori_size = ori_size;
    in.current_size = current_size;
    in.coarse_size = coarse_size;
    in.nr_classes = K;
    in.iclass_min = exp_iclass_min;
    in.iclass_max = exp_iclass_max;
    in.nr_groups = G;
    in.adaptive_oversampling = adaptive_oversampling;
    in.nr_psi = exp_nr_psi;
    in.nr_trans = exp_nr_trans;
    in.over_psi[0] = t0.psi.data();
    in.over_psi[1] = t1.psi.data();
    in.over_trans_x[0] = t0.otx.data();
    in.over_trans_x[1] = t1.otx.data();
    in.over_trans_y[0] = t0.oty.data();
    in.over_trans_y[1] = t1.oty.data();
    in.trans_x = trx.data();
    in.trans_y = try_.data();
    in.Fimg_real = fr.data();
    in.Fimg_imag = fi.data();
    in.Fimg_nomask_real = fnr.data();
    in.Fimg_nomask_imag = fni.data();
    in.Fctf = fctf.data();
    in.highres_Xi2 = exp_highres_Xi2_imgs.wptrAll();
    in.old_offsetx = exp_old_offsetx.wptrAll();
    in.old_offsety = exp_old_offsety.wptrAll();
    in.group = grp.data();
    in.sigma2_noise = s2.data();
    in.Mresol_fine = Mresol_fine.wptrAll();
    in.Mresol_coarse = Mresol_coarse.wptrAll();
    in.pdf_class = mlModel.pdf_class.wptrAll();
    in.pdf_direction = pdir.data();
    in.prior_offsetx_class = mlModel.prior_offsetx_class.wptrAll();
    in.prior_offsety_class = mlModel.prior_offsety_class.wptrAll();
    in.sigma2_offset = mlModel.sigma2_offset;
    in.sigma2_fudge = sigma2_fudge;
    in.adaptive_fraction = adaptive_fraction;
    in.do_ctf_correction = do_ctf_correction;
    in.refs_are_ctf_corrected = refs_are_ctf_corrected;
    in.do_map = do_map;

    std::vector<double> o_min(P), o_sum(P), o_sig(P), o_wnc(P), o_pmax(P), o_psi(P), o_xo(P), o_yo(P), o_nsign(P);
    std::vector<int> o_cls(P);
    std::vector<double> o_wsn((size_t)G * oF), o_wpc(K), o_wpd(K), o_wpx(K), o_wpy(K), o_wso(1), o_wsg(G);
    RomeMap2dPoolOut out = {};
    out.min_diff2 = o_min.data();
    out.sum_weight = o_sum.data();
    out.significant_weight = o_sig.data();
    out.wsum_norm_correction = o_wnc.data();
    out.pmax = o_pmax.data();
    out.cls = o_cls.data();
    out.psi = o_psi.data();
    out.xoff = o_xo.data();
    out.yoff = o_yo.data();
    out.nr_sign = o_nsign.data();
    out.wsum_sigma2_noise = o_wsn.data();
    out.wsum_pdf_class = o_wpc.data();
    out.wsum_pdf_direction = o_wpd.data();
    out.wsum_prior_offsetx_class = o_wpx.data();
    out.wsum_prior_offsety_class = o_wpy.data();
    out.wsum_sigma2_offset = o_wso.data();
    out.wsum_sumw_group = o_wsg.data();
    CHECK_ROME(rome_gpu_map2d_estep_pool(g, &in, &out));

    // ---- the reference's own E-step on the same pool ----
    const int npass = adaptive_oversampling > 0 ? 2 : 1;
    for (exp_ipass = 0; exp_ipass < npass; exp_ipass++) {
        exp_current_size = (exp_ipass == 0 && adaptive_oversampling > 0) ? coarse_size : current_size;
        exp_current_oversampling = (exp_ipass == 0) ? 0 : adaptive_oversampling;
        samplingGrid.computeGrid2D(sampler2d, exp_current_oversampling);
        exp_nr_over_rot = samplingGrid.exp_nr_over_rot();
        exp_nr_over_trans = samplingGrid.exp_nr_over_trans();
        particleModel.preShiftedImagesCtfsAndInvSigma2s(exp_Fimgs_shifted_real, exp_Fimgs_shifted_imag,
                                                        exp_local_Minvsigma2s, exp_local_sqrtXi2, exp_local_Fctfs,
                                                        exp_current_size, false, exp_ipass == 0, samplingGrid, mlModel,
                                                        Mresol_coarse, Mresol_fine);
        getReferenceAllOrientations();
        getAllSquaredDifferences();
        convertSquaredDifferencesToWeights();
        findAllSignificantPoints();
    }
    exp_current_size = current_size;
    updateOtherParams();
    backProjection();

    // ---- comparison ----
    std::vector<double> r_pmax(P);
    int same_pose = 0, same_nsign = 0;
    for (int i = 0; i < P; i++) {
        r_pmax[i] = exp_metadata[i].PMAX;
        same_pose += o_cls[i] == exp_metadata[i].CLASS && o_psi[i] == exp_metadata[i].PSI &&
                     o_xo[i] == exp_metadata[i].XOFF && o_yo[i] == exp_metadata[i].YOFF;
        same_nsign += o_nsign[i] == exp_metadata[i].NR_SIGN;
    }
    std::vector<double> r_wsn((size_t)G * oF), r_wpd(K);
    for (int q = 0; q < G; q++)
        for (int n = 0; n < oF; n++) r_wsn[(size_t)q * oF + n] = mlModel.wsum_sigma2_noise[q][n];
    for (int k = 0; k < K; k++) r_wpd[k] = mlModel.wsum_pdf_direction[k][0];
    const int pad = mapModel.backprojector[0].pad_size, padF = mapModel.backprojector[0].pad_Fsize;
    const size_t vox = (size_t)pad * padF;
    std::vector<double> gdata(vox * 2), gweight(vox);
    double bp_d = 0.0, bp_w = 0.0;
    for (int k = 0; k < K; k++) {
        CHECK_ROME(rome_gpu_get_backprojector(g, k, gdata.data(), gweight.data()));
        bp_d = std::max(bp_d, rel_to_max(gdata.data(), (const double*)mapModel.backprojector[k].data.wptr(), vox * 2));
        bp_w = std::max(bp_w, rel_to_max(gweight.data(), mapModel.backprojector[k].weight.wptr(), vox));
    }
    const double e_min = max_rel(o_min.data(), exp_min_diff2.wptrAll(), P);
    const double e_sum = max_rel(o_sum.data(), exp_sum_weight.wptrAll(), P);
    const double e_sig = max_rel(o_sig.data(), exp_significant_weight.wptrAll(), P);
    const double e_pmax = max_rel(o_pmax.data(), r_pmax.data(), P);
    const double e_wsn = rel_to_max(o_wsn.data(), r_wsn.data(), r_wsn.size());
    const double e_wpc = rel_to_max(o_wpc.data(), mlModel.wsum_pdf_class.wptrAll(), K);
    const double e_wpd = rel_to_max(o_wpd.data(), r_wpd.data(), K);
    const double e_wpx = rel_to_max(o_wpx.data(), mlModel.wsum_prior_offsetx_class.wptrAll(), K);
    std::printf("DROPIN particles=%d same_pose=%d same_nr_sign=%d min_diff2=%.3e sum_weight=%.3e "
                "significant_weight=%.3e pmax=%.3e wsum_sigma2_noise=%.3e wsum_pdf_class=%.3e "
                "wsum_pdf_direction=%.3e wsum_prior_offsetx=%.3e bp_data=%.3e bp_weight=%.3e passes=%d\n",
                P, same_pose, same_nsign, e_min, e_sum, e_sig, e_pmax, e_wsn, e_wpc, e_wpd, e_wpx, bp_d, bp_w, npass);
    rome_gpu_destroy(g);
    const bool ok = e_min <= 1e-5 && e_sum <= 1e-3 && e_sig <= 1e-3 && e_pmax <= 1e-3 && e_wsn <= 1e-3 &&
                    e_wpc <= 1e-3 && e_wpd <= 1e-3 && e_wpx <= 1e-3 && bp_d <= 1e-3 && bp_w <= 1e-3 &&
                    same_pose >= P - 1;
    return ok ? 0 : 1;
}
