// Timing harness for the reference's own MAP2D E-step (CPU baseline; links
// oracle/_ref/libromeref.a, the reference sources compiled unchanged).
//
// Drives Map2dOptimizer_old like apps/rome_map2d.cpp:27-139: iteration 1
// runs through the reference's iterate() (src/map2d_optimizer.cpp:456-565),
// then iteration 2 is set up exactly as iterate() does, except that the
// current resolution is set to Nyquist first so that the E-step runs at the
// full image size (current_size = ori_size, the size the GPU benchmark
// uses) and every class has a positive prior (all K classes are searched).
// With -refs_raw (K float64 images [K][ori][ori]) iteration 1 is skipped and
// those images are the class references of iteration 2 (the templates the
// particles were made from, which is what the GPU benchmark searches): the
// work per particle then no longer depends on how well a short iteration 1
// on the timing sample seeded the classes (it seeds each class from 1/K of
// the sample, src/map2d_optimizer.cpp:731-760, so a small sample gives
// noisier references, broader posteriors and more significant hypotheses).
// The first -warm_pools + -time_pools pools of iteration 2 are then
// processed as expectation() does (src/map2d_optimizer.cpp:760-799) and
// expectationSomeParticles() (:802-854) of the last -time_pools is timed
// with the reference's own dtime(); every OpenMP thread of the host is
// used.  Prints one line per timed pool and a total:
//   map2d_bench_pool index=<i> particles=<n> estep_s=<t>
//   map2d_bench particles=<n> estep_s=<t> prep_s=<t> current_size=<s> threads=<n>
#include "map2d_optimizer.h"
#include "option.h"

#include <omp.h>

#include <cstdio>
#include <vector>

using namespace Map2dOptimizer_old;

int main(int argc, char* argv[]) {
    Option option;
    option.addOption("-i", "Input STAR file");
    option.addOption("-K", "Number of classes");
    option.addOption("-angpix", "Pixel size (A)");
    option.addOption("-tau2_fudge", "Regularisation parameter", "2");
    option.addOption("-oversampling", "Adaptive oversampling order", "0");
    option.addOption("-particle_diameter", "Particle diameter", "-1");
    option.addOption("-pool", "Pool size", "50");
    option.addOption("-random_seed", "Random seed", "33");
    option.addOption("-offset_step", "Offset step (pixels)", "2");
    option.addOption("-offset_range", "Offset range (pixels)", "10");
    option.addOption("-psi_step", "Psi step (degrees)", "10");
    option.addOption("-ctf", "CTF correction", "0");
    option.addOption("-time_pools", "Pools of iteration 2 to time", "1");
    option.addOption("-warm_pools", "Pools of iteration 2 run before timing", "0");
    option.addOption("-refs_raw", "K class references, float64 [K][ori][ori] raw (skips iteration 1)", "NULL");
    option.readCommandLine(argc, argv);

    star_fn = pathRemoveSuffix(option.getStrOption("-i")) + ".star";
    mrcs_dir = pathGetDir(star_fn);
    write_path = "NULL";
    write_fn = "NULL";
    nr_classes = option.getIntOption("-K");
    nr_pool = option.getIntOption("-pool");
    pixel_size = option.getFloatOption("-angpix");
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
    const int time_pools = option.getIntOption("-time_pools");

    const int warm_pools = option.getIntOption("-warm_pools");
    const std::string refs_raw = option.getStrOption("-refs_raw");

    setupMap2dOptimizer();
    readImages();
    Map2dOptimizer_old::prepare();
    if (refs_raw == "NULL") {
        nr_iter = 1;
        Map2dOptimizer_old::iterate();
    } else {
        const size_t n2 = (size_t)ori_size * ori_size;
        std::vector<double> buf(n2 * nr_classes);
        FILE* f = std::fopen(refs_raw.c_str(), "rb");
        if (!f || std::fread(buf.data(), sizeof(double), buf.size(), f) != buf.size()) {
            std::fprintf(stderr, "map2d_bench: cannot read %zu doubles from -refs_raw\n", buf.size());
            return 2;
        }
        std::fclose(f);
        for (int k = 0; k < nr_classes; k++) {
            auto r = mapModel.Irefs[k].wptr();
            for (size_t i = 0; i < n2; i++) r[i] = buf[k * n2 + i];
        }
    }
    nr_iter = 2;
    iter = 2;

    // Iteration 1 seeds one class per pool, so a small timing sample leaves
    // most classes with pdf_class = 0, which iteration 2 would skip.  Start
    // iteration 2 from the uniform class prior MLModel::initialize sets so
    // that every class is searched, as in a full-size run.
    for (int k = 0; k < nr_classes; k++) mlModel.pdf_class.wptrAll()[k] = 1. / nr_classes;
    // iteration 2 at full size
    mapModel.current_resolution = 1. / (2. * pixel_size);
    double ang = sampler2d.getAngularSampling();
    mapModel.updateImageSizeAndResolutionPointers(Npix_per_shell, Mresol_coarse, Mresol_fine, coarse_size, current_size,
                                                  adaptive_oversampling, ang, mlModel.ave_Pmax);
    prepareExpData();

    double t_estep = 0, t_prep = 0;
    int nr_done = 0, pool_index = 0, timed = 0;
    while (nr_done < nr_local_images && pool_index < warm_pools + time_pools) {
        int first = first_local_image + nr_done;
        int last = std::min(first_local_image + nr_local_images - 1, first + nr_pool - 1);
        exp_first_image = first;
        exp_last_image = last;
        exp_nr_images = last - first + 1;
        exp_iclass_min = 0;
        exp_iclass_max = nr_classes - 1;
        const double t0 = dtime();
        for (int i = 0; i < exp_nr_images; i++) {
            auto dst = exp_imgs[i].wptr(ori_size * ori_size);
            auto src = images[(first - first_local_image) + i].wptrAll();
            for (int j = 0; j < ori_size * ori_size; j++) dst[j] = src[j];
            exp_metadata[i] = metadata[i + first];
        }
        particleModel.prepare(exp_imgs, exp_metadata, exp_first_image, exp_nr_images);
        particleModel.setFourierTransforms(exp_power_imgs, exp_highres_Xi2_imgs, exp_old_offsetx, exp_old_offsety, mlModel,
                                           do_ctf_correction);
        const double t1 = dtime();
        expectationSomeParticles();
        const double t2 = dtime();
        if (pool_index >= warm_pools) {
            std::printf("map2d_bench_pool index=%d particles=%d estep_s=%.6f\n", pool_index, exp_nr_images, t2 - t1);
            std::fflush(stdout);
            t_prep += t1 - t0;
            t_estep += t2 - t1;
            timed += exp_nr_images;
        }
        for (int i = 0; i < exp_nr_images; i++) metadata[i + first] = exp_metadata[i];
        nr_done += last - first + 1;
        pool_index++;
    }
    std::printf("map2d_bench particles=%d estep_s=%.6f prep_s=%.6f current_size=%d threads=%d\n", timed, t_estep,
                t_prep, current_size, omp_get_max_threads());
    return 0;
}
