// Timing harness for the reference's own MAP3D E-step (CPU baseline; links
// oracle/_ref/libromeref.a, the reference sources compiled unchanged).
//
// Sets Map3dOptimizer_old up like apps/rome_map3d.cpp:27-139 and prepare()
// (src/map3d_optimizer.cpp:330-517), then replaces the class references by
// the K volumes given in -refs_raw (the volumes the particles were projected
// from, as the GPU benchmark searches them) and runs iteration 2 of the EM
// loop as iterate() (:519-612) and expectation() (:788-881) do, with every
// class searched (iteration 1 would restrict each pool to one seed class,
// :800-838) at the full image size (current_size = ori_size), from the
// uniform class and direction priors MLModel::initialize sets.  The first
// -warm_pools pools are run and not counted; expectationSomeParticles()
// (:883-953) of the next -time_pools pools is timed with the reference's
// own dtime() on every OpenMP thread of the host.  Prints one line per pool
// and a total:
//   map3d_bench_pool index=<i> particles=<n> estep_s=<t>
//   map3d_bench particles=<n> estep_s=<t> current_size=<s> coarse_size=<s> threads=<n>
#include "map3d_optimizer.h"
#include "option.h"

#include <omp.h>

#include <cstdio>
#include <vector>

namespace Map3dOptimizer_old {
extern Images images;
}

using namespace Map3dOptimizer_old;

int main(int argc, char* argv[]) {
    Option option;
    option.addOption("-i", "Input STAR file");
    option.addOption("-ref", "Starting reference volume (MRC)");
    option.addOption("-refs_raw", "K class volumes, float64 [K][ori][ori][ori] raw, replacing the references");
    option.addOption("-K", "Number of classes");
    option.addOption("-angpix", "Pixel size (A)");
    option.addOption("-ini_high", "Initial low-pass resolution (A)", "30");
    option.addOption("-tau2_fudge", "Regularisation parameter", "2");
    option.addOption("-oversampling", "Adaptive oversampling order (>= 1)", "1");
    option.addOption("-healpix_order", "HEALPix order", "2");
    option.addOption("-particle_diameter", "Particle diameter", "-1");
    option.addOption("-pool", "Pool size", "50");
    option.addOption("-random_seed", "Random seed", "33");
    option.addOption("-offset_step", "Offset step (pixels)", "2");
    option.addOption("-offset_range", "Offset range (pixels)", "4");
    option.addOption("-ctf", "CTF correction", "1");
    option.addOption("-warm_pools", "Pools run before timing", "1");
    option.addOption("-time_pools", "Pools timed", "4");
    option.readCommandLine(argc, argv);

    star_fn = pathRemoveSuffix(option.getStrOption("-i")) + ".star";
    write_path = "NULL";
    write_fn = "NULL";
    ref_fn = option.getStrOption("-ref");
    nr_classes = option.getIntOption("-K");
    nr_pool = option.getIntOption("-pool");
    pixel_size = option.getFloatOption("-angpix");
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
    do_firstiter_cc = false;
    do_always_cc = false;
    do_scale_correction = false;
    do_norm_correction = false;
    do_zero_mask = false;
    do_solvent = false;
    do_map = true;
    mask_fn = "NULL";
    data_stream_in_fn = "NULL";
    data_stream_out_fn = "NULL";
    continue_fn = "NULL";
    guidance_fn = "NULL";
    iter = 0;
    const int warm_pools = option.getIntOption("-warm_pools");
    const int time_pools = option.getIntOption("-time_pools");

    Map3dOptimizer_old::setupMLoptimizer();
    Map3dOptimizer_old::prepare();

    // the K class volumes replace the starting reference
    {
        const size_t ov = (size_t)ori_size * ori_size * ori_size;
        std::vector<double> buf(ov * nr_classes);
        FILE* f = std::fopen(option.getStrOption("-refs_raw").c_str(), "rb");
        if (!f || std::fread(buf.data(), sizeof(double), buf.size(), f) != buf.size()) {
            std::fprintf(stderr, "map3d_bench: cannot read %zu doubles from -refs_raw\n", buf.size());
            return 2;
        }
        std::fclose(f);
        for (int k = 0; k < nr_classes; k++) {
            auto r = mapModel.Irefs[k].wptr();
            for (size_t i = 0; i < ov; i++) r[i] = buf[k * ov + i];
        }
    }
    for (int k = 0; k < nr_classes; k++) {
        mlModel.pdf_class.wptrAll()[k] = 1. / nr_classes;
        for (int j = 0; j < sampler3d.NrDir(); j++)
            mlModel.pdf_direction[k][j] = 1. / ((double)nr_classes * sampler3d.NrDir());
    }

    // iteration 2 at the full size (iterate() body up to expectation())
    nr_iter = 2;
    iter = 2;
    mapModel.current_resolution = 1. / (2. * pixel_size);
    double ang = sampler3d.getAngularSampling();
    mapModel.updateImageSizeAndResolutionPointers(Npix_per_shell, Mresol_coarse, Mresol_fine, coarse_size, current_size,
                                                  adaptive_oversampling, ang, mlModel.ave_Pmax);
    prepareExpData();

    double t_estep = 0;
    int nr_done = 0, pool_index = 0, timed = 0;
    while (nr_done < nr_local_images && pool_index < warm_pools + time_pools) {
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
        const double t1 = dtime();
        expectationSomeParticles();
        const double t2 = dtime();
        if (pool_index >= warm_pools) {
            std::printf("map3d_bench_pool index=%d particles=%d estep_s=%.6f\n", pool_index, exp_nr_images, t2 - t1);
            std::fflush(stdout);
            t_estep += t2 - t1;
            timed += exp_nr_images;
        }
        for (int i = 0; i < exp_nr_images; i++) metadata[i + first] = exp_metadata[i];
        nr_done += last - first + 1;
        pool_index++;
    }
    std::printf("map3d_bench particles=%d estep_s=%.6f current_size=%d coarse_size=%d threads=%d\n", timed, t_estep,
                current_size, coarse_size, omp_get_max_threads());
    return 0;
}
