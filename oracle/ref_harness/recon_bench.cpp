// Reference timing harness for reconstruction at known poses (test
// infrastructure; links the reference's own objects from
// oracle/_ref/libromeref.a).
//
// Times the per-image work of the image loop of apps/rome_reconstruct.cpp
// (:160-330) on spectra that are already Fourier transformed:
// shiftImageInFourierTransform (src/image.h:1478-1575), the CTF image
// (CTF::setValues / getFftwImage, src/ctf.cpp), the CTF products and
// MyBackProjector::backproject (src/reconstruct.cpp:977-1164) into the
// padded grid -- the work rome_gpu_backproject_images does on the device.
// The reference scales this loop over MPI ranks, each rank back-projecting
// its own images into its own MyBackProjector before the all-reduce
// (:333-351); here each OpenMP thread stands for one rank, with its own
// back-projector and images.  The spectra, poses and CTF parameters are
// seeded random values, a few hundred distinct spectra used in turn (the
// work does not depend on them).  Prints one line "RECON_BENCH images=N
// threads=T seconds=S per_image_median=... checksum=...".
#include "reconstruct.h"
#include "ctf.h"
#include "image.h"
#include "math.h"
#include "option.h"
#include "time.h"

#include <omp.h>

#include <algorithm>
#include <cstdio>
#include <random>
#include <vector>

int main(int argc, char* argv[]) {
    Option option;
    option.addOption("-n", "Number of images", "2000");
    option.addOption("-size", "Image size", "128");
    option.addOption("-angpix", "Pixel size (A)", "1.5");
    option.addOption("-seed", "Seed of the random spectra and poses", "5");
    option.addOption("-distinct", "Distinct spectra, used in turn (the work does not depend on their values)", "256");
    option.readCommandLine(argc, argv);
    const int n = option.getIntOption("-n"), ori = option.getIntOption("-size");
    const int nd_spec = std::max(1, std::min(n, option.getIntOption("-distinct")));
    const double angpix = option.getFloatOption("-angpix");
    const int seed = option.getIntOption("-seed");
    const int F2 = ori * (ori / 2 + 1), r_max = ori / 2;
    const int T = omp_get_max_threads();

    // inputs of every image: spectrum (real, imag), pose, shift, CTF parameters
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    std::uniform_real_distribution<double> ud(0.0, 1.0);
    std::vector<double> spec_r((size_t)nd_spec * F2), spec_i((size_t)nd_spec * F2), par((size_t)n * 8);
    for (size_t q = 0; q < spec_r.size(); q++) {
        spec_r[q] = nd(rng);
        spec_i[q] = nd(rng);
    }
    for (int i = 0; i < n; i++) {
        double* p = &par[(size_t)i * 8];
        p[0] = 360 * ud(rng);
        p[1] = std::acos(2 * ud(rng) - 1) * 180. / 3.14159265358979323846;
        p[2] = 360 * ud(rng);
        p[3] = 8 * ud(rng) - 4;
        p[4] = 8 * ud(rng) - 4;
        p[5] = 1e4 + 2e4 * ud(rng);
        p[6] = 1e4 + 2e4 * ud(rng);
        p[7] = 180 * ud(rng);
    }

    // one back-projector per rank (thread), as the app initialises it (:127-128)
    std::vector<MyBackProjector> bp(T);
    for (int t = 0; t < T; t++) bp[t].initialize(ori, 2 * r_max, 3, "C1", 2, TRILINEAR, 1, 0, 1.9, 15);
    {
        // the shift of one image on the master first (any lazily built table is built once)
        std::vector<double> a(F2), b(F2);
        double *pa = a.data(), *pb = b.data();
        const double *xr = &spec_r[0], *xi = &spec_i[0];
        shiftImageInFourierTransform(xr, xi, pa, pb, ori, 0.5, 0.5, ori);
    }
    std::vector<double> per_image(n);
    const double t0 = dtime();
#pragma omp parallel
    {
        const int t = omp_get_thread_num();
        std::vector<double> sr(F2), si(F2), fctf(F2);
        double *psr = sr.data(), *psi = si.data();
        CTF ctf;
        FDOUBLE A3D[3][3];
#pragma omp for schedule(static)
        for (int i = 0; i < n; i++) {
            const double ti = dtime();
            const double* p = &par[(size_t)i * 8];
            const double* xr = &spec_r[(size_t)(i % nd_spec) * F2];
            const double* xi = &spec_i[(size_t)(i % nd_spec) * F2];
            Euler_angles2matrix(p[0], p[1], p[2], A3D);
            shiftImageInFourierTransform(xr, xi, psr, psi, ori, p[3], p[4], ori);
            ctf.setValues(p[5], p[6], p[7], 300., 2.7, 0.1, 0.);
            ctf.getFftwImage(fctf.data(), ori, ori, ori, angpix, false, false, false, true);
            for (int q = 0; q < F2; q++) {
                sr[q] *= fctf[q];
                si[q] *= fctf[q];
                fctf[q] *= fctf[q];
            }
            bp[t].backproject(sr.data(), si.data(), ori, A3D, IS_NOT_INV, bp[t].data, bp[t].weight, fctf.data());
            per_image[i] = dtime() - ti;
        }
    }
    const double secs = dtime() - t0;
    std::vector<double> s = per_image;
    std::sort(s.begin(), s.end());
    // sum of every rank's weight volume: nonzero once every image was back-projected
    double chk = 0.0;
    const size_t vox = (size_t)bp[0].pad_size * bp[0].pad_size * bp[0].pad_Fsize;
    for (int t = 0; t < T; t++) {
        const FDOUBLE* w = bp[t].weight.wptr();
        for (size_t v = 0; v < vox; v++) chk += w[v];
    }
    std::printf("RECON_BENCH images=%d threads=%d seconds=%.6f per_image_min=%.6f per_image_median=%.6f "
                "per_image_max=%.6f checksum=%.6e\n",
                n, T, secs, s.front(), s[s.size() / 2], s.back(), chk);
    return 0;
}
