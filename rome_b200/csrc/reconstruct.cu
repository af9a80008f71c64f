// M-step reconstruction of one class on the GPU.
//
// Replaces MAPModel::reconstruction (src/map_model.cpp:233-241) ->
// MyBackProjector::reconstruct (src/reconstruct.cpp:1929-2526) for the
// map2d/map3d settings (trilinear, padding 2, C1, no FSC-based tau2):
//   enforceHermitianSymmetry (:1501-1537)        hermitian_kernel
//   radial sigma2 of the reconstruction (:2019-2075) + MAP Wiener term and
//   data_vs_prior (:2076-2158)                   radial_kernel, map_term_kernel
//   normalise by wsum_pdf_class (:2167-2188)     scale kernels
//   10 Pipe & Menon preweighting iterations (:2224-2286) with the
//   Kaiser-Bessel blob convolution done by cuFFT (convoluteBlobRealSpace,
//   :1721-1788)                                  gridding kernels + cuFFT Z2D/D2Z
//   Fconv = decenter(data) * Fnewweight (:2312-2332)
//   windowToOridimRealSpace (:1790-1927): window, inverse FFT, centre, crop,
//   /normfft, softMaskOutsideMap (reconstruct.h:214-275)
//   griddingCorrect (:61-103)
// All arithmetic is FP64 (the reference keeps Fnewweight in double,
// :1946-1949).  Radial sums use FP64 atomics, so they match the reference to
// summation-order rounding.
#include <cufft.h>

#include <cmath>
#include <vector>

#include "common.cuh"

using namespace rome;

namespace {

#define ROME_CUFFT(call)                                                              \
    do {                                                                              \
        cufftResult r_ = (call);                                                      \
        if (r_ != CUFFT_SUCCESS) fail(ROME_ERR_CUDA, "%s failed (%d)", #call, (int)r_); \
    } while (0)

struct Geo {
    int Z, Y, Xf;  // complex grid dims (Z = 1 in 2D)
    int pad;       // pad_size (odd)
    long vox;
    int ref_dim;
    int ori;
    int r_max;
    int padding;
    long max_r2;
};

// centred (projector) coordinates of element (k, i, j): origin at pad/2
__device__ __forceinline__ void centred(const Geo& g, long q, int& kp, int& ip, int& jp) {
    int j = (int)(q % g.Xf);
    long t = q / g.Xf;
    int i = (int)(t % g.Y);
    int k = (int)(t / g.Y);
    jp = j;
    ip = i - g.pad / 2;
    kp = g.ref_dim == 3 ? k - g.pad / 2 : 0;
}

// FFTW (decentred) coordinates of element (k, i, j) of a pad x pad x padF array
__device__ __forceinline__ void decentred(const Geo& g, long q, int& kp, int& ip, int& jp, int& k, int& i, int& j) {
    j = (int)(q % g.Xf);
    long t = q / g.Xf;
    i = (int)(t % g.Y);
    k = (int)(t / g.Y);
    jp = j;
    ip = i < g.Xf ? i : i - g.Y;
    kp = g.ref_dim == 3 ? (k < g.Xf ? k : k - g.Z) : 0;
}

// index of the centred element holding decentred frequency (kp, ip, jp)
__device__ __forceinline__ long centred_index(const Geo& g, int kp, int ip, int jp) {
    int k2 = g.ref_dim == 3 ? kp + g.pad / 2 : 0;
    int i2 = ip + g.pad / 2;
    return ((long)k2 * g.Y + i2) * g.Xf + jp;
}

__global__ void hermitian_kernel(Geo g, double2* __restrict__ data, double* __restrict__ weight) {
    // representatives: (iz < 0, iy >= 0) and (iz >= 0, iy >= 1), xmipp origin -pad/2
    const int oz = g.ref_dim == 3 ? -(g.pad / 2) : 0, oy = -(g.pad / 2);
    const int nz = g.ref_dim == 3 ? g.pad : 1, ny_half = g.Y + oy;  // iy in [0, Y + oy)
    long n = (long)nz * ny_half;
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    int iz = (int)(q / ny_half) + oz;
    int iy = (int)(q % ny_half);
    if (iz >= 0 && iy < 1) return;
    int zl = -iz - oz, zr = iz - oz, yl = -iy - oy, yr = iy - oy;
    long a = ((long)zr * g.Y + yr) * g.Xf, b = ((long)zl * g.Y + yl) * g.Xf;
    double2 dr = data[a], dl = data[b];
    double fr = dr.x + dl.x, fi = dr.y - dl.y;
    data[a] = make_double2(fr, fi);
    data[b] = make_double2(fr, -fi);
    double s = weight[a] + weight[b];
    weight[a] = s;
    weight[b] = s;
}

// Fweight = decenter(weight) (r2 <= max_r2, else 0); radial sums of the
// noise power (sigma2) on r2 < max_r2
__global__ void decenter_weight_kernel(Geo g, const double* __restrict__ weight, double* __restrict__ Fw,
                                       double osc, double* __restrict__ sig_sum, double* __restrict__ sig_cnt) {
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.vox) return;
    int kp, ip, jp, k, i, j;
    decentred(g, q, kp, ip, jp, k, i, j);
    long r2 = (long)kp * kp + (long)ip * ip + (long)jp * jp;
    double v = r2 <= g.max_r2 ? weight[centred_index(g, kp, ip, jp)] : 0.0;
    Fw[q] = v;
    if (r2 < g.max_r2) {
        int ires = (int)round(sqrt((double)r2) / g.padding);
        atomicAdd(&sig_sum[ires], osc * v);
        atomicAdd(&sig_cnt[ires], 1.0);
    }
}

// MAP term: Fweight += 1 / (osc * tau2_fudge * tau2[ires]) for ires >= minres_map,
// and the data_vs_prior radial sums
__global__ void map_term_kernel(Geo g, double* __restrict__ Fw, const double* __restrict__ tau2, double osc,
                                double tau2_fudge, int minres, double* __restrict__ dvp_sum,
                                double* __restrict__ dvp_cnt, int* __restrict__ bad) {
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.vox) return;
    int kp, ip, jp, k, i, j;
    decentred(g, q, kp, ip, jp, k, i, j);
    long r2 = (long)kp * kp + (long)ip * ip + (long)jp * jp;
    if (r2 >= g.max_r2) return;
    int ires = (int)round(sqrt((double)r2) / g.padding);
    double invw = Fw[q];
    double t = tau2[ires], invtau2;
    if (t > 0.) invtau2 = 1. / (osc * tau2_fudge * t);
    else if (t == 0.) invtau2 = 1. / (0.001 * invw);
    else {
        atomicExch(bad, 1);
        return;
    }
    atomicAdd(&dvp_sum[ires], invw / invtau2);
    atomicAdd(&dvp_cnt[ires], 1.0);
    if (ires >= minres) Fw[q] = invw + invtau2;
}

__global__ void scale_kernel(long n, double* __restrict__ a, double s) {
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) a[q] /= s;
}

// Fnewweight = 1 inside r2 < max_r2 (decenter of the indicator), and the
// backprojector weight becomes that indicator (the reference reuses it)
__global__ void init_newweight_kernel(Geo g, double* __restrict__ Fnw, double* __restrict__ weight) {
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.vox) return;
    int kp, ip, jp, k, i, j;
    decentred(g, q, kp, ip, jp, k, i, j);
    long r2 = (long)kp * kp + (long)ip * ip + (long)jp * jp;
    Fnw[q] = r2 < g.max_r2 ? 1.0 : 0.0;
    int ckp, cip, cjp;
    centred(g, q, ckp, cip, cjp);
    long cr2 = (long)ckp * ckp + (long)cip * cip + (long)cjp * cjp;
    weight[q] = cr2 < g.max_r2 ? 1.0 : 0.0;
}

__global__ void conv_prep_kernel(long n, const double* __restrict__ Fnw, const double* __restrict__ Fw,
                                 double2* __restrict__ Fconv) {
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) Fconv[q] = make_double2(Fnw[q] * Fw[q], 0.0);
}

// real-space multiplication by the blob's Fourier transform (normalised at 0)
__global__ void blob_multiply_kernel(int Z, int pad, int ref_dim, int ori, int padding, double* __restrict__ M,
                                     const double* __restrict__ tab, int ntab, double tab_sampling, double norm0) {
    long n = (long)Z * pad * pad;
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    int j = (int)(q % pad);
    long t = q / pad;
    int i = (int)(t % pad);
    int k = (int)(t / pad);
    int ph = pad / 2;
    int kp = ref_dim == 3 ? (k < ph ? k : k - pad) : 0;
    int ip = i < ph ? i : i - pad;
    int jp = j < ph ? j : j - pad;
    double rval = sqrt((double)((long)kp * kp + (long)ip * ip + (long)jp * jp)) / (ori * padding);
    int idx = (int)(fabs(rval) / tab_sampling);
    double b = idx >= ntab ? 0. : tab[idx];
    M[q] *= b / norm0;
}

// after the forward FFT (normalised by the real size): Fnewweight /= max(1e-6, |Fconv|)
__global__ void newweight_update_kernel(Geo g, const double2* __restrict__ Fconv, double inv_n,
                                        double* __restrict__ Fnw) {
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.vox) return;
    int kp, ip, jp, k, i, j;
    decentred(g, q, kp, ip, jp, k, i, j);
    long r2 = (long)kp * kp + (long)ip * ip + (long)jp * jp;
    if (r2 < g.max_r2) {
        double2 c = Fconv[q];
        double cr = c.x * inv_n, ci = c.y * inv_n;
        double w = fmax(1e-6, sqrt(cr * cr + ci * ci));
        Fnw[q] /= w;
    }
}

// Fconv = decenter(data) * Fnewweight, windowed straight into the
// padoridim transform (windowFourierTransform, reconstruct.h:471-545)
__global__ void final_fconv_kernel(Geo g, int P2, const double2* __restrict__ data, const double* __restrict__ Fnw,
                                   double2* __restrict__ Ftmp) {
    // output grid: Z2 x P2 x (P2/2+1)
    const int Z2 = g.ref_dim == 3 ? P2 : 1, X2 = P2 / 2 + 1;
    long n = (long)Z2 * P2 * X2;
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    int j = (int)(q % X2);
    long t = q / X2;
    int i = (int)(t % P2);
    int k = (int)(t / P2);
    double2 v = make_double2(0.0, 0.0);
    // frequency of the output element; copied from the input element of the
    // same frequency when the input holds it (both branches of
    // windowFourierTransform; growing also drops corners beyond (Xf-1)^2)
    int kp = g.ref_dim == 3 ? (k < X2 ? k : k - Z2) : 0;
    int ip = i < X2 ? i : i - P2;
    const int hi = g.Xf - 1, lo = -(g.Y - g.Xf);  // input frequency range [lo, hi]
    bool in_range = j <= hi && ip >= lo && ip <= hi && (g.ref_dim != 3 || (kp >= lo && kp <= hi));
    long fr2 = (long)kp * kp + (long)ip * ip + (long)j * j;
    if (X2 > g.Xf && fr2 > (long)hi * hi) in_range = false;
    if (in_range) {
        int k2 = g.ref_dim == 3 ? (kp < 0 ? kp + g.Z : kp) : 0;
        int i2 = ip < 0 ? ip + g.Y : ip;
        long src = ((long)k2 * g.Y + i2) * g.Xf + j;
        if (fr2 <= g.max_r2) {
            double2 d = data[centred_index(g, kp, ip, j)];
            double w = Fnw[src];
            v = make_double2(d.x * w, d.y * w);
        }
    }
    Ftmp[q] = v;
}

// MoutCenter -> window to ori_size -> / normfft ; writes the ori^d volume
__global__ void crop_kernel(int ref_dim, int P2, int ori, const double* __restrict__ Mout, double normfft,
                            double* __restrict__ vol) {
    const int Zo = ref_dim == 3 ? ori : 1;
    long n = (long)Zo * ori * ori;
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    int j = (int)(q % ori);
    long t = q / ori;
    int i = (int)(t % ori);
    int k = (int)(t / ori);
    // vol(k,i,j) = MoutCenter(k+off, ...) = Mout((k - ori/2) mod P2, ...)
    int a = ((i - ori / 2) % P2 + P2) % P2;
    int b = ((j - ori / 2) % P2 + P2) % P2;
    int c = ref_dim == 3 ? ((k - ori / 2) % P2 + P2) % P2 : 0;
    vol[q] = Mout[((long)c * P2 + a) * P2 + b] / normfft;
}

__device__ __forceinline__ double centred_r(int ref_dim, int ori, long q) {
    int j = (int)(q % ori);
    long t = q / ori;
    int i = (int)(t % ori);
    int k = (int)(t / ori);
    int o = -(int)((float)ori / 2.0f);
    int kp = ref_dim == 3 ? k + o : 0, ip = i + o, jp = j + o;
    return sqrt((double)((long)kp * kp + (long)ip * ip + (long)jp * jp));
}

// softMaskOutsideMap background average (radius ori/2, cosine width 3)
__global__ void softmask_sum_kernel(int ref_dim, int ori, const double* __restrict__ vol, double* __restrict__ acc) {
    const int Zo = ref_dim == 3 ? ori : 1;
    long n = (long)Zo * ori * ori;
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double s = 0.0, sb = 0.0;
    if (q < n) {
        const double radius = (double)ori / 2., width = 3., radius_p = radius + width;
        double r = centred_r(ref_dim, ori, q);
        if (r >= radius) {
            if (r > radius_p) {
                s = 1.;
                sb = vol[q];
            } else {
                double rc = 0.5 + 0.5 * cos(kPi * (radius_p - r) / width);
                s = rc;
                sb = rc * vol[q];
            }
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, off);
        sb += __shfl_down_sync(0xffffffffu, sb, off);
    }
    if ((threadIdx.x & 31) == 0 && (s != 0.0 || sb != 0.0)) {
        atomicAdd(&acc[0], s);
        atomicAdd(&acc[1], sb);
    }
}

// apply the soft mask, then griddingCorrect (divide by sinc^2 of r / (ori * padding))
__global__ void softmask_gridding_kernel(int ref_dim, int ori, int padding, double* __restrict__ vol,
                                         const double* __restrict__ acc) {
    const int Zo = ref_dim == 3 ? ori : 1;
    long n = (long)Zo * ori * ori;
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const double radius = (double)ori / 2., width = 3., radius_p = radius + width;
    const double bg = acc[1] / acc[0];
    double r = centred_r(ref_dim, ori, q);
    double v = vol[q];
    if (r >= radius) {
        if (r > radius_p) v = bg;
        else {
            double rc = 0.5 + 0.5 * cos(kPi * (radius_p - r) / width);
            v = (1 - rc) * v + rc * bg;
        }
    }
    if (r > 0.) {
        double rval = r / (ori * padding);
        double sinc = sin(kPi * rval) / (kPi * rval);
        v /= sinc * sinc;
    }
    vol[q] = v;
}

// Kaiser-Bessel blob Fourier transform, order 0 (bessel.cpp kaiser_Fourier_value
// with m = 0): proportional to i_{3/2}(s)/s^{3/2} or j_{3/2}(s)/s^{3/2},
// s = sqrt(|alpha^2 - (2 pi a w)^2|); the constant factor cancels in
// tab(w)/tab(0) and is dropped.  Half-integer Bessel functions in closed form.
double blob_ft_shape(double w, double a, double alpha) {
    double x = 2. * kPi * a * w;
    double s = sqrt(fabs(alpha * alpha - x * x));
    if (s == 0.) return 0.;
    double v;
    if (x > alpha) v = sqrt(2. / (kPi * s)) * (sin(s) / s - cos(s));
    else v = sqrt(2. / (kPi * s)) * (cosh(s) - sinh(s) / s);
    return v / pow(s, 1.5);
}

void check(cudaStream_t st) { ROME_CHECK_LAUNCH(); }

unsigned blocks(long n) { return (unsigned)((n + 255) / 256); }

}  // namespace

extern "C" int rome_gpu_reconstruct(RomeGpuCtx* ctx, const RomeReconIn* in, RomeReconOut* out) {
    if (!ctx || !in || !out) return ROME_ERR_ARG;
    return guarded(ctx, [&] {
        if (!ctx->bp_data) fail(ROME_ERR_STATE, "no backprojectors (rome_gpu_set_projectors)");
        ROME_REQUIRE(in->iclass >= 0 && in->iclass < ctx->nr_classes, "iclass out of range");
        ROME_REQUIRE(in->tau2_in && out->vol && out->sigma2 && out->data_vs_prior, "missing arrays");
        ROME_CUDA(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        Profiler prof(ctx);
        Geo g;
        g.ref_dim = ctx->ref_dim;
        g.pad = ctx->pad_size;
        g.Z = g.ref_dim == 3 ? g.pad : 1;
        g.Y = g.pad;
        g.Xf = g.pad / 2 + 1;
        g.vox = ctx->vox;
        g.ori = ctx->ori_size;
        g.r_max = ctx->r_max;
        g.padding = ctx->padding;
        g.max_r2 = (long)g.r_max * g.r_max * g.padding * g.padding;
        const int oriF = g.ori / 2 + 1;
        const double osc = g.ref_dim == 3 ? (double)(g.padding * g.padding * g.padding) : (double)(g.padding * g.padding);
        double2* data = ctx->bp_data + (long)in->iclass * g.vox;
        double* weight = ctx->bp_weight + (long)in->iclass * g.vox;
        const long nreal = (long)g.Z * g.pad * g.pad;
        const int P2 = g.padding * g.ori;
        const int Z2 = g.ref_dim == 3 ? P2 : 1;
        const long n2c = (long)Z2 * P2 * (P2 / 2 + 1), n2r = (long)Z2 * P2 * P2;
        const long nvol = (long)(g.ref_dim == 3 ? g.ori : 1) * g.ori * g.ori;

        double* Fw = ctx->ws[S_REC_FW].as<double>(g.vox);
        double* Fnw = ctx->ws[S_REC_FNW].as<double>(g.vox);
        double2* Fconv = ctx->ws[S_REC_FCONV].as<double2>(std::max(g.vox, n2c));
        double* Mreal = ctx->ws[S_REC_REAL].as<double>(std::max(nreal, n2r));
        double* small = ctx->ws[S_REC_SMALL].as<double>((size_t)6 * oriF + 16);
        double* dvol = ctx->ws[S_REC_VOL].as<double>(nvol);
        int* bad = (int*)(small + 6 * oriF + 8);
        ROME_CUDA(cudaMemsetAsync(small, 0, sizeof(double) * (6 * oriF + 16), st));
        double* sig_sum = small;
        double* sig_cnt = small + oriF;
        double* dvp_sum = small + 2 * oriF;
        double* dvp_cnt = small + 3 * oriF;
        double* dtau2 = small + 4 * oriF;
        double* sm_acc = small + 6 * oriF;
        ROME_CUDA(cudaMemcpyAsync(dtau2, in->tau2_in, sizeof(double) * oriF, cudaMemcpyHostToDevice, st));

        prof.begin(ROME_PHASE_RECONSTRUCT);
        {
            long nh = (long)(g.ref_dim == 3 ? g.pad : 1) * (g.Y - g.pad / 2);
            hermitian_kernel<<<blocks(nh), 256, 0, st>>>(g, data, weight);
            check(st);
            prof.launched(ROME_PHASE_RECONSTRUCT);
        }
        decenter_weight_kernel<<<blocks(g.vox), 256, 0, st>>>(g, weight, Fw, osc, sig_sum, sig_cnt);
        check(st);
        prof.launched(ROME_PHASE_RECONSTRUCT);
        // sigma2 = counter / sum (src/reconstruct.cpp:2049-2062)
        std::vector<double> hs(2 * oriF);
        ROME_CUDA(cudaMemcpyAsync(hs.data(), sig_sum, sizeof(double) * 2 * oriF, cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaStreamSynchronize(st));
        for (int q = 0; q < oriF; q++) {
            double s = hs[q], c = hs[oriF + q];
            if (s > 1e-10) out->sigma2[q] = c / s;
            else if (s == 0) out->sigma2[q] = 0.;
            else fail(ROME_ERR_NUMERIC, "unexpectedly small, yet non-zero sigma2 value");
        }
        for (int q = 0; q < oriF; q++) out->data_vs_prior[q] = 0.;
        if (in->do_map) {
            map_term_kernel<<<blocks(g.vox), 256, 0, st>>>(g, Fw, dtau2, osc, in->tau2_fudge, in->minres_map, dvp_sum,
                                                           dvp_cnt, bad);
            check(st);
            prof.launched(ROME_PHASE_RECONSTRUCT);
            std::vector<double> hd(2 * oriF);
            int hbad = 0;
            ROME_CUDA(cudaMemcpyAsync(hd.data(), dvp_sum, sizeof(double) * 2 * oriF, cudaMemcpyDeviceToHost, st));
            ROME_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
            ROME_CUDA(cudaStreamSynchronize(st));
            if (hbad) fail(ROME_ERR_NUMERIC, "negative tau2 spectrum");
            for (int q = 0; q < oriF; q++) {
                if (q > g.r_max) out->data_vs_prior[q] = 0.;
                else if (hd[oriF + q] < 0.001) out->data_vs_prior[q] = 999.;
                else out->data_vs_prior[q] = hd[q] / hd[oriF + q];
            }
        }
        ROME_REQUIRE(in->normalise != 0.0, "normalise (wsum_pdf_class) is zero");
        scale_kernel<<<blocks(g.vox), 256, 0, st>>>(g.vox, Fw, in->normalise);
        scale_kernel<<<blocks(2 * g.vox), 256, 0, st>>>(2 * g.vox, (double*)data, in->normalise);
        init_newweight_kernel<<<blocks(g.vox), 256, 0, st>>>(g, Fnw, weight);
        check(st);
        prof.launched(ROME_PHASE_RECONSTRUCT, 3);

        // blob table (MyBackProjector::initialize: radius 1.9 * padding, alpha 15, order 0, 10000 samples)
        const int ntab = 10000;
        const double tab_sampling = 0.5 / (double)ntab;
        std::vector<double> htab(ntab);
        for (int q = 0; q < ntab; q++) htab[q] = blob_ft_shape((double)q * tab_sampling, 1.9 * g.padding, 15.);
        double* dtab = ctx->ws[S_REC_TAB].as<double>(ntab);
        ROME_CUDA(cudaMemcpyAsync(dtab, htab.data(), sizeof(double) * ntab, cudaMemcpyHostToDevice, st));

        cufftHandle inv, fwd;
        if (g.ref_dim == 3) {
            ROME_CUFFT(cufftPlan3d(&inv, g.pad, g.pad, g.pad, CUFFT_Z2D));
            ROME_CUFFT(cufftPlan3d(&fwd, g.pad, g.pad, g.pad, CUFFT_D2Z));
        } else {
            ROME_CUFFT(cufftPlan2d(&inv, g.pad, g.pad, CUFFT_Z2D));
            ROME_CUFFT(cufftPlan2d(&fwd, g.pad, g.pad, CUFFT_D2Z));
        }
        ROME_CUFFT(cufftSetStream(inv, st));
        ROME_CUFFT(cufftSetStream(fwd, st));
        for (int it = 0; it < in->gridding_nr_iter; it++) {
            conv_prep_kernel<<<blocks(g.vox), 256, 0, st>>>(g.vox, Fnw, Fw, Fconv);
            check(st);
            ROME_CUFFT(cufftExecZ2D(inv, (cufftDoubleComplex*)Fconv, Mreal));
            blob_multiply_kernel<<<blocks(nreal), 256, 0, st>>>(g.Z, g.pad, g.ref_dim, g.ori, g.padding, Mreal, dtab,
                                                               ntab, tab_sampling, htab[0]);
            check(st);
            ROME_CUFFT(cufftExecD2Z(fwd, Mreal, (cufftDoubleComplex*)Fconv));
            newweight_update_kernel<<<blocks(g.vox), 256, 0, st>>>(g, Fconv, 1.0 / (double)nreal, Fnw);
            check(st);
            prof.launched(ROME_PHASE_RECONSTRUCT, 5);
        }
        cufftDestroy(inv);
        cufftDestroy(fwd);

        // windowToOridimRealSpace
        final_fconv_kernel<<<blocks(n2c), 256, 0, st>>>(g, P2, data, Fnw, Fconv);
        check(st);
        cufftHandle inv2;
        if (g.ref_dim == 3) ROME_CUFFT(cufftPlan3d(&inv2, P2, P2, P2, CUFFT_Z2D));
        else ROME_CUFFT(cufftPlan2d(&inv2, P2, P2, CUFFT_Z2D));
        ROME_CUFFT(cufftSetStream(inv2, st));
        ROME_CUFFT(cufftExecZ2D(inv2, (cufftDoubleComplex*)Fconv, Mreal));
        const double normfft = g.ref_dim == 3 ? (double)(g.padding * g.padding * g.padding * g.ori)
                                              : (double)(g.padding * g.padding);
        crop_kernel<<<blocks(nvol), 256, 0, st>>>(g.ref_dim, P2, g.ori, Mreal, normfft, dvol);
        softmask_sum_kernel<<<blocks(nvol), 256, 0, st>>>(g.ref_dim, g.ori, dvol, sm_acc);
        softmask_gridding_kernel<<<blocks(nvol), 256, 0, st>>>(g.ref_dim, g.ori, g.padding, dvol, sm_acc);
        check(st);
        prof.launched(ROME_PHASE_RECONSTRUCT, 5);
        prof.end(ROME_PHASE_RECONSTRUCT);
        ROME_CUDA(cudaMemcpyAsync(out->vol, dvol, sizeof(double) * nvol, cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaStreamSynchronize(st));
        cufftDestroy(inv2);
        prof.collect();
        if (out->tau2)
            for (int q = 0; q < oriF; q++) out->tau2[q] = in->tau2_in[q];
    });
}
