// FFTW3-API subset backed by a project-written mixed-radix FFT.
//
// Test infrastructure only: it lets the ROME reference sources
// (src/fft_base.cpp, src/fft_fftw3.cpp, src/exp_model.h, src/reconstruct.cpp)
// link without FFTW/MKL so the reference can serve as the parity oracle.
// Semantics follow the public FFTW3 documentation:
//   r2c: out[k] = sum_j in[j] e^{-2 pi i <j,k>/n}, unnormalised, last axis halved
//   c2r: out[j] = sum_k in[k] e^{+2 pi i <j,k>/n}, unnormalised, Hermitian input
// Algorithm: recursive decimation-in-time Cooley-Tukey over the prime
// factorisation of each axis length, with a direct DFT for prime lengths
// (handles the odd padded sizes such as 131 and 259 = 7 * 37).
// Accuracy is checked against numpy.fft in tests/test_oracle_fft.py.
#include "fftw/fftw3.h"

#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

typedef std::complex<double> cplx;

struct Twiddles {
    int n = 0;
    std::vector<cplx> fwd;  // e^{-2 pi i j / n}
};

Twiddles make_twiddles(int n) {
    Twiddles t;
    t.n = n;
    t.fwd.resize(n);
    const long double two_pi = 6.283185307179586476925286766559L;
    for (int j = 0; j < n; j++) {
        long double a = two_pi * (long double)j / (long double)n;
        t.fwd[j] = cplx((double)std::cos(a), (double)-std::sin(a));
    }
    return t;
}

int smallest_factor(int n) {
    if (n % 2 == 0) return 2;
    for (int p = 3; (long)p * p <= n; p += 2)
        if (n % p == 0) return p;
    return n;
}

// Transform n points read from in[0], in[stride], ... into out[0..n).
// tw: twiddles of the top-level length N; tw_step = N / n.
void fft_rec(int n, const cplx* in, long stride, cplx* out, const Twiddles& tw, int tw_step, int sign,
             cplx* scratch) {
    if (n == 1) {
        out[0] = in[0];
        return;
    }
    const int N = tw.n;
    auto W = [&](long e) -> cplx {  // e^{sign * 2 pi i e / n}
        long idx = ((e % n) * tw_step) % N;
        cplx w = tw.fwd[idx];
        return sign < 0 ? w : std::conj(w);
    };
    int p = smallest_factor(n);
    if (p == n) {
        for (int k = 0; k < n; k++) {
            cplx acc(0.0, 0.0);
            for (int j = 0; j < n; j++) acc += in[j * stride] * W((long)j * k);
            out[k] = acc;
        }
        return;
    }
    int m = n / p;
    // sub-transforms of the p decimated sequences, stored contiguously
    for (int r = 0; r < p; r++) fft_rec(m, in + r * stride, stride * p, out + r * m, tw, tw_step * p, sign, scratch + n);
    // butterflies: X[k + q m] = sum_r out[r m + k] W^{r (k + q m)}
    for (int k = 0; k < m; k++) {
        for (int q = 0; q < p; q++) {
            cplx acc(0.0, 0.0);
            long kk = k + (long)q * m;
            for (int r = 0; r < p; r++) acc += out[r * m + k] * W((long)r * kk);
            scratch[kk] = acc;
        }
    }
    std::memcpy(out, scratch, sizeof(cplx) * n);
}

// In-place complex transform along one axis of a row-major array.
void fft_axis(cplx* data, const std::vector<int>& dims, int axis, int sign) {
    int n = dims[axis];
    if (n <= 1) return;
    long inner = 1, outer = 1;
    for (size_t d = axis + 1; d < dims.size(); d++) inner *= dims[d];
    for (int d = 0; d < axis; d++) outer *= dims[d];
    Twiddles tw = make_twiddles(n);
    std::vector<cplx> line(n), res(n), scratch(4 * n + 64);
    for (long o = 0; o < outer; o++) {
        for (long i = 0; i < inner; i++) {
            cplx* base = data + o * n * inner + i;
            for (int j = 0; j < n; j++) line[j] = base[(long)j * inner];
            fft_rec(n, line.data(), 1, res.data(), tw, 1, sign, scratch.data());
            for (int j = 0; j < n; j++) base[(long)j * inner] = res[j];
        }
    }
}

}  // namespace

struct rome_fft_plan_s {
    std::vector<int> dims;  // logical (real-space) dims
    bool r2c;
    bool single;
    void* in;
    void* out;
};

namespace {

template <typename R>
void exec_r2c(const std::vector<int>& dims, const R* in, R (*out)[2]) {
    long total = 1;
    for (int d : dims) total *= d;
    std::vector<cplx> buf(total);
    for (long i = 0; i < total; i++) buf[i] = cplx((double)in[i], 0.0);
    for (size_t a = 0; a < dims.size(); a++) fft_axis(buf.data(), dims, (int)a, -1);
    int nl = dims.back(), hl = nl / 2 + 1;
    long rows = total / nl;
    for (long r = 0; r < rows; r++)
        for (int k = 0; k < hl; k++) {
            out[r * hl + k][0] = (R)buf[r * nl + k].real();
            out[r * hl + k][1] = (R)buf[r * nl + k].imag();
        }
}

template <typename R>
void exec_c2r(const std::vector<int>& dims, R (*in)[2], R* out) {
    long total = 1;
    for (int d : dims) total *= d;
    int nl = dims.back(), hl = nl / 2 + 1;
    long rows = total / nl;
    std::vector<cplx> buf(total);
    // rebuild the full spectrum from the stored half using Hermitian symmetry
    std::vector<int> lead(dims.begin(), dims.end() - 1);
    for (long r = 0; r < rows; r++) {
        // mirrored row index: negate every leading coordinate
        long rem = r, mr = 0, mul = 1;
        std::vector<int> coord(lead.size());
        for (int d = (int)lead.size() - 1; d >= 0; d--) {
            coord[d] = (int)(rem % lead[d]);
            rem /= lead[d];
        }
        for (int d = (int)lead.size() - 1; d >= 0; d--) {
            int c = coord[d] == 0 ? 0 : lead[d] - coord[d];
            mr += c * mul;
            mul *= lead[d];
        }
        for (int k = 0; k < nl; k++) {
            if (k < hl)
                buf[r * nl + k] = cplx((double)in[r * hl + k][0], (double)in[r * hl + k][1]);
            else {
                int kk = nl - k;
                buf[r * nl + k] = std::conj(cplx((double)in[mr * hl + kk][0], (double)in[mr * hl + kk][1]));
            }
        }
    }
    for (size_t a = 0; a < dims.size(); a++) fft_axis(buf.data(), dims, (int)a, +1);
    for (long i = 0; i < total; i++) out[i] = (R)buf[i].real();
}

rome_fft_plan_s* make_plan(std::vector<int> dims, bool r2c, bool single, void* in, void* out) {
    rome_fft_plan_s* p = new rome_fft_plan_s;
    p->dims = dims;
    p->r2c = r2c;
    p->single = single;
    p->in = in;
    p->out = out;
    return p;
}

}  // namespace

extern "C" {

fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double* in, fftw_complex* out, unsigned) {
    return make_plan({n0, n1}, true, false, in, out);
}
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex* in, double* out, unsigned) {
    return make_plan({n0, n1}, false, false, in, out);
}
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in, fftw_complex* out, unsigned) {
    return make_plan({n0, n1, n2}, true, false, in, out);
}
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in, double* out, unsigned) {
    return make_plan({n0, n1, n2}, false, false, in, out);
}
fftwf_plan fftwf_plan_dft_r2c_2d(int n0, int n1, float* in, fftwf_complex* out, unsigned) {
    return make_plan({n0, n1}, true, true, in, out);
}
fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex* in, float* out, unsigned) {
    return make_plan({n0, n1}, false, true, in, out);
}
fftwf_plan fftwf_plan_dft_r2c_3d(int n0, int n1, int n2, float* in, fftwf_complex* out, unsigned) {
    return make_plan({n0, n1, n2}, true, true, in, out);
}
fftwf_plan fftwf_plan_dft_c2r_3d(int n0, int n1, int n2, fftwf_complex* in, float* out, unsigned) {
    return make_plan({n0, n1, n2}, false, true, in, out);
}

void fftw_execute(const fftw_plan p) {
    if (!p) return;
    if (p->single) {
        if (p->r2c) exec_r2c<float>(p->dims, (float*)p->in, (float(*)[2])p->out);
        else exec_c2r<float>(p->dims, (float(*)[2])p->in, (float*)p->out);
    } else {
        if (p->r2c) exec_r2c<double>(p->dims, (double*)p->in, (double(*)[2])p->out);
        else exec_c2r<double>(p->dims, (double(*)[2])p->in, (double*)p->out);
    }
}
void fftwf_execute(const fftwf_plan p) { fftw_execute(p); }
void fftw_destroy_plan(fftw_plan p) { delete p; }
void fftwf_destroy_plan(fftwf_plan p) { delete p; }
void fftw_cleanup(void) {}
void fftwf_cleanup(void) {}
int fftw_init_threads(void) { return 1; }
int fftwf_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int) {}
void fftwf_plan_with_nthreads(int) {}
void fftw_cleanup_threads(void) {}
void fftwf_cleanup_threads(void) {}
void* fftw_malloc(size_t n) {
    void* p = nullptr;
    if (posix_memalign(&p, 64, n ? n : 64) != 0) return nullptr;
    return p;
}
void fftw_free(void* p) { free(p); }
void* fftwf_malloc(size_t n) { return fftw_malloc(n); }
void fftwf_free(void* p) { free(p); }

}  // extern "C"
