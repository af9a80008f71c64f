/*
 * FFTW3-compatible subset used by the ROME reference (src/fft_base.cpp,
 * src/fft_fftw3.cpp): real<->complex 2D/3D plans, execute, destroy,
 * thread setup no-ops and malloc/free.  Backed by a project-written
 * mixed-radix FFT (fftw_shim.cpp).  Not FFTW code.
 * Conventions follow the FFTW documentation: r2c is unnormalised with
 * e^{-2 pi i jk/n}; c2r is unnormalised with e^{+2 pi i jk/n}; the complex
 * half-array has n_last/2+1 entries on its last axis; row-major.
 */
#ifndef ROME_ORACLE_FFTW3_SHIM_H
#define ROME_ORACLE_FFTW3_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef double fftw_complex[2];
typedef float fftwf_complex[2];
typedef struct rome_fft_plan_s* fftw_plan;
typedef struct rome_fft_plan_s* fftwf_plan;
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_MEASURE (0U)
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)

fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double* in, fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex* in, double* out, unsigned flags);
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in, fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in, double* out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void fftw_cleanup(void);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int n);
void fftw_cleanup_threads(void);
void* fftw_malloc(size_t n);
void fftw_free(void* p);

fftwf_plan fftwf_plan_dft_r2c_2d(int n0, int n1, float* in, fftwf_complex* out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex* in, float* out, unsigned flags);
fftwf_plan fftwf_plan_dft_r2c_3d(int n0, int n1, int n2, float* in, fftwf_complex* out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_3d(int n0, int n1, int n2, fftwf_complex* in, float* out, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);
void fftwf_cleanup(void);
int fftwf_init_threads(void);
void fftwf_plan_with_nthreads(int n);
void fftwf_cleanup_threads(void);
void* fftwf_malloc(size_t n);
void fftwf_free(void* p);
#ifdef __cplusplus
}
#endif
#endif
