/*
 * Minimal stand-in for the parts of Intel MKL that the ROME MAP hot path
 * touches, so the reference sources build with g++ for use as a test oracle.
 * Project-written; contains no MKL code.
 *   - MKL_Complex8 / MKL_Complex16: plain {real, imag} structs
 *     (used as Vol<MKL_Complex16> in src/array.h and src/reconstruct.cpp)
 *   - LAPACKE_dlasrt('I'|'D', n, d): in-place sort
 *     (src/map3d_optimizer.cpp:1848, src/findBestPoints.cpp:77)
 *   - LAPACKE_dgels/sgels: abort if called (GTM-only, off the MAP path)
 */
#ifndef ROME_ORACLE_MKL_SHIM_H
#define ROME_ORACLE_MKL_SHIM_H
#include <stdlib.h>
#ifdef __cplusplus
#include <algorithm>
#include <functional>
extern "C++" {
#endif
typedef struct { float real, imag; } MKL_Complex8;
typedef struct { double real, imag; } MKL_Complex16;
typedef int lapack_int;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
#ifdef __cplusplus
static inline lapack_int LAPACKE_dlasrt(char id, lapack_int n, double* d) {
    if (n < 0) return -2;
    if (id == 'I' || id == 'i') std::sort(d, d + n);
    else if (id == 'D' || id == 'd') std::sort(d, d + n, std::greater<double>());
    else return -1;
    return 0;
}
static inline lapack_int LAPACKE_slasrt(char id, lapack_int n, float* d) {
    if (n < 0) return -2;
    if (id == 'I' || id == 'i') std::sort(d, d + n);
    else if (id == 'D' || id == 'd') std::sort(d, d + n, std::greater<float>());
    else return -1;
    return 0;
}
// Least-squares solvers are only reached from GTM initialisation
// (src/initialize.cpp:220-260), which the MAP path never calls.
static inline lapack_int LAPACKE_dgels(int, char, lapack_int, lapack_int, lapack_int, double*, lapack_int, double*,
                                       lapack_int) {
    abort();
}
static inline lapack_int LAPACKE_sgels(int, char, lapack_int, lapack_int, lapack_int, float*, lapack_int, float*,
                                       lapack_int) {
    abort();
}
}
#endif
#endif
