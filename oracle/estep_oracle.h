/*
 * CPU restatement of the ROME MAP E-step (test infrastructure only).
 *
 * This is the parity oracle for the GPU path: plain C, FP64, following the
 * reference's operation order.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg use it; the product never links it.
 * It is pinned against the reference itself (oracle/_ref, built from the
 * reference sources) through the golden vectors in tests/golden/.
 */
#ifndef ROME_ESTEP_ORACLE_H
#define ROME_ESTEP_ORACLE_H
#include "../include/rome_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Map2dOptimizer_old::expectationSomeParticles minus storeWeightedSums
 * (src/map2d_optimizer.cpp:802-854).  proj_data: MyProjector::data of the
 * K classes [K][pad_size][pad_size/2+1][2]; bp_data/bp_weight: the K
 * backprojectors, accumulated (+=) like MyBackProjector::backrotate2D. */
int oracle_map2d_estep_pool(const RomeMap2dPool* in, RomeMap2dPoolOut* out, int pad_size, int r_max,
                            int padding_factor, const double* proj_data, double* bp_data, double* bp_weight);

/* shiftImageInFourierTransform (src/image.h:1478-1575) */
void oracle_shift_image(const double* fin_real, const double* fin_imag, double* fout_real, double* fout_imag,
                        int size, double shift_x, double shift_y, int ori_size);

/* MyProjector::rotate2D (src/reconstruct.cpp:823-958), A = Euler(0,0,psi) */
void oracle_rotate2d(const double* proj_data, int pad_size, int r_max, int padding_factor, double psi_deg,
                     int f2d_size, double* f2d_real, double* f2d_imag);

/* MyBackProjector::backrotate2D (src/reconstruct.cpp:1353-1500) */
void oracle_backrotate2d(const double* f2d_real, const double* f2d_imag, const double* Mweight, int f2d_size,
                         double psi_deg, int pad_size, int r_max, int padding_factor, double* bp_data,
                         double* bp_weight);

/* findAllSignificantPoints selection for one row (src/map2d_optimizer.cpp:1243-1263) */
void oracle_select_significant(long len, const double* weights, double sum_weight, double adaptive_fraction,
                               double* significant_weight, double* nr_significant);

/* Euler_angles2matrix (src/math.cpp:86-115) */
void oracle_euler_matrix(double rot, double tilt, double psi, double A[9]);

#ifdef __cplusplus
}
#endif
#endif
