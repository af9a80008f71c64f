/*
 * rome_gpu.h - C ABI of the B200 (sm_100a) MAP classification hot path.
 *
 * Drop-in replacement for the E-step / M-step functions of ROME 1.1.2's
 * MAP optimizers.  The reference keeps its optimizer driver, options and
 * STAR/MRCS I/O; at each call site it hands plain host arrays (FP64, the
 * reference's FDOUBLE, src/macros.h:29-33) to the entry points below.
 * Each entry point names the reference function whose work it replaces.
 *
 * Conventions
 *  - Every function returns ROME_OK (0) or a ROME_ERR_* code; the text of
 *    the last error is available from rome_gpu_last_error().  Nothing
 *    throws and nothing exits the process (the reference's ERROR_REPORT,
 *    src/error.h:95-99, becomes an error code).
 *  - Arrays use the reference layouts: Fourier images in the FFTW half
 *    plane [size][size/2+1], row-major, rows wrapping to negative
 *    frequencies (src/reconstruct.cpp:279-291); complex data as separate
 *    real / imaginary arrays unless stated otherwise.
 *  - A context is bound to one CUDA device and is not thread-safe; use one
 *    context per host thread.  Calls block until their outputs are in the
 *    caller's buffers.
 *  - Accumulated outputs (wsum_*, backprojectors) are added to (+=), as the
 *    reference accumulates into mlModel.wsum_* and backprojector[k].
 */
#ifndef ROME_GPU_H
#define ROME_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ROME_GPU_ABI_VERSION 4

enum RomeStatus {
    ROME_OK = 0,
    ROME_ERR_ARG = 1,         /* invalid argument or inconsistent sizes */
    ROME_ERR_OOM = 2,         /* device allocation failed */
    ROME_ERR_CUDA = 3,        /* CUDA runtime / launch error */
    ROME_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up */
    ROME_ERR_NUMERIC = 5,     /* NaN/Inf or an empty posterior (exp_sum_weight == 0) */
    ROME_ERR_STATE = 6,       /* call order violated (e.g. no projectors uploaded) */
    ROME_ERR_UNSUPPORTED = 7  /* option combination not implemented */
};

/* Arithmetic of the diff2 cross term Re<X_i, P_j> (the dense contraction).
 * The min-diff2 subtraction, exp/normalisation of posteriors and all
 * Fourier-weight sums are FP64 in every mode. */
enum RomePrecision {
    ROME_PREC_FP32 = 0,   /* CUDA-core FP32 FMA, FP32 accumulate ("plain FP32") */
    ROME_PREC_BF16 = 1,   /* tcgen05 BF16 x BF16, FP32 accumulate in TMEM */
    ROME_PREC_BF16X3 = 2  /* tcgen05 split precision: hi*hi + hi*lo + lo*hi */
};

typedef struct RomeGpuCtx RomeGpuCtx;

typedef struct {
    int precision;           /* RomePrecision */
    int deterministic;       /* nonzero: fixed-order reductions where the ABI allows */
    size_t workspace_limit;  /* device scratch cap in bytes, 0 = automatic (1.5 GiB); bounds the
                                work buffers of rome_gpu_prepare_particles, which then runs in chunks */
    int profile;             /* nonzero: time each phase with CUDA events (rome_gpu_get_timings) */
} RomeGpuConfig;

/* Per-phase device time (CUDA events on the context's stream, summed over
 * calls since the last reset) and launch counts.  The phases follow the
 * reference's E-step functions. */
enum RomePhase {
    ROME_PHASE_PREP = 0,      /* window, CTF, Minvsigma2 */
    ROME_PHASE_PROJECT,       /* getReferenceAllOrientations */
    ROME_PHASE_SHIFT,         /* shifted images -> contraction operand */
    ROME_PHASE_NORM_GEMM,     /* sum_n Minvsigma2 ctf^2 |P|^2 */
    ROME_PHASE_CROSS_GEMM,    /* Re<X_t, P> over all images x orientations (dominant) */
    ROME_PHASE_POSTERIOR,     /* weights, sum, argmax, significance */
    ROME_PHASE_WSUM,          /* updateOtherParams */
    ROME_PHASE_BACKPROJECT,   /* backProjection */
    ROME_PHASE_RECONSTRUCT,   /* MyBackProjector::reconstruct */
    ROME_PHASE_RESTRICTED,    /* diff2 over each particle's proposed orientations only */
    ROME_PHASE_PROPOSE,       /* proposal network: features, forward, top-k, expansion */
    ROME_PHASE_IMAGES,        /* setFourierTransforms: translate, noise, soft mask, FFTs, CTF */
    ROME_PHASE_COUNT
};

typedef struct {
    double ms[ROME_PHASE_COUNT];        /* device milliseconds per phase */
    long launches[ROME_PHASE_COUNT];    /* kernel launches per phase */
    double flops[ROME_PHASE_COUNT];     /* algorithmic flops per phase (contractions) */
    double bytes[ROME_PHASE_COUNT];     /* algorithmic bytes per phase (HBM-bound kernels) */
    long total_launches;                /* all kernels of this library since the last reset */
} RomeGpuTimings;

int rome_gpu_get_timings(RomeGpuCtx* ctx, RomeGpuTimings* out);

/* The tensor-core contractions' tile-shape autotuner (no reference
 * counterpart): the first call of a contraction with a new key (kind,
 * operand planes, device, N, Kp, 128-row tiles rounded up to a power of
 * two) times every candidate tile shape on its own operands and keeps the
 * fastest; all candidates give identical outputs.  ROME_TC_TUNE=0 in the
 * environment disables it (default shapes); ROME_TC_SHAPE=<i> pins
 * candidate i of every list.  Writes one line per key with
 * the choice and every candidate's time (process-wide, all contexts) into
 * buf (NUL-terminated, truncated to len) and returns the full length. */
size_t rome_gpu_tuning_report(char* buf, size_t len);
int rome_gpu_reset_timings(RomeGpuCtx* ctx);

/* Context lifetime.  Replaces nothing in the reference (it owns no device). */
int rome_gpu_create(int device, const RomeGpuConfig* cfg, RomeGpuCtx** out);
int rome_gpu_destroy(RomeGpuCtx* ctx);
const char* rome_gpu_last_error(const RomeGpuCtx* ctx);
int rome_gpu_set_precision(RomeGpuCtx* ctx, int precision);
int rome_gpu_abi_version(void);

/* Upload the K class projectors and reset the K backprojectors to zero.
 * Replaces the projector side of MAPModel::setFourierTransformMaps
 * (src/map_model.cpp:136-160): `data` is MyProjector::data of every class
 * (src/reconstruct.cpp:44-59, 106-223), interleaved complex
 * [K][pad_z][pad_size][pad_size/2+1][2], pad_z = pad_size (3D) or 1 (2D).
 * r_max and padding_factor are ProjectorBase::r_max / padding_factor. */
int rome_gpu_set_projectors(RomeGpuCtx* ctx, int ref_dim, int nr_classes, int ori_size, int pad_size, int r_max,
                            int padding_factor, const double* data);

/* The pools of one EM iteration share the coarse-pass projections of every
 * class and orientation: a 2D pool whose model, sampling tables and
 * precision equal the previous call's reuses them (the reference recomputes
 * them per pool, getReferenceAllOrientations, src/map2d_optimizer.cpp:
 * 857-905).  rome_gpu_set_projectors starts a new model; this marks the
 * cached projections stale without uploading anything, so that the next
 * pool recomputes them (one projection per iteration when the model changed
 * on the device, or to time an iteration as a whole). */
int rome_gpu_invalidate_projections(RomeGpuCtx* ctx);

/* Download (and optionally reset) the accumulated backprojector of one
 * class: MyBackProjector::data (interleaved complex) and ::weight, same
 * shape as the projector.  Used for the reduction across ranks
 * (src/map_model.cpp:604-620) and before MAPModel::reconstruction. */
int rome_gpu_get_backprojector(RomeGpuCtx* ctx, int iclass, double* data, double* weight);
int rome_gpu_set_backprojector(RomeGpuCtx* ctx, int iclass, const double* data, const double* weight);
/* dst's back-projectors (all classes, data and weight) += src's, on the
 * device; both contexts on the same device with the same projector shape.
 * clear_src: zero src's afterwards.  For pools of one iteration spread over
 * several contexts (e.g. one per host thread); the reference's counterpart is
 * the per-thread replica reduction MAPModel::reduceThreadMap
 * (src/map_model.cpp:209-231). */
int rome_gpu_add_backprojectors(RomeGpuCtx* dst, RomeGpuCtx* src, int clear_src);

/* Device-resident exchange of the back-projectors across ranks (the
 * reference's MAPModel::reduceData, src/map_model.cpp:604-666, all-reduces
 * or reduces them over MPI).  rome_gpu_backprojector_size gives the number
 * of doubles of all classes' back-projectors, 3 * voxels * K: data as
 * interleaved complex [K][voxels][2], then weight [K][voxels].
 * rome_gpu_backprojector_device_copy copies them between the library and a
 * caller's device buffer of that size on the context's device (to_library
 * 0: library -> dev_buf, 1: dev_buf -> library), device to device, on
 * `stream` (NULL: the context's stream) after the context's pending work;
 * it returns when the copy is done.  A collective (NCCL all-reduce or
 * per-class reduce) then runs on the buffer without any host copy. */
int rome_gpu_backprojector_size(RomeGpuCtx* ctx, size_t* doubles);
int rome_gpu_backprojector_device_copy(RomeGpuCtx* ctx, int to_library, void* dev_buf, void* stream);

/* Back-projection of n particle images at known poses into class iclass's
 * 3D back-projector: the per-image loop of the reference's rome_reconstruct
 * (apps/rome_reconstruct.cpp:160-330).  Fimg_real/imag: [n][size][size/2+1]
 * FFTW half-plane transforms of the centred images (what the image
 * preparation returns as the unmasked transform, with zero old offsets, at
 * current size = size).  Fctf: [n][size][size/2+1] CTF images, or NULL for
 * no CTF.  poses: [n][5] = rot, tilt, psi (degrees), xoff, yoff (pixels),
 * host memory.  Each image is shifted by (xoff, yoff) with the tabulated
 * phases of shiftImageInFourierTransform (src/image.h:1478-1575),
 * multiplied by its CTF and scattered with weight CTF^2 by
 * MyBackProjector::backproject (src/reconstruct.cpp:977-1164); the volume
 * accumulates (+=) until rome_gpu_set_projectors or
 * rome_gpu_set_backprojector replaces it.  A zero
 * offset leaves the spectrum unshifted.  inputs_on_device: Fimg_* and Fctf
 * are device pointers.  size must equal the back-projector's ori_size;
 * follow with rome_gpu_reconstruct (do_map 0, normalise 1) for the
 * reference's reconstruction. */
int rome_gpu_backproject_images(RomeGpuCtx* ctx, int iclass, int n, int size, const double* Fimg_real,
                                const double* Fimg_imag, const double* Fctf, const double* poses,
                                int inputs_on_device);

/* ---------------------------------------------------------------------
 * Particle image preparation for one pool.  Replaces
 * ParticleModel::setFourierTransforms (src/exp_model.h:397-640), called by
 * the optimizers' expectation() before expectationSomeParticles: norm
 * correction, translation by the rounded old offsets (no wrap), the
 * centred, normalised Fourier transform windowed to current_size
 * (Fimages_nomask); a noise image drawn from sigma2_noise with the
 * reference's seeded generator (seed random_seed + first_image + i, glibc
 * srand/rand through Random_generator::rnd_gaus) blended outside the
 * particle diameter with a raised-cosine edge (softMaskOutsideMap), or the
 * background average when do_zero_mask; its windowed transform
 * (Fimages_mask_fine), power spectrum and highres_Xi2 (when current_size <
 * ori_size), and the CTF image (CTF::getFftwImage).  The outputs are the
 * image inputs of rome_gpu_map2d_estep_pool; with outputs_on_device they
 * can be handed to it without leaving the device (inputs_on_device).
 * Even ori_size only; current_size <= ori_size.
 * ------------------------------------------------------------------- */
typedef struct {
    int nr_images;          /* exp_nr_images (P) */
    int ori_size;
    int current_size;       /* fine_size */
    int nr_groups;
    int first_image;        /* exp_first_image: part of the noise seed */
    const void* images;     /* exp_images as read [P][ori_size][ori_size] */
    int image_type;         /* 0: double (FDOUBLE), 1: float (MRC mode 2 as stored) */
    int images_on_device;   /* nonzero: `images` is a device pointer on the context's device */
    /* exp_metadata fields [P] (host) */
    const double* norm;     /* NORM */
    const double* xoff;     /* XOFF, YOFF (the old offsets before rounding) */
    const double* yoff;
    const double* ctf_defocus_u;
    const double* ctf_defocus_v;
    const double* ctf_defocus_angle;
    const double* ctf_voltage;
    const double* ctf_cs;
    const double* ctf_q0;
    const double* ctf_bfac;
    const int* group;                /* GROUP_NO - 1 [P] */
    const double* sigma2_noise;      /* mlModel.sigma2_noise [nr_groups][ori_size/2+1] */
    double avg_norm_correction;      /* mlModel.avg_norm_correction */
    double pixel_size;
    double particle_diameter;        /* Angstrom */
    double sigma2_fudge;
    int width_mask_edge;             /* pixels */
    int random_seed;
    int do_norm_correction;
    int do_zero_mask;
    int do_ctf_correction;
    int ctf_phase_flipped;           /* CTF image as |ctf| */
    int only_flip_phases;            /* CTF image as sign(ctf) */
    int intact_ctf_first_peak;
} RomePrepIn;

typedef struct {
    /* [P][current_size][current_size/2+1]: Fimages_mask_fine, Fimages_nomask, Fctfs */
    double* Fimg_real;
    double* Fimg_imag;
    double* Fimg_nomask_real;
    double* Fimg_nomask_imag;
    double* Fctf;
    int outputs_on_device;  /* nonzero: the five arrays above are device pointers on the context's device */
    /* host [P] */
    double* highres_Xi2;    /* exp_highres_Xi2_imgs */
    double* old_offsetx;    /* exp_old_offsetx / y: round(XOFF), round(YOFF) */
    double* old_offsety;
    double* power_imgs;     /* host [P][ori_size/2+1] exp_power_imgs (zero when current_size == ori_size); NULL to skip */
} RomePrepOut;

int rome_gpu_prepare_particles(RomeGpuCtx* ctx, const RomePrepIn* in, RomePrepOut* out);

/* ---------------------------------------------------------------------
 * MAP2D E-step for one pool of particles.
 * Replaces Map2dOptimizer_old::expectationSomeParticles
 * (src/map2d_optimizer.cpp:802-854): for every pass, the shifted images
 * (ParticleModel::preShiftedImagesCtfsAndInvSigma2s, src/exp_model.cpp:935-1104),
 * getReferenceAllOrientations (:856-904), getAllSquaredDifferences
 * (:907-1074), convertSquaredDifferencesToWeights (:1077-1224) and
 * findAllSignificantPoints (:1226-1311); then updateOtherParams
 * (:1417-1663) and backProjection (:1666-1873).  storeWeightedSums
 * (:1314-1414) stays on the host: it needs only the per-particle outputs.
 * ------------------------------------------------------------------- */
typedef struct {
    int nr_images;             /* exp_nr_images (P) */
    int ori_size;              /* image size */
    int current_size;          /* fine size of this iteration */
    int coarse_size;           /* size of pass 0 when adaptive_oversampling > 0 */
    int nr_classes;            /* K */
    int iclass_min, iclass_max;/* exp_iclass_min/max */
    int nr_groups;
    int adaptive_oversampling; /* 0: one pass; 1: coarse + fine pass */
    int nr_psi;                /* coarse in-plane angles (exp_nr_psi) */
    int nr_trans;              /* coarse translations (exp_nr_trans) */
    /* SamplingGrid::exp_over_psi [nr_psi][nr_over_rot] for pass 0 and 1
     * (pass 1 only if adaptive_oversampling > 0); degrees */
    const double* over_psi[2];
    /* SamplingGrid::exp_over_trans_x/y [nr_trans][nr_over_trans] per pass */
    const double* over_trans_x[2];
    const double* over_trans_y[2];
    /* HealpixSampler translations_x/y [nr_trans] (the coarse grid the
     * offset prior uses, src/map2d_optimizer.cpp:1116-1121) */
    const double* trans_x;
    const double* trans_y;
    /* particle images after ParticleModel::setFourierTransforms, at
     * current_size: Fimages_mask_fine, Fimages_nomask, Fctfs
     * [P][current_size][current_size/2+1] */
    const double* Fimg_real;
    const double* Fimg_imag;
    const double* Fimg_nomask_real;
    const double* Fimg_nomask_imag;
    const double* Fctf;
    const double* highres_Xi2;  /* exp_highres_Xi2_imgs [P] */
    const double* old_offsetx;  /* exp_old_offsetx [P] (rounded old offsets) */
    const double* old_offsety;
    const int* group;           /* GROUP_NO - 1 [P] */
    /* model */
    const double* sigma2_noise;        /* [nr_groups][ori_size/2+1] */
    const int* Mresol_fine;            /* [current_size][current_size/2+1] */
    const int* Mresol_coarse;          /* [coarse_size][coarse_size/2+1] */
    const double* pdf_class;           /* [K] */
    const double* pdf_direction;       /* [K] (one direction in 2D) */
    const double* prior_offsetx_class; /* [K] */
    const double* prior_offsety_class; /* [K] */
    double sigma2_offset;
    double sigma2_fudge;
    double adaptive_fraction;
    int do_ctf_correction;
    int refs_are_ctf_corrected;
    int do_map;
    /* nonzero: Fimg_real/imag, Fimg_nomask_real/imag and Fctf are device
     * pointers on the context's device (no host-to-device copy) */
    int inputs_on_device;
    /* optional search restriction (adaptive_oversampling 0 only; no
     * reference counterpart): per particle nr_proposals orientation indices
     * j = class * nr_psi + psi, ascending and distinct (host array
     * [P][nr_proposals]); only those orientations, with every translation,
     * are evaluated, and the posterior is normalised over them.  NULL: the
     * exhaustive search of the reference. */
    const int* proposals;
    int nr_proposals;
    /* optional, with inputs_on_device only (no reference counterpart): host
     * array [P]; particle i's images are row particle_rows[i] of the device
     * image arrays (a subset of a staged pool without copying it).  The
     * per-particle host arrays (highres_Xi2, offsets, group, proposals) are
     * given in the processed order.  NULL: row i. */
    const int* particle_rows;
} RomeMap2dPool;

typedef struct {
    /* per particle [P] */
    double* min_diff2;           /* exp_min_diff2 (last pass) */
    double* sum_weight;          /* exp_sum_weight (last pass) */
    double* significant_weight;  /* exp_significant_weight (last pass) */
    double* wsum_norm_correction;/* exp_wsum_norm_correction (updateOtherParams) */
    double* pmax;                /* exp_metadata PMAX, CLASS (1-based), PSI, XOFF, YOFF, NR_SIGN */
    int* cls;
    double* psi;
    double* xoff;
    double* yoff;
    double* nr_sign;
    /* accumulated model sums (+=) */
    double* wsum_sigma2_noise;        /* [nr_groups][ori_size/2+1] */
    double* wsum_pdf_class;           /* [K] */
    double* wsum_pdf_direction;       /* [K] */
    double* wsum_prior_offsetx_class; /* [K] */
    double* wsum_prior_offsety_class; /* [K] */
    double* wsum_sigma2_offset;       /* [1] */
    double* wsum_sumw_group;          /* [nr_groups] */
    /* optional checkpoints in the reference's exp_Mweight layout
     * [P][K * NrPoints(pass)] (class -> psi -> over_rot -> trans -> over_trans);
     * entries that were not computed hold INT_MIN (diff2) or 0 (weight).
     * NULL to skip. */
    double* diff2[2];
    double* weight[2];
    char* Mcoarse_significant;        /* [P][K * nr_psi * nr_trans] (pass 0) */
    /* optional [P][K * nr_psi]: the significant normalised weights of the
     * last pass summed per (class, psi) (the posterior the proposal network
     * is trained on); NULL to skip */
    double* post_class_psi;
} RomeMap2dPoolOut;

int rome_gpu_map2d_estep_pool(RomeGpuCtx* ctx, const RomeMap2dPool* in, RomeMap2dPoolOut* out);

/* ---------------------------------------------------------------------
 * MAP3D E-step for one pool of particles: both sampling passes,
 * updateOtherParams and backProjection.  Replaces
 * Map3dOptimizer_old::expectationSomeParticles minus storeWeightedSums
 * (src/map3d_optimizer.cpp:883-953): preShiftedImagesCtfsAndInvSigma2s,
 * getReferenceAllOrientations (:956-985), getAllSquaredDifferences
 * (coarse :1195-1259, fine :1261-1372), convertSquaredDifferencesToWeights
 * (:1610-1810), findAllSignificantPoints (:1812-1931), updateOtherParams
 * (:2059-2236, CoarseAndFineSearch::updateModel :1484-1602) and
 * backProjection (:2242-2506, MyBackProjector::backproject
 * src/reconstruct.cpp:977-1164), with adaptive_oversampling 1 (the
 * reference's 3D path always has the fine pass).  Maximum-likelihood mode,
 * or cross-correlation mode (do_cross_correlation: the reference's
 * (iter == 1 && do_firstiter_cc) || do_always_cc, :907): every hypothesis
 * scored by -sum(Frefctf . X) / (|Frefctf| |X|) (get_diff, :1086-1102) and
 * only the best one kept with weight 1 (:1626-1671).  Intensity-scale
 * correction (do_scale_correction): each group's scale multiplies the
 * references and the CTF of the back-projection (applyCtfToClass
 * :1054-1066, :2274-2282) and the per-particle XA/AA spectra of
 * updateModel (:1426-1502, :2090-2112) are returned.  Either mode with
 * proposals returns ROME_ERR_UNSUPPORTED.  Projectors must be set with
 * ref_dim 3.
 * ------------------------------------------------------------------- */
typedef struct {
    int nr_images;
    int ori_size, current_size, coarse_size;
    int nr_classes, iclass_min, iclass_max;
    int nr_groups;
    int adaptive_oversampling;       /* 1 */
    int nr_dir, nr_psi, nr_trans;    /* coarse grid: HEALPix directions, psi, translations */
    /* samplingGrid.setOrientation of every (dir, psi), per pass:
     * [nr_dir][nr_psi][nr_over_rot][3] = (rot, tilt, psi) in degrees;
     * nr_over_rot = 1 in pass 0, 8 in pass 1 */
    const double* angles[2];
    /* samplingGrid.exp_over_trans_x/y per pass: [nr_trans][nr_over_trans] (1 / 4) */
    const double* over_trans_x[2];
    const double* over_trans_y[2];
    const double* trans_x;           /* sampler3d.getTranslation: [nr_trans] */
    const double* trans_y;
    /* particle data at current_size (Fourier half-planes), as in RomeMap2dPool */
    const double* Fimg_real;
    const double* Fimg_imag;
    const double* Fimg_nomask_real;
    const double* Fimg_nomask_imag;
    const double* Fctf;
    const double* highres_Xi2;
    const double* old_offsetx;
    const double* old_offsety;
    const int* group;
    const double* sigma2_noise;      /* [G][ori/2+1] */
    const int* Mresol_fine;
    const int* Mresol_coarse;
    const double* pdf_class;         /* [K] */
    const double* pdf_direction;     /* [K][nr_dir] */
    const double* prior_offsetx_class;
    const double* prior_offsety_class;
    double sigma2_offset;
    double sigma2_fudge;
    double adaptive_fraction;
    int do_ctf_correction;
    int refs_are_ctf_corrected;
    int do_map;
    int do_scale_correction;
    int do_cross_correlation;
    int inputs_on_device;
    /* optional coarse-pass search restriction (no reference counterpart): per
     * particle nr_proposals coarse orientations j = (class * nr_dir + dir) *
     * nr_psi + psi, ascending and distinct (host array [P][nr_proposals]);
     * the coarse pass evaluates only those, with every translation, and the
     * fine pass refines the coarse-significant points among them as usual.
     * NULL: the exhaustive coarse pass of the reference. */
    const int* proposals;
    int nr_proposals;
    /* with do_scale_correction: mlModel.scale_correction [nr_groups] and
     * mlModel.data_vs_prior_class [nr_classes][ori_size/2+1] (the shells
     * whose data_vs_prior exceeds 3 enter the XA/AA spectra); a scale is
     * checked like check_scale (:1000-1018): NaN, Inf or > 10000 is
     * ROME_ERR_NUMERIC, below 0.001 it is raised to 0.001 */
    const double* scale_correction;
    const double* data_vs_prior_class;
} RomeMap3dPool;

typedef struct {
    /* per particle, final pass (NULL to skip) */
    double* min_diff2;
    double* sum_weight;
    double* significant_weight;
    double* wsum_norm_correction;
    double* pmax;
    int* cls;                        /* 1-based */
    double* rot;
    double* tilt;
    double* psi;
    double* xoff;
    double* yoff;
    double* nr_sign;                 /* coarse-pass NR_SIGN */
    /* model sums, accumulated */
    double* wsum_sigma2_noise;       /* [G][ori/2+1] */
    double* wsum_pdf_class;          /* [K] */
    double* wsum_pdf_direction;      /* [K][nr_dir] */
    double* wsum_sigma2_offset;      /* [1] */
    double* wsum_sumw_group;         /* [G] */
    /* optional checkpoints (NULL to skip) */
    double* pass_min_diff2[2];       /* [P] */
    double* pass_sum_weight[2];      /* [P] */
    double* pass_significant_weight[2]; /* [P] */
    double* coarse_diff2;            /* [P][K][nr_dir][nr_psi][nr_trans], INT_MIN where not computed */
    char* Mcoarse_significant;       /* [P][K * nr_dir * nr_psi * nr_trans] */
    /* fine-pass hypotheses in the reference's list order: per particle
     * fine_count[i] records of (coarse index (k,dir,psi,trans) * 32 +
     * over_rot * 4 + over_trans, diff2, weight); capacity fine_capacity */
    long fine_capacity;
    int* fine_count;                 /* [P] */
    long* fine_index;
    double* fine_diff2;
    double* fine_weight;
    /* optional (no reference counterpart): the coarse pass's significant
     * normalised weights summed per coarse orientation, [P][K * nr_dir * nr_psi]
     * (training targets of the proposal network) */
    double* post_coarse;
    /* with do_scale_correction: exp_wsum_scale_correction_XA / _AA as
     * updateOtherParams leaves them, [nr_images][ori_size/2+1] per resolution
     * shell (overwritten, not accumulated; storeWeightedSums divides them by
     * the scale and its square and adds them to the group spectra); NULL to
     * skip */
    double* wsum_scale_correction_XA;
    double* wsum_scale_correction_AA;
} RomeMap3dPoolOut;

int rome_gpu_map3d_estep_pool(RomeGpuCtx* ctx, const RomeMap3dPool* in, RomeMap3dPoolOut* out);

/* Significance selection on given weights (findAllSignificantPoints,
 * src/map2d_optimizer.cpp:1226-1311 and src/map3d_optimizer.cpp:1812-1931):
 * for each of n rows of `len` weights, sort the positive weights, walk from
 * the largest until the running FP64 sum exceeds adaptive_fraction * sum[i],
 * and return that weight and the number of weights walked.  Exposed for
 * bit-exact checks of the selection with caller-provided weights. */
int rome_gpu_select_significant(RomeGpuCtx* ctx, int n, long len, const double* weights, const double* sum_weight,
                                double adaptive_fraction, double* significant_weight, double* nr_significant);

/* Same selection and results as rome_gpu_select_significant, without any
 * device allocation: every device buffer lives in one fixed array compiled
 * into the library (about 16.5 MiB per device).  No counterpart in the
 * reference; it is for callers that must not allocate device memory during
 * the call (all HBM handed to their own pool, a hard memory budget, or no
 * implicit synchronisation from cudaMalloc/cudaFree allowed).
 * Limits: n <= ROME_SELECT_STATIC_MAX_IMAGES, n * len <=
 * ROME_SELECT_STATIC_MAX_WEIGHTS; beyond them it returns ROME_ERR_ARG.
 * The first call on a device looks the array up (cudaGetSymbolAddress) and
 * should come before any stream capture on that device.  With lazy module
 * loading (CUDA's default) that first call may also load the library's
 * device code on the device, which is when the driver reserves the array
 * and the code: treat it as a warm-up; from the second call on, nothing is
 * allocated.  The call is synchronous: it returns once the results are in
 * the caller's host arrays.  Calls on one device share the array, so
 * overlapping calls would race: the function takes a process-wide lock and
 * returns after its stream work is done. */
#define ROME_SELECT_STATIC_MAX_IMAGES 4096
#define ROME_SELECT_STATIC_MAX_WEIGHTS (1 << 20)
int rome_gpu_select_significant_static(RomeGpuCtx* ctx, int n, long len, const double* weights,
                                       const double* sum_weight, double adaptive_fraction,
                                       double* significant_weight, double* nr_significant);

/* ---------------------------------------------------------------------
 * Host -> device copy of page-locked host memory by a kernel on the given
 * CUDA stream (0: the context's stream), reading the host buffer through
 * the unified address space instead of using a copy engine.  No reference
 * counterpart: callers staging the next pool's images while the current
 * pool computes use it so that the E-step's own small uploads do not queue
 * behind the large transfer.  host: page-locked (cudaHostAlloc /
 * cudaHostRegister), dst: device memory; both 16-byte aligned.  Returns
 * ROME_ERR_ARG for pageable or unaligned buffers.  Asynchronous.
 * ------------------------------------------------------------------- */
int rome_gpu_copy_from_host(RomeGpuCtx* ctx, void* dst, const void* host, size_t bytes, void* stream);

/* ---------------------------------------------------------------------
 * Failure-handling check of the bounded device waits.  No reference
 * counterpart (the reference has no device code): every tensor-core kernel
 * waits on mbarriers with a bound (2 s) after which it records a timeout in
 * the context's error flag, drains and returns, and the entry point reports
 * ROME_ERR_TIMEOUT with the context still usable.  This launches one wait
 * on an mbarrier that nothing arrives on, bounded by limit_seconds (1e-4 to
 * 2), so that callers and tests can see that path run out: it returns
 * ROME_ERR_TIMEOUT and the measured wait in *waited_seconds (may be null).
 * ------------------------------------------------------------------- */
int rome_gpu_wait_selftest(RomeGpuCtx* ctx, double limit_seconds, double* waited_seconds);

/* ---------------------------------------------------------------------
 * M-step reconstruction of one class from its accumulated backprojector.
 * Replaces MAPModel::reconstruction (src/map_model.cpp:233-241) ->
 * MyBackProjector::reconstruct (src/reconstruct.cpp:1929-2526) with the
 * map2d/map3d defaults (trilinear, padding 2, no FSC update, C1).
 * ------------------------------------------------------------------- */
typedef struct {
    int iclass;
    int gridding_nr_iter;     /* max_iter_preweight (10) */
    int do_map;
    int minres_map;
    double tau2_fudge;
    double normalise;         /* wsum_pdf_class[iclass] */
    const double* tau2_in;    /* [ori_size/2+1] */
} RomeReconIn;

typedef struct {
    double* vol;              /* [ori_size^ref_dim] real-space reference (Irefs[iclass]) */
    double* tau2;             /* [ori_size/2+1] (unchanged unless FSC update) */
    double* sigma2;           /* [ori_size/2+1] */
    double* data_vs_prior;    /* [ori_size/2+1] */
} RomeReconOut;

int rome_gpu_reconstruct(RomeGpuCtx* ctx, const RomeReconIn* in, RomeReconOut* out);

/* ---------------------------------------------------------------------
 * Learned pose proposals (no counterpart in the reference).  A small
 * network over a particle's Fourier magnitude in polar coordinates
 * (rotation = circular shift along the angle, every layer equivariant to
 * it) predicts a distribution over (class, psi mod 180); it is trained on
 * the GPU on (image, posterior) pairs produced by the exhaustive E-step, and
 * its top-k outputs restrict the E-step's search (RomeMap2dPool.proposals).
 * Input: x[n][2][n_r][n_theta] (rome_gpu_proposal_features); output index
 * o = class * n_theta + psi index mod n_theta, n_theta = nr_psi / 2.
 * ------------------------------------------------------------------- */
typedef struct {
    int n_r;            /* radial samples */
    int n_theta;        /* angular samples over [0, 180) deg: nr_psi / 2 */
    int channels[2];    /* the two 3x3 convolution layers */
    int n_classes;      /* K */
    double r_lo, r_hi;  /* radius range in Fourier pixels of the feature image */
} RomeProposalSpec;

typedef struct RomeProposalNet RomeProposalNet;

int rome_gpu_proposal_create(RomeGpuCtx* ctx, const RomeProposalSpec* spec, unsigned long long seed,
                             RomeProposalNet** net);
void rome_gpu_proposal_destroy(RomeProposalNet* net);
long rome_gpu_proposal_num_params(const RomeProposalNet* net);
/* flat parameters w0 b0 w1 b1 wf bf, each block at a multiple of 4 floats */
int rome_gpu_proposal_get_params(RomeProposalNet* net, float* params);
int rome_gpu_proposal_set_params(RomeProposalNet* net, const float* params);
/* network input of P particles from their masked Fourier images and CTFs
 * at size cur (FFTW half-planes, FP64; host arrays, or device arrays with
 * inputs_on_device), written to host memory */
int rome_gpu_proposal_features(RomeProposalNet* net, int P, int cur, const double* Fimg_real,
                               const double* Fimg_imag, const double* ctf, int inputs_on_device, float* x);
/* mean soft-target cross-entropy of n samples, its gradient (flat, as the
 * parameters) and the logits [n][n_classes * n_theta]; outputs may be NULL */
int rome_gpu_proposal_loss_grad(RomeProposalNet* net, int n, const float* x, const float* targets, double* loss,
                                float* grad, float* logits);
/* Adam (beta 0.9 / 0.999) over shuffled mini-batches; epoch_loss[epochs] */
int rome_gpu_proposal_train(RomeProposalNet* net, int n, const float* x, const float* targets, int epochs,
                            int batch, float lr, unsigned long long seed, double* epoch_loss);
/* top-k outputs per sample (descending) and their softmax probabilities */
int rome_gpu_proposal_predict(RomeProposalNet* net, int n, const float* x, int k, int* idx, float* prob);
/* features + top-k of P particles (Fourier images and CTFs at size cur,
 * host arrays, or device arrays on the context's device when
 * inputs_on_device), expanded to the restricted E-step's input: proposals
 * [P][2k] ascending orientation indices class * 2 n_theta + psi (host), and
 * the probability mass of the k outputs per particle (host, may be NULL);
 * k <= 64 */
int rome_gpu_proposal_propose(RomeProposalNet* net, int P, int cur, const double* Fimg_real, const double* Fimg_imag,
                              const double* ctf, int inputs_on_device, int k, int* proposals, float* mass);

#ifdef __cplusplus
}
#endif

#endif /* ROME_GPU_H */
