"""ctypes view of the C ABI declared in include/rome_gpu.h.

The structures mirror the header field by field; `load_library()` opens the
in-tree ``librome_b200.so`` built by ``rome_b200/build.py`` and raises if it
is missing (the product has no CPU fallback).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

ROME_OK = 0
ROME_ERR_ARG = 1
ROME_ERR_OOM = 2
ROME_ERR_CUDA = 3
ROME_ERR_TIMEOUT = 4
ROME_ERR_NUMERIC = 5
ROME_ERR_STATE = 6
ROME_ERR_UNSUPPORTED = 7

ROME_PREC_FP32 = 0
ROME_PREC_BF16 = 1
ROME_PREC_BF16X3 = 2

PRECISIONS = {"fp32": ROME_PREC_FP32, "bf16": ROME_PREC_BF16, "bf16x3": ROME_PREC_BF16X3}

_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)
_CP = C.POINTER(C.c_char)


class RomeGpuConfig(C.Structure):
    _fields_ = [("precision", C.c_int), ("deterministic", C.c_int), ("workspace_limit", C.c_size_t),
                ("profile", C.c_int)]


ABI_VERSION = 4  # ROME_GPU_ABI_VERSION of include/rome_gpu.h

PHASES = ["prep", "project", "shift", "norm_gemm", "cross_gemm", "posterior", "wsum", "backproject", "reconstruct",
          "restricted", "propose", "images"]


class RomeGpuTimings(C.Structure):
    _fields_ = [("ms", C.c_double * len(PHASES)), ("launches", C.c_long * len(PHASES)),
                ("flops", C.c_double * len(PHASES)), ("bytes", C.c_double * len(PHASES)),
                ("total_launches", C.c_long)]


class RomeMap2dPool(C.Structure):
    _fields_ = [
        ("nr_images", C.c_int), ("ori_size", C.c_int), ("current_size", C.c_int), ("coarse_size", C.c_int),
        ("nr_classes", C.c_int), ("iclass_min", C.c_int), ("iclass_max", C.c_int), ("nr_groups", C.c_int),
        ("adaptive_oversampling", C.c_int), ("nr_psi", C.c_int), ("nr_trans", C.c_int),
        ("over_psi", _DP * 2), ("over_trans_x", _DP * 2), ("over_trans_y", _DP * 2),
        ("trans_x", _DP), ("trans_y", _DP),
        ("Fimg_real", _DP), ("Fimg_imag", _DP), ("Fimg_nomask_real", _DP), ("Fimg_nomask_imag", _DP),
        ("Fctf", _DP), ("highres_Xi2", _DP), ("old_offsetx", _DP), ("old_offsety", _DP), ("group", _IP),
        ("sigma2_noise", _DP), ("Mresol_fine", _IP), ("Mresol_coarse", _IP),
        ("pdf_class", _DP), ("pdf_direction", _DP), ("prior_offsetx_class", _DP), ("prior_offsety_class", _DP),
        ("sigma2_offset", C.c_double), ("sigma2_fudge", C.c_double), ("adaptive_fraction", C.c_double),
        ("do_ctf_correction", C.c_int), ("refs_are_ctf_corrected", C.c_int), ("do_map", C.c_int),
        ("inputs_on_device", C.c_int), ("proposals", _IP), ("nr_proposals", C.c_int), ("particle_rows", _IP),
    ]


class RomeMap2dPoolOut(C.Structure):
    _fields_ = [
        ("min_diff2", _DP), ("sum_weight", _DP), ("significant_weight", _DP), ("wsum_norm_correction", _DP),
        ("pmax", _DP), ("cls", _IP), ("psi", _DP), ("xoff", _DP), ("yoff", _DP), ("nr_sign", _DP),
        ("wsum_sigma2_noise", _DP), ("wsum_pdf_class", _DP), ("wsum_pdf_direction", _DP),
        ("wsum_prior_offsetx_class", _DP), ("wsum_prior_offsety_class", _DP), ("wsum_sigma2_offset", _DP),
        ("wsum_sumw_group", _DP),
        ("diff2", _DP * 2), ("weight", _DP * 2), ("Mcoarse_significant", _CP), ("post_class_psi", _DP),
    ]


class RomeMap3dPool(C.Structure):
    _fields_ = [
        ("nr_images", C.c_int), ("ori_size", C.c_int), ("current_size", C.c_int), ("coarse_size", C.c_int),
        ("nr_classes", C.c_int), ("iclass_min", C.c_int), ("iclass_max", C.c_int), ("nr_groups", C.c_int),
        ("adaptive_oversampling", C.c_int), ("nr_dir", C.c_int), ("nr_psi", C.c_int), ("nr_trans", C.c_int),
        ("angles", _DP * 2), ("over_trans_x", _DP * 2), ("over_trans_y", _DP * 2),
        ("trans_x", _DP), ("trans_y", _DP),
        ("Fimg_real", _DP), ("Fimg_imag", _DP), ("Fimg_nomask_real", _DP), ("Fimg_nomask_imag", _DP),
        ("Fctf", _DP), ("highres_Xi2", _DP), ("old_offsetx", _DP), ("old_offsety", _DP), ("group", _IP),
        ("sigma2_noise", _DP), ("Mresol_fine", _IP), ("Mresol_coarse", _IP),
        ("pdf_class", _DP), ("pdf_direction", _DP), ("prior_offsetx_class", _DP), ("prior_offsety_class", _DP),
        ("sigma2_offset", C.c_double), ("sigma2_fudge", C.c_double), ("adaptive_fraction", C.c_double),
        ("do_ctf_correction", C.c_int), ("refs_are_ctf_corrected", C.c_int), ("do_map", C.c_int),
        ("do_scale_correction", C.c_int), ("do_cross_correlation", C.c_int), ("inputs_on_device", C.c_int),
        ("proposals", _IP), ("nr_proposals", C.c_int),
        ("scale_correction", _DP), ("data_vs_prior_class", _DP),
    ]


class RomeMap3dPoolOut(C.Structure):
    _fields_ = [
        ("min_diff2", _DP), ("sum_weight", _DP), ("significant_weight", _DP), ("wsum_norm_correction", _DP),
        ("pmax", _DP), ("cls", _IP), ("rot", _DP), ("tilt", _DP), ("psi", _DP), ("xoff", _DP), ("yoff", _DP),
        ("nr_sign", _DP),
        ("wsum_sigma2_noise", _DP), ("wsum_pdf_class", _DP), ("wsum_pdf_direction", _DP), ("wsum_sigma2_offset", _DP),
        ("wsum_sumw_group", _DP),
        ("pass_min_diff2", _DP * 2), ("pass_sum_weight", _DP * 2), ("pass_significant_weight", _DP * 2),
        ("coarse_diff2", _DP), ("Mcoarse_significant", _CP),
        ("fine_capacity", C.c_long), ("fine_count", _IP), ("fine_index", C.POINTER(C.c_long)),
        ("fine_diff2", _DP), ("fine_weight", _DP), ("post_coarse", _DP),
        ("wsum_scale_correction_XA", _DP), ("wsum_scale_correction_AA", _DP),
    ]


class RomeProposalSpec(C.Structure):
    _fields_ = [("n_r", C.c_int), ("n_theta", C.c_int), ("channels", C.c_int * 2), ("n_classes", C.c_int),
                ("r_lo", C.c_double), ("r_hi", C.c_double)]


class RomeReconIn(C.Structure):
    _fields_ = [("iclass", C.c_int), ("gridding_nr_iter", C.c_int), ("do_map", C.c_int), ("minres_map", C.c_int),
                ("tau2_fudge", C.c_double), ("normalise", C.c_double), ("tau2_in", _DP)]


class RomeReconOut(C.Structure):
    _fields_ = [("vol", _DP), ("tau2", _DP), ("sigma2", _DP), ("data_vs_prior", _DP)]


class RomePrepIn(C.Structure):
    _fields_ = [("nr_images", C.c_int), ("ori_size", C.c_int), ("current_size", C.c_int), ("nr_groups", C.c_int),
                ("first_image", C.c_int), ("images", C.c_void_p), ("image_type", C.c_int),
                ("images_on_device", C.c_int), ("norm", _DP), ("xoff", _DP), ("yoff", _DP),
                ("ctf_defocus_u", _DP), ("ctf_defocus_v", _DP), ("ctf_defocus_angle", _DP), ("ctf_voltage", _DP),
                ("ctf_cs", _DP), ("ctf_q0", _DP), ("ctf_bfac", _DP), ("group", _IP), ("sigma2_noise", _DP),
                ("avg_norm_correction", C.c_double), ("pixel_size", C.c_double), ("particle_diameter", C.c_double),
                ("sigma2_fudge", C.c_double), ("width_mask_edge", C.c_int), ("random_seed", C.c_int),
                ("do_norm_correction", C.c_int), ("do_zero_mask", C.c_int), ("do_ctf_correction", C.c_int),
                ("ctf_phase_flipped", C.c_int), ("only_flip_phases", C.c_int), ("intact_ctf_first_peak", C.c_int)]


class RomePrepOut(C.Structure):
    _fields_ = [("Fimg_real", _DP), ("Fimg_imag", _DP), ("Fimg_nomask_real", _DP), ("Fimg_nomask_imag", _DP),
                ("Fctf", _DP), ("outputs_on_device", C.c_int), ("highres_Xi2", _DP), ("old_offsetx", _DP),
                ("old_offsety", _DP), ("power_imgs", _DP)]


def _need(a: np.ndarray, dtype) -> None:
    """An array handed to the library as a raw pointer: the element type and
    C-contiguous layout the C side reads."""
    if a.dtype != dtype or not a.flags.c_contiguous:
        raise TypeError(f"expected a C-contiguous {np.dtype(dtype).name} array, got {a.dtype} "
                        f"(C-contiguous: {a.flags.c_contiguous})")


def dptr(a: Optional[np.ndarray]):
    if a is None:
        return _DP()
    _need(a, np.float64)
    return a.ctypes.data_as(_DP)


def iptr(a: Optional[np.ndarray]):
    if a is None:
        return _IP()
    _need(a, np.int32)
    return a.ctypes.data_as(_IP)


def cptr(a: Optional[np.ndarray]):
    if a is None:
        return _CP()
    _need(a, np.int8)
    return a.ctypes.data_as(_CP)


#: every symbol include/rome_gpu.h declares (checked by the CPU tests)
EXPORTED_SYMBOLS = [
    "rome_gpu_create", "rome_gpu_destroy", "rome_gpu_last_error", "rome_gpu_set_precision",
    "rome_gpu_abi_version", "rome_gpu_set_projectors", "rome_gpu_get_backprojector",
    "rome_gpu_set_backprojector", "rome_gpu_map2d_estep_pool", "rome_gpu_select_significant",
    "rome_gpu_select_significant_static", "rome_gpu_map3d_estep_pool",
    "rome_gpu_proposal_create", "rome_gpu_proposal_destroy", "rome_gpu_proposal_num_params",
    "rome_gpu_proposal_get_params", "rome_gpu_proposal_set_params", "rome_gpu_proposal_features",
    "rome_gpu_proposal_loss_grad", "rome_gpu_proposal_train", "rome_gpu_proposal_predict",
    "rome_gpu_proposal_propose",
    "rome_gpu_reconstruct", "rome_gpu_get_timings", "rome_gpu_reset_timings", "rome_gpu_copy_from_host",
    "rome_gpu_add_backprojectors", "rome_gpu_prepare_particles", "rome_gpu_backproject_images",
    "rome_gpu_tuning_report", "rome_gpu_wait_selftest", "rome_gpu_backprojector_size",
    "rome_gpu_backprojector_device_copy", "rome_gpu_invalidate_projections",
]

_LIB = None


def tuning_report() -> list:
    """The tensor-core autotuner's choices, one dict per key."""
    lib = load_library()
    n = lib.rome_gpu_tuning_report(None, 0)
    buf = C.create_string_buffer(n + 1)
    lib.rome_gpu_tuning_report(buf, n + 1)
    out = []
    for line in buf.value.decode().splitlines():
        f = line.split()
        d = {"kind": f[0]}
        for kv in f[1:]:
            k, v = kv.split("=", 1) if "=" in kv else kv.split(":", 1)
            d[k] = v
        out.append(d)
    return out


def library_path() -> str:
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "librome_b200.so")


def load_library():
    """Open librome_b200.so (in-tree).  Raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m rome_b200.build` (no CPU fallback exists)")
    lib = C.CDLL(path)
    lib.rome_gpu_abi_version.restype = C.c_int
    if lib.rome_gpu_abi_version() != ABI_VERSION:
        raise RuntimeError(f"{path} has ABI version {lib.rome_gpu_abi_version()}, this binding expects {ABI_VERSION}: "
                           "rebuild it with `python -m rome_b200.build`")
    lib.rome_gpu_create.argtypes = [C.c_int, C.POINTER(RomeGpuConfig), C.POINTER(C.c_void_p)]
    lib.rome_gpu_destroy.argtypes = [C.c_void_p]
    lib.rome_gpu_last_error.argtypes = [C.c_void_p]
    lib.rome_gpu_last_error.restype = C.c_char_p
    lib.rome_gpu_set_precision.argtypes = [C.c_void_p, C.c_int]
    lib.rome_gpu_set_projectors.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _DP]
    lib.rome_gpu_get_backprojector.argtypes = [C.c_void_p, C.c_int, _DP, _DP]
    lib.rome_gpu_set_backprojector.argtypes = [C.c_void_p, C.c_int, _DP, _DP]
    lib.rome_gpu_map2d_estep_pool.argtypes = [C.c_void_p, C.POINTER(RomeMap2dPool), C.POINTER(RomeMap2dPoolOut)]
    lib.rome_gpu_map3d_estep_pool.argtypes = [C.c_void_p, C.POINTER(RomeMap3dPool), C.POINTER(RomeMap3dPoolOut)]
    _FP = C.POINTER(C.c_float)
    lib.rome_gpu_proposal_create.argtypes = [C.c_void_p, C.POINTER(RomeProposalSpec), C.c_ulonglong,
                                             C.POINTER(C.c_void_p)]
    lib.rome_gpu_proposal_destroy.argtypes = [C.c_void_p]
    lib.rome_gpu_proposal_destroy.restype = None
    lib.rome_gpu_proposal_num_params.argtypes = [C.c_void_p]
    lib.rome_gpu_proposal_num_params.restype = C.c_long
    lib.rome_gpu_proposal_get_params.argtypes = [C.c_void_p, _FP]
    lib.rome_gpu_proposal_set_params.argtypes = [C.c_void_p, _FP]
    lib.rome_gpu_proposal_features.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                               C.c_int, _FP]
    lib.rome_gpu_proposal_loss_grad.argtypes = [C.c_void_p, C.c_int, _FP, _FP, _DP, _FP, _FP]
    lib.rome_gpu_proposal_train.argtypes = [C.c_void_p, C.c_int, _FP, _FP, C.c_int, C.c_int, C.c_float,
                                            C.c_ulonglong, _DP]
    lib.rome_gpu_proposal_predict.argtypes = [C.c_void_p, C.c_int, _FP, C.c_int, _IP, _FP]
    lib.rome_gpu_proposal_propose.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                              C.c_int, C.c_int, _IP, _FP]
    lib.rome_gpu_select_significant.argtypes = [C.c_void_p, C.c_int, C.c_long, _DP, _DP, C.c_double, _DP, _DP]
    lib.rome_gpu_copy_from_host.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]
    lib.rome_gpu_add_backprojectors.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    lib.rome_gpu_backproject_images.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                                C.c_void_p, _DP, C.c_int]
    lib.rome_gpu_select_significant_static.argtypes = [C.c_void_p, C.c_int, C.c_long, _DP, _DP, C.c_double, _DP,
                                                       _DP]
    lib.rome_gpu_reconstruct.argtypes = [C.c_void_p, C.POINTER(RomeReconIn), C.POINTER(RomeReconOut)]
    lib.rome_gpu_prepare_particles.argtypes = [C.c_void_p, C.POINTER(RomePrepIn), C.POINTER(RomePrepOut)]
    lib.rome_gpu_get_timings.argtypes = [C.c_void_p, C.POINTER(RomeGpuTimings)]
    lib.rome_gpu_reset_timings.argtypes = [C.c_void_p]
    lib.rome_gpu_wait_selftest.argtypes = [C.c_void_p, C.c_double, _DP]
    lib.rome_gpu_invalidate_projections.argtypes = [C.c_void_p]
    lib.rome_gpu_backprojector_size.argtypes = [C.c_void_p, C.POINTER(C.c_size_t)]
    lib.rome_gpu_backprojector_device_copy.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    lib.rome_gpu_tuning_report.argtypes = [C.c_char_p, C.c_size_t]
    lib.rome_gpu_tuning_report.restype = C.c_size_t
    _LIB = lib
    return lib
