"""ctypes wrapper of the C oracle (oracle/estep_oracle.c).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and
the CPU-baseline leg of bench.py, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from rome_b200 import abi
from rome_b200.map2d import Map2dPool, alloc_outputs, pack_pool

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "_ref", "librome_oracle.so")
        if not os.path.exists(path):
            # the C restatement needs only gcc (not the reference tree)
            import subprocess
            subprocess.check_call(["make", "-C", _HERE, "_ref/librome_oracle.so"], stdout=subprocess.DEVNULL)
        L = C.CDLL(path)
        DP = C.POINTER(C.c_double)
        L.oracle_map2d_estep_pool.argtypes = [C.POINTER(abi.RomeMap2dPool), C.POINTER(abi.RomeMap2dPoolOut), C.c_int,
                                              C.c_int, C.c_int, DP, DP, DP]
        L.oracle_shift_image.argtypes = [DP, DP, DP, DP, C.c_int, C.c_double, C.c_double, C.c_int]
        L.oracle_rotate2d.argtypes = [DP, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, DP, DP]
        L.oracle_backrotate2d.argtypes = [DP, DP, DP, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, DP, DP]
        L.oracle_select_significant.argtypes = [C.c_long, DP, C.c_double, C.c_double, DP, DP]
        L.oracle_euler_matrix.argtypes = [C.c_double, C.c_double, C.c_double, DP]
        _LIB = L
    return _LIB


def map2d_estep_pool(p: Map2dPool, proj_data: np.ndarray, r_max: int, padding_factor: int = 2,
                     checkpoints: bool = False):
    """Oracle E-step of one pool; returns (outputs dict, bp_data, bp_weight)."""
    proj = np.ascontiguousarray(proj_data, dtype=np.float64)
    K, pad = proj.shape[0], proj.shape[1]
    s, keep = pack_pool(p)
    so, o = alloc_outputs(p, checkpoints)
    bp_data = np.zeros_like(proj)
    bp_weight = np.zeros(proj.shape[:-1], np.float64)
    rc = lib().oracle_map2d_estep_pool(C.byref(s), C.byref(so), pad, r_max, padding_factor, abi.dptr(proj),
                                       abi.dptr(bp_data), abi.dptr(bp_weight))
    o["status"] = rc
    return o, bp_data, bp_weight


def shift_image(fr, fi, size, sx, sy, ori_size):
    fr = np.ascontiguousarray(fr, np.float64)
    fi = np.ascontiguousarray(fi, np.float64)
    outr, outi = np.zeros_like(fr), np.zeros_like(fi)
    lib().oracle_shift_image(abi.dptr(fr), abi.dptr(fi), abi.dptr(outr), abi.dptr(outi), size, sx, sy, ori_size)
    return outr, outi


def select_significant(weights, sum_weight, adaptive_fraction):
    w = np.ascontiguousarray(weights, np.float64)
    sw, ns = C.c_double(), C.c_double()
    lib().oracle_select_significant(w.size, abi.dptr(w), float(sum_weight), adaptive_fraction, C.byref(sw),
                                    C.byref(ns))
    return sw.value, ns.value


def euler_matrix(rot, tilt, psi):
    A = np.zeros(9)
    lib().oracle_euler_matrix(rot, tilt, psi, abi.dptr(A))
    return A.reshape(3, 3)
