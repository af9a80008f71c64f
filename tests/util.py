"""Shared helpers of the parity tests."""
import numpy as np

from rome_b200.map2d import pool_from_dump


def golden_pool(g):
    return pool_from_dump(g, 0), g["projector_data"], int(g["projector_r_max"][0])


def relerr(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(a - b))) / scale


def computed_mask(diff2):
    return np.asarray(diff2) > -1e9  # entries the reference left at INT_MIN were not computed
