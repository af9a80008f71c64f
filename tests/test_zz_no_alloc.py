"""rome_gpu_select_significant_static (no device allocation, fixed scratch
compiled into the library) returns exactly what rome_gpu_select_significant
returns, on two calls in a row, and refuses requests beyond its limits.

Named so that it is collected last: it must pass both in a fresh process and
after every other GPU test has used the same library."""
import ctypes as C

import numpy as np
import pytest

from rome_b200 import abi
from rome_b200.map2d import GpuContext

pytestmark = pytest.mark.gpu

MAX_IMAGES = 4096        # ROME_SELECT_STATIC_MAX_IMAGES
MAX_WEIGHTS = 1 << 20    # ROME_SELECT_STATIC_MAX_WEIGHTS


def _call(ctx, name, W, s, frac):
    W = np.ascontiguousarray(W, np.float64)
    s = np.ascontiguousarray(s, np.float64)
    n, ln = W.shape
    sw = np.full(n, -1.0)
    ns = np.full(n, -1.0)
    rc = getattr(ctx.lib, name)(ctx.h, n, ln, abi.dptr(W), abi.dptr(s), frac, abi.dptr(sw), abi.dptr(ns))
    return rc, sw, ns


def _batches():
    rng = np.random.default_rng(11)
    out = []
    # peaked posteriors, many rows
    W = np.exp(-rng.exponential(20.0, (300, 3000)))
    out.append(W)
    # flat rows: candidate sets overflow shared memory -> fallback sort slots
    out.append(rng.uniform(0.9, 1.0, (6, 20000)) * 1e-3)
    # mixed: zeros, duplicates, one dominant weight
    W = np.zeros((5, 5000))
    W[:, rng.integers(0, 5000, 3000)] = 0.125
    W[:, :10] = 0.5
    W[2] = 0.0
    W[2, 4321] = 2.0
    out.append(W)
    # a single row at the weight limit (one fallback slot of 2^20 doubles)
    out.append(rng.uniform(0.5, 1.0, (1, MAX_WEIGHTS)))
    return out


def test_static_matches_allocating_entry_point_twice():
    with GpuContext(0) as ctx:
        for W in _batches():
            s = W.sum(axis=1)
            for frac in (0.999, 0.5):
                rc, rw, rn = _call(ctx, "rome_gpu_select_significant", W, s, frac)
                assert rc == abi.ROME_OK, ctx.lib.rome_gpu_last_error(ctx.h)
                for _ in range(2):  # two calls in a row on the same static scratch
                    rc, sw, ns = _call(ctx, "rome_gpu_select_significant_static", W, s, frac)
                    assert rc == abi.ROME_OK, ctx.lib.rome_gpu_last_error(ctx.h)
                    # identical kernels on identical FP64 inputs: tolerance 0
                    np.testing.assert_array_equal(sw, rw)
                    np.testing.assert_array_equal(ns, rn)


def test_static_rejects_sizes_beyond_its_limits():
    with GpuContext(0) as ctx:
        W = np.ones((1, MAX_WEIGHTS + 1))
        rc, sw, ns = _call(ctx, "rome_gpu_select_significant_static", W, W.sum(axis=1), 0.999)
        assert rc == abi.ROME_ERR_ARG
        assert b"static limit" in ctx.lib.rome_gpu_last_error(ctx.h)
        assert (sw == -1.0).all() and (ns == -1.0).all()
        W = np.ones((MAX_IMAGES + 1, 2))
        rc, _, _ = _call(ctx, "rome_gpu_select_significant_static", W, W.sum(axis=1), 0.999)
        assert rc == abi.ROME_ERR_ARG
        # still usable after a refusal
        W = np.exp(-np.arange(50.0))[None, :]
        rc, rw, rn = _call(ctx, "rome_gpu_select_significant", W, W.sum(axis=1), 0.999)
        rc2, sw, ns = _call(ctx, "rome_gpu_select_significant_static", W, W.sum(axis=1), 0.999)
        assert rc == rc2 == abi.ROME_OK
        assert sw[0] == rw[0] and ns[0] == rn[0]
