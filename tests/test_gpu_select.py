"""Significance selection on the GPU is bit-exact with the reference's
sort-and-walk (findAllSignificantPoints, src/map2d_optimizer.cpp:1226-1311)
for identical FP64 weights and sums, including the paths where the
candidate set overflows shared memory."""
import numpy as np
import pytest

from rome_b200.map2d import GpuContext

pytestmark = pytest.mark.gpu


def rows(seed):
    rng = np.random.default_rng(seed)
    out = []
    # peaked posterior (typical)
    d = rng.exponential(30.0, 4000)
    out.append(np.exp(-(d - d.min())) * 0.01)
    # flat posterior: every weight needed (fallback path, > 8192 candidates)
    out.append(rng.uniform(0.9, 1.0, 20000) * 1e-3)
    # many exact duplicates and zeros
    w = np.zeros(5000)
    w[rng.integers(0, 5000, 3000)] = 0.125
    w[:10] = 0.5
    out.append(w)
    # a single positive weight
    w = np.zeros(777)
    w[500] = 3.0
    out.append(w)
    # weights spanning many binades
    out.append(np.exp(-rng.uniform(0, 600, 10000)))
    # tiny subnormal-ish values with one dominant
    w = np.full(300, 1e-310)
    w[7] = 1e-300
    out.append(w)
    return out


def test_select_bit_exact():
    from oracle import oracle_py
    with GpuContext(0) as ctx:
        for seed in range(3):
            for w in rows(seed):
                W = np.ascontiguousarray(w[None, :])
                s = np.array([w.sum()])
                for frac in (0.999, 0.5, 1.0):
                    sw, ns = ctx.select_significant(W, s, frac)
                    rw, rn = oracle_py.select_significant(w, s[0], frac)
                    assert sw[0] == rw and ns[0] == rn, (seed, frac, sw[0], rw, ns[0], rn)


def test_select_many_rows():
    from oracle import oracle_py
    rng = np.random.default_rng(5)
    W = np.exp(-rng.exponential(20.0, (64, 3000)))
    s = W.sum(axis=1)
    with GpuContext(0) as ctx:
        sw, ns = ctx.select_significant(W, s, 0.999)
    for i in range(W.shape[0]):
        rw, rn = oracle_py.select_significant(W[i], s[i], 0.999)
        assert sw[i] == rw and ns[i] == rn
