"""Pool plumbing on the GPU: a subset of a staged pool read through
particle_rows gives the outputs of the same particles copied into a pool of
their own; projections reused across pools (same model and sampling) give
the outputs of freshly computed ones, and set_projectors / a precision
change invalidate them."""
import numpy as np
import pytest

from rome_b200.map2d import GpuContext, take_pool
from rome_b200.workload import Map2dWorkload, build_map2d, subset
from tests.util import relerr

pytestmark = pytest.mark.gpu

KEYS = ("cls", "psi", "xoff", "yoff")


def _workload(seed):
    w = Map2dWorkload(n_particles=240, ori_size=48, n_classes=3, n_blobs=12, psi_step=15, offset_range=2,
                      offset_step=1, max_shift=2, pixel=2.5, snr=0.1, seed=seed)
    return build_map2d(w)


@pytest.mark.parametrize("prec", ["fp32", "bf16"])
def test_particle_rows_subset_equals_copied_subset(prec):
    p, proj, r_max, _ = _workload(3)
    idx = np.arange(1, p.nr_images, 3)
    with GpuContext(0, prec) as ctx:
        ctx.set_projectors(proj, p.ori_size, r_max)
        staged = ctx.stage_pool(p)
        a = ctx.map2d_estep_pool(take_pool(staged, idx))
        b = ctx.map2d_estep_pool(ctx.stage_pool(take_pool(p, idx)))
        rng = np.random.default_rng(0)
        J = p.nr_classes * p.nr_psi
        props = np.sort(np.stack([rng.choice(J, 12, replace=False) for _ in idx]), axis=1).astype(np.int32)
        c = ctx.map2d_estep_pool(take_pool(staged, idx), proposals=props)
        d = ctx.map2d_estep_pool(ctx.stage_pool(take_pool(p, idx)), proposals=props)
    for x, y in ((a, b), (c, d)):
        for k in KEYS:
            assert np.array_equal(x[k], y[k]), k
        for k in ("min_diff2", "sum_weight", "significant_weight", "wsum_norm_correction"):
            assert relerr(x[k], y[k]) == 0.0, k
        assert relerr(x["wsum_sigma2_noise"], y["wsum_sigma2_noise"]) <= 1e-12


def test_projection_reuse_across_pools():
    p, proj, r_max, _ = _workload(5)
    A, B = subset(p, 0, 120), subset(p, 120, 240)
    with GpuContext(0, "bf16") as ctx:
        ctx.set_projectors(proj, p.ori_size, r_max)
        ctx.map2d_estep_pool(A)
        ctx.reset_timings()
        reused = ctx.map2d_estep_pool(B)  # projections of A's call
        assert ctx.get_timings()["project"]["launches"] == 2  # rot_sig + jvalid only: no projection
        ctx.set_projectors(proj, p.ori_size, r_max)  # invalidates
        ctx.reset_timings()
        fresh = ctx.map2d_estep_pool(B)
        assert ctx.get_timings()["project"]["launches"] == 3
        ctx.set_precision("bf16x3")  # a new operand type: recomputed
        ctx.reset_timings()
        split = ctx.map2d_estep_pool(B)
        assert ctx.get_timings()["project"]["launches"] == 3
    for k in KEYS:
        assert np.array_equal(reused[k], fresh[k]), k
    assert relerr(reused["sum_weight"], fresh["sum_weight"]) == 0.0
    assert np.mean(split["cls"] == fresh["cls"]) >= 0.95
