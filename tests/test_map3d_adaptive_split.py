"""Host logic of map3d_estep_pools_adaptive (no GPU): a pool whose fine pass
the library refuses with ROME_ERR_OOM ("fine pass ... use smaller pools") is
split in halves, recursively, and the halves' results are joined --
per-particle outputs concatenated in particle order, model sums added.  The
library call is replaced by a fake that refuses pools above a size."""
import dataclasses

import numpy as np
import pytest

from rome_b200 import abi, map3d
from rome_b200.map2d import RomeError


def fake_pool(P, seed=0):
    rng = np.random.default_rng(seed)
    F = 6
    z = lambda *s: rng.standard_normal(s)  # noqa: E731
    return map3d.Map3dPool(
        ori_size=4, current_size=4, coarse_size=4, nr_classes=2, nr_groups=3, nr_dir=5,
        angles=[np.zeros((5, 2, 1, 3)), np.zeros((5, 2, 8, 3))],
        over_trans_x=[np.zeros((3, 1)), np.zeros((3, 4))], over_trans_y=[np.zeros((3, 1)), np.zeros((3, 4))],
        trans_x=np.zeros(3), trans_y=np.zeros(3),
        Fimg_real=z(P, F), Fimg_imag=z(P, F), Fimg_nomask_real=z(P, F), Fimg_nomask_imag=z(P, F),
        Fctf=z(P, F), highres_Xi2=z(P), old_offsetx=z(P), old_offsety=z(P), group=np.arange(P) % 3,
        sigma2_noise=np.ones((3, 3)), Mresol_fine=np.zeros(F, np.int32), Mresol_coarse=np.zeros(F, np.int32),
        pdf_class=np.ones(2), pdf_direction=np.ones((2, 5)), prior_offsetx_class=np.zeros(2),
        prior_offsety_class=np.zeros(2), sigma2_offset=1.0)


def test_split_joins_halves_in_order(monkeypatch):
    calls = []

    def fake(ctx, p, dev=None):
        calls.append(p.nr_images)
        if p.nr_images > 3:
            raise RomeError(abi.ROME_ERR_OOM, "fine pass: 9 significant coarse orientations need 1.0 GB of "
                                              "projections (0.5 GB free); use smaller pools")
        out = {k: p.highres_Xi2.copy() for k in ("min_diff2", "sum_weight", "rot")}
        out["cls"] = (p.old_offsetx > 0).astype(np.int32)
        out["wsum_scale_correction_XA"] = np.tile(p.highres_Xi2[:, None], (1, 3))
        out["wsum_sigma2_noise"] = np.full((3, 3), float(p.nr_images))
        out["wsum_pdf_class"] = np.array([1.0, 2.0])
        return out

    monkeypatch.setattr(map3d, "map3d_estep_pool", fake)
    p = fake_pool(10)
    o = map3d.map3d_estep_pools_adaptive(None, p)
    assert calls[0] == 10 and max(calls[1:]) <= 5 and sum(c for c in calls if c <= 3) == 10
    np.testing.assert_array_equal(o["min_diff2"], p.highres_Xi2)
    np.testing.assert_array_equal(o["cls"], (p.old_offsetx > 0).astype(np.int32))
    np.testing.assert_array_equal(o["wsum_scale_correction_XA"][:, 0], p.highres_Xi2)
    # model sums: every leaf call added once
    leaves = [c for c in calls if c <= 3]
    np.testing.assert_array_equal(o["wsum_sigma2_noise"], np.full((3, 3), float(sum(leaves))))
    np.testing.assert_array_equal(o["wsum_pdf_class"], np.array([1.0, 2.0]) * len(leaves))


def test_other_errors_are_not_split(monkeypatch):
    def fake(ctx, p, dev=None):
        raise RomeError(abi.ROME_ERR_NUMERIC, "exp_sum_weight[0] == 0")

    monkeypatch.setattr(map3d, "map3d_estep_pool", fake)
    with pytest.raises(RomeError):
        map3d.map3d_estep_pools_adaptive(None, fake_pool(4))


def test_single_particle_pool_is_not_split(monkeypatch):
    def fake(ctx, p, dev=None):
        raise RomeError(abi.ROME_ERR_OOM, "fine pass: 1 significant coarse orientations need 900 GB")

    monkeypatch.setattr(map3d, "map3d_estep_pool", fake)
    with pytest.raises(RomeError):
        map3d.map3d_estep_pools_adaptive(None, fake_pool(1))
    q = dataclasses.replace(fake_pool(4))
    with pytest.raises(RomeError):
        map3d.map3d_estep_pools_adaptive(None, q, min_pool=4)
