"""Tensor-core (tcgen05) precisions of the diff2 cross term.

BF16X3 (split hi/lo products, FP32 accumulation in TMEM) must stay within
the plain-FP32 tolerance of the oracle: diff2 relative error <= 1e-5 and
identical poses except near ties.  Plain BF16 is the fast mode; its diff2
error is bounded by 5e-3 relative here and its pose agreement with the
FP64 oracle must be >= 99% of particles (near ties excepted), the agreement
bar of the learned/BF16 mode.
"""
import numpy as np
import pytest

from rome_b200.map2d import GpuContext
from rome_b200.workload import Map2dWorkload, build_map2d
from tests.util import relerr

pytestmark = pytest.mark.gpu

WL = {
    # partial M and N tiles (M = 40*29 rows, N = 3*72 orientations)
    "cfg2_shape": Map2dWorkload(n_particles=40, ori_size=128, n_classes=3, n_blobs=40, psi_step=5, offset_range=6,
                                offset_step=2, max_shift=6, pixel=1.5, snr=0.03, seed=31),
    "cfg1_shape": Map2dWorkload(n_particles=64, ori_size=64, n_classes=5, n_blobs=20, psi_step=10, offset_range=5,
                                offset_step=1, max_shift=4, pixel=2.0, snr=0.05, seed=32),
}
TOL = {"bf16x3": 1e-5, "bf16": 5e-3}


def poses_agree(o, r):
    same = (o["cls"] == r["cls"]) & (o["psi"] == r["psi"]) & (o["xoff"] == r["xoff"]) & (o["yoff"] == r["yoff"])
    near = np.zeros_like(same)
    for i in np.nonzero(~same)[0]:
        top = np.sort(r["weight_0"][i])[::-1][:2]
        near[i] = top[1] >= top[0] * 0.5
    return float(np.mean(same | near)), float(np.mean(same))


@pytest.mark.parametrize("name", list(WL))
@pytest.mark.parametrize("prec", ["bf16x3", "bf16"])
def test_tensor_core_modes(name, prec):
    from oracle import oracle_py
    p, proj, r_max, truth = build_map2d(WL[name])
    r, bpd, bpw = oracle_py.map2d_estep_pool(p, proj, r_max, checkpoints=True)
    with GpuContext(0, prec) as ctx:
        ctx.set_projectors(proj, p.ori_size, r_max)
        o = ctx.map2d_estep_pool(p, checkpoints=True)
    ok = r["diff2_0"] > -1e9
    assert np.array_equal(ok, o["diff2_0"] > -1e9)
    rel = np.abs(o["diff2_0"][ok] - r["diff2_0"][ok]) / np.abs(r["diff2_0"][ok])
    print(f"{name} {prec}: diff2 max rel err {rel.max():.3e} mean {rel.mean():.3e}")
    assert rel.max() <= TOL[prec]
    agree, exact = poses_agree(o, r)
    print(f"{name} {prec}: pose agreement {agree:.3f} (exact {exact:.3f})")
    assert agree >= 0.99
    if prec == "bf16x3":
        assert relerr(o["wsum_pdf_class"], r["wsum_pdf_class"]) < 1e-3


def test_tensor_core_matches_fp32_path():
    """BF16X3 and FP32 GPU paths agree with each other to the FP32 tolerance."""
    p, proj, r_max, _ = build_map2d(WL["cfg1_shape"])
    outs = {}
    for prec in ["fp32", "bf16x3"]:
        with GpuContext(0, prec) as ctx:
            ctx.set_projectors(proj, p.ori_size, r_max)
            outs[prec] = ctx.map2d_estep_pool(p, checkpoints=True)
    a, b = outs["fp32"]["diff2_0"], outs["bf16x3"]["diff2_0"]
    ok = a > -1e9
    assert np.max(np.abs(a[ok] - b[ok]) / np.abs(a[ok])) < 1e-5
