"""GPU MAP2D E-step parity (CUDA path through the C ABI).

Checked against (a) the reference's own outputs recorded in tests/golden
and (b) the C oracle on seeded synthetic pools.  Tolerances of the plain
FP32 mode: diff2 relative error <= 1e-5 per hypothesis; identical best
class / psi / offset except where the reference's own top two weights are
within 1e-3 of each other (a near tie that FP32 rounding may flip);
FP64-accumulated sums within 1e-3 relative (they inherit the FP32 diff2
error through exp(-diff2)).
"""
import numpy as np
import pytest

from rome_b200.map2d import GpuContext
from rome_b200.workload import Map2dWorkload, build_map2d
from tests.util import golden_pool, relerr

pytestmark = pytest.mark.gpu

CASES = ["map2d_a", "map2d_b", "map2d_c"]
DIFF2_TOL = 1e-5
SUM_TOL = 1e-3


@pytest.fixture(scope="module")
def ctx():
    c = GpuContext(0, "fp32")
    yield c
    c.close()


def run_gpu(ctx, p, proj, r_max, checkpoints=True):
    ctx.set_projectors(proj, p.ori_size, r_max)
    o = ctx.map2d_estep_pool(p, checkpoints=checkpoints)
    bp = [ctx.get_backprojector(k) for k in range(p.nr_classes)]
    o["bp_data"] = np.stack([b[0] for b in bp])
    o["bp_weight"] = np.stack([b[1] for b in bp])
    return o


def check_diff2(gpu_d2, ref_d2):
    ref_ok = ref_d2 > -1e9
    gpu_ok = gpu_d2 > -1e9
    assert np.array_equal(ref_ok, gpu_ok), "different hypotheses computed"
    rel = np.abs(gpu_d2[ref_ok] - ref_d2[ref_ok]) / np.maximum(np.abs(ref_d2[ref_ok]), 1e-30)
    assert rel.max() <= DIFF2_TOL, rel.max()
    return rel.max()


def check_poses(o, ref_cls, ref_psi, ref_x, ref_y, ref_w):
    same = (o["cls"] == ref_cls) & (o["psi"] == ref_psi) & (o["xoff"] == ref_x) & (o["yoff"] == ref_y)
    for i in np.nonzero(~same)[0]:
        top = np.sort(ref_w[i])[::-1][:2]
        assert top[1] >= top[0] * (1 - 1e-3), f"particle {i}: pose differs without a near tie"
    return same.mean()


@pytest.mark.parametrize("case", CASES)
def test_gpu_matches_reference_golden(ctx, golden, case):
    g = golden[case]
    p, proj, r_max = golden_pool(g)
    o = run_gpu(ctx, p, proj, r_max)
    for ip in range(p.npass()):
        check_diff2(o[f"diff2_{ip}"], g[f"pool0_pass{ip}_diff2"])
        wref = g[f"pool0_pass{ip}_weight"]
        assert relerr(o[f"weight_{ip}"], wref) < SUM_TOL
    last = f"pool0_pass{p.npass() - 1}_"
    assert relerr(o["min_diff2"], g[last + "min_diff2"]) < DIFF2_TOL
    assert relerr(o["sum_weight"], g[last + "sum_weight"]) < SUM_TOL
    frac = check_poses(o, g[last + "class"], g[last + "psi"], g[last + "xoff"], g[last + "yoff"], g[last + "weight"])
    assert frac >= 0.9
    assert relerr(o["significant_weight"], g[last + "significant_weight"]) < SUM_TOL
    if p.npass() > 1:
        # coarse significance decides which fine hypotheses are evaluated
        agree = (o["Mcoarse_significant"] == g["pool0_pass0_Mcoarse_significant"]).mean()
        assert agree >= 0.999
    assert relerr(o["wsum_norm_correction"], g["pool0_wsum_norm_correction"]) < SUM_TOL
    for k in ["wsum_sigma2_noise", "wsum_pdf_class", "wsum_pdf_direction", "wsum_prior_offsetx_class",
              "wsum_prior_offsety_class", "wsum_sigma2_offset", "wsum_sumw_group"]:
        assert relerr(o[k], g["pool0_after_update_" + k]) < SUM_TOL, k
    assert relerr(o["bp_data"], g["pool0_after_bp_bp_data"]) < SUM_TOL
    assert relerr(o["bp_weight"], g["pool0_after_bp_bp_weight"]) < SUM_TOL


WORKLOADS = {
    "small32": Map2dWorkload(n_particles=24, ori_size=32, n_classes=3, n_blobs=8, blob_sigma=(1.5, 3.0), psi_step=15,
                             offset_range=3, offset_step=1, max_shift=2, pixel=4.0, snr=0.1, seed=11),
    "cfg1_shape": Map2dWorkload(n_particles=40, ori_size=64, n_classes=4, n_blobs=20, psi_step=10, offset_range=5,
                                offset_step=1, max_shift=4, pixel=2.0, snr=0.05, seed=12, random_perturbation=0.3),
    "cfg2_shape": Map2dWorkload(n_particles=8, ori_size=128, n_classes=3, n_blobs=40, psi_step=5, offset_range=6,
                                offset_step=2, max_shift=6, pixel=1.5, snr=0.03, seed=13),
}


@pytest.mark.parametrize("name", list(WORKLOADS))
def test_gpu_matches_oracle_seeded(ctx, name):
    from oracle import oracle_py
    p, proj, r_max, truth = build_map2d(WORKLOADS[name])
    o = run_gpu(ctx, p, proj, r_max)
    r, bpd, bpw = oracle_py.map2d_estep_pool(p, proj, r_max, checkpoints=True)
    assert r["status"] == 0
    check_diff2(o["diff2_0"], r["diff2_0"])
    frac = check_poses(o, r["cls"], r["psi"], r["xoff"], r["yoff"], r["weight_0"])
    assert frac >= 0.95
    assert relerr(o["sum_weight"], r["sum_weight"]) < SUM_TOL
    for k in ["wsum_sigma2_noise", "wsum_pdf_class", "wsum_sumw_group", "wsum_sigma2_offset"]:
        assert relerr(o[k], r[k]) < SUM_TOL, k
    assert relerr(o["bp_data"], bpd) < SUM_TOL
    assert relerr(o["bp_weight"], bpw) < SUM_TOL


def test_gpu_accumulates_over_pools(ctx):
    """Two pools in a row add into the same backprojector and wsums (the
    reference accumulates across expectationSomeParticles calls)."""
    from rome_b200.workload import subset
    p, proj, r_max, _ = build_map2d(WORKLOADS["small32"])
    ctx.set_projectors(proj, p.ori_size, r_max)
    a = ctx.map2d_estep_pool(subset(p, 0, 12))
    b = ctx.map2d_estep_pool(subset(p, 12, 24))
    two = np.stack([ctx.get_backprojector(k)[1] for k in range(p.nr_classes)])
    ctx.set_projectors(proj, p.ori_size, r_max)
    c = ctx.map2d_estep_pool(p)
    one = np.stack([ctx.get_backprojector(k)[1] for k in range(p.nr_classes)])
    assert relerr(two, one) < 1e-12
    assert relerr(a["wsum_pdf_class"] + b["wsum_pdf_class"], c["wsum_pdf_class"]) < 1e-12


def test_gpu_rejects_bad_input(ctx):
    p, proj, r_max, _ = build_map2d(WORKLOADS["small32"])
    ctx.set_projectors(proj, p.ori_size, r_max)
    import dataclasses
    bad = dataclasses.replace(p, current_size=p.current_size + 1)
    with pytest.raises(Exception):
        ctx.map2d_estep_pool(bad)
