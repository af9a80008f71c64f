"""GPU MAP3D E-step and 3D M-step parity (CUDA path through the C ABI)
against the reference's own outputs recorded in tests/golden/map3d_a.npz
(oracle/_ref/map3d_dump driving Map3dOptimizer_old, HEALPix order 1,
oversampling 1, +-2 px translations, CTF on, iteration 2).

Tolerances of the plain FP32 mode: diff2 relative error <= 1e-5 per
hypothesis in both passes; exactly the reference's hypothesis lists (same
coarse hypotheses computed, same fine lists for every particle whose
coarse significance agrees); FP64-accumulated sums, weights and model sums
within 1e-3 relative (they inherit the FP32 diff2 error through
exp(-diff2)); identical best class / rot / tilt / psi / offset except at a
near tie of the reference's top two weights.  M-step: FSC >= 0.999 at every
shell and <= 1e-6 relative RMS against the reference reconstruction.
"""
import numpy as np
import pytest

from rome_b200.map2d import GpuContext
from rome_b200.map3d import fine_lists_from_dump, map3d_estep_pool, pool3d_from_dump
from tests.test_gpu_reconstruct import fsc
from tests.util import relerr

pytestmark = pytest.mark.gpu

DIFF2_TOL = 1e-5
SUM_TOL = 1e-3


@pytest.fixture(scope="module")
def run3d(golden):
    g = golden["map3d_a"]
    p = pool3d_from_dump(g, 0)
    with GpuContext(0, "fp32") as ctx:
        ctx.set_projectors(g["projector_data"], p.ori_size, int(g["projector_r_max"][0]))
        o = map3d_estep_pool(ctx, p, checkpoints=True)
        bp = [ctx.get_backprojector(k) for k in range(p.nr_classes)]
    o["bp_data"] = np.stack([b[0] for b in bp])
    o["bp_weight"] = np.stack([b[1] for b in bp])
    return g, p, o


def coarse_ref(g, p):
    """Reference coarse lists as a dense [P][ncoarse] array (INT_MIN where not listed)."""
    out = np.full((p.nr_images, p.ncoarse), float(np.iinfo(np.int32).min))
    lists = fine_lists_from_dump(g, "pool0_pass0_diff2_", p.nr_trans, nh=1)
    for i, (idx, v) in enumerate(lists):
        out[i, idx] = v
    return out


def test_coarse_pass_matches_reference(run3d):
    g, p, o = run3d
    ref = coarse_ref(g, p)
    ok = ref > -1e9
    assert np.array_equal(ok, o["coarse_diff2"] > -1e9), "different coarse hypotheses computed"
    rel = np.abs(o["coarse_diff2"][ok] - ref[ok]) / np.abs(ref[ok])
    assert rel.max() <= DIFF2_TOL, rel.max()
    assert relerr(o["pass_min_diff20"], g["pool0_pass0_min_diff2"]) < DIFF2_TOL
    assert relerr(o["pass_sum_weight0"], g["pool0_pass0_sum_weight"]) < SUM_TOL
    assert relerr(o["pass_significant_weight0"], g["pool0_pass0_significant_weight"]) < SUM_TOL
    agree = (o["Mcoarse_significant"] == g["pool0_pass0_Mcoarse_significant"]).mean()
    assert agree >= 0.999, agree
    nr = np.abs(o["nr_sign"] - g["pool0_pass0_nr_sign"]) / g["pool0_pass0_nr_sign"]
    assert nr.max() <= 0.01, nr.max()


def test_fine_pass_lists_match_reference(run3d):
    g, p, o = run3d
    d2 = fine_lists_from_dump(g, "pool0_pass1_diff2_", p.nr_trans)
    wt = fine_lists_from_dump(g, "pool0_pass1_weight_", p.nr_trans)
    mc_same = (o["Mcoarse_significant"] == g["pool0_pass0_Mcoarse_significant"]).all(axis=1)
    q = 0
    checked = 0
    for i in range(p.nr_images):
        n = int(o["fine_count"][i])
        idx, dv = o["fine_index"][q:q + n], o["fine_diff2"][q:q + n]
        w = o["fine_weight"][q:q + n]
        q += n
        if not mc_same[i]:
            continue
        ridx, rd = d2[i]
        assert np.array_equal(idx, ridx), f"particle {i}: fine list differs"
        rel = np.abs(dv - rd) / np.abs(rd)
        assert rel.max() <= DIFF2_TOL, (i, rel.max())
        assert relerr(w, wt[i][1]) < SUM_TOL, i
        checked += 1
    assert checked >= p.nr_images - 1


def test_fine_pass_results_match_reference(run3d):
    g, p, o = run3d
    last = "pool0_pass1_"
    assert relerr(o["min_diff2"], g[last + "min_diff2"]) < DIFF2_TOL
    assert relerr(o["sum_weight"], g[last + "sum_weight"]) < SUM_TOL
    assert relerr(o["significant_weight"], g[last + "significant_weight"]) < SUM_TOL
    assert relerr(o["pmax"], g[last + "pmax"]) < SUM_TOL
    same = ((o["cls"] == g[last + "class"]) & (o["rot"] == g[last + "rot"]) & (o["tilt"] == g[last + "tilt"])
            & (o["psi"] == g[last + "psi"]) & (o["xoff"] == g[last + "xoff"]) & (o["yoff"] == g[last + "yoff"]))
    wt = fine_lists_from_dump(g, last + "weight_", p.nr_trans)
    for i in np.nonzero(~same)[0]:
        top = np.sort(wt[i][1])[::-1][:2]
        assert top[1] >= top[0] * (1 - 1e-3), f"particle {i}: pose differs without a near tie"


def test_wsums_and_backprojection_match_reference(run3d):
    g, p, o = run3d
    assert relerr(o["wsum_norm_correction"], g["pool0_wsum_norm_correction"]) < SUM_TOL
    for k in ["wsum_sigma2_noise", "wsum_pdf_class", "wsum_pdf_direction", "wsum_sigma2_offset", "wsum_sumw_group"]:
        assert relerr(o[k], g["pool0_after_update_" + k]) < SUM_TOL, k
    assert relerr(o["bp_data"], g["pool0_after_bp_bp_data"]) < SUM_TOL
    assert relerr(o["bp_weight"], g["pool0_after_bp_bp_weight"]) < SUM_TOL


def test_tensor_core_coarse_pass_poses(golden):
    """BF16 / split-BF16 cross term in the coarse pass: same final poses."""
    g = golden["map3d_a"]
    p = pool3d_from_dump(g, 0)
    for prec in ("bf16x3", "bf16"):
        with GpuContext(0, prec) as ctx:
            ctx.set_projectors(g["projector_data"], p.ori_size, int(g["projector_r_max"][0]))
            o = map3d_estep_pool(ctx, p)
        same = (o["cls"] == g["pool0_pass1_class"]) & (o["rot"] == g["pool0_pass1_rot"]) & (
            o["tilt"] == g["pool0_pass1_tilt"]) & (o["psi"] == g["pool0_pass1_psi"])
        assert same.mean() >= 0.75, (prec, same.mean())
        assert relerr(o["sum_weight"], g["pool0_pass1_sum_weight"]) < 0.05


def test_reconstruct_3d_matches_reference(golden):
    g = golden["map3d_a"]
    ori = int(g["ori_size"][0])
    K = int(g["nr_classes"][0])
    with GpuContext(0) as ctx:
        ctx.set_projectors(g["projector_data"], ori, int(g["projector_r_max"][0]))
        for k in range(K):
            ctx.set_backprojector(k, g["iter_bp_data"][k], g["iter_bp_weight"][k])
            o = ctx.reconstruct(k, ori, 3, g["tau2_class_before"][k], float(g["tau2_fudge_factor"][0]),
                                float(g["iter_wsum_pdf_class"][k]), int(g["gridding_nr_iter"][0]),
                                bool(g["do_map"][0]), int(g["minres_map"][0]))
            ref = g["Irefs_after"][k]
            rms = np.sqrt(np.mean((o["vol"] - ref) ** 2)) / np.sqrt(np.mean(ref ** 2))
            f = fsc(o["vol"], ref)
            print(f"map3d_a class {k}: rel rms {rms:.2e}, min FSC {f.min():.6f}")
            assert f.min() >= 0.999
            assert rms <= 1e-6
            assert relerr(o["sigma2"], g["sigma2_class_after"][k]) <= 1e-9
            assert relerr(o["data_vs_prior"], g["data_vs_prior_after"][k]) <= 1e-9


def test_rejects_unsupported_modes(golden):
    import dataclasses  # noqa: F401
    from rome_b200 import abi
    g = golden["map3d_a"]
    p = pool3d_from_dump(g, 0)
    with GpuContext(0) as ctx:
        ctx.set_projectors(g["projector_data"], p.ori_size, int(g["projector_r_max"][0]))
        p.adaptive_oversampling = 0
        with pytest.raises(Exception) as e:
            map3d_estep_pool(ctx, p)
        assert getattr(e.value, "code", abi.ROME_ERR_UNSUPPORTED) == abi.ROME_ERR_UNSUPPORTED
