"""GPU MAP3D E-step with intensity-scale correction (-scale) against the
reference's own outputs recorded in tests/golden/map3d_scale.npz
(oracle/_ref/map3d_dump, 24^2, K=2, HEALPix order 1, seven micrograph groups
whose scales iteration 1 moved away from 1).

With scale correction the reference multiplies every reference projection
by its particle's group scale (applyCtfToClass,
src/map3d_optimizer.cpp:1054-1066) and the back-projection's CTF by it
(:2274-2282), and updateModel adds w Re(Frefctf conj X) and w |Frefctf|^2
to per-particle XA/AA spectra over the shells whose data_vs_prior exceeds 3
(:1488-1502, binned in updateOtherParams :2090-2112).  Tolerances as in the
plain FP32 3D test: diff2 <= 1e-5 relative, FP64 sums within 1e-3
relative, identical poses except at a near tie; XA/AA within 1e-3 of the
largest value, and storeWeightedSums' division of them by the scale
(:1985-1995, done by the caller) reproduces the reference's group spectra.
"""
import numpy as np
import pytest

from rome_b200.map2d import GpuContext
from rome_b200.map3d import fine_lists_from_dump, map3d_estep_pool, pool3d_from_dump
from tests.util import relerr

pytestmark = pytest.mark.gpu

DIFF2_TOL = 1e-5
SUM_TOL = 1e-3


@pytest.fixture(scope="module")
def runscale(golden):
    g = golden["map3d_scale"]
    p = pool3d_from_dump(g, 0)
    assert p.do_scale_correction and np.abs(p.scale_correction - 1).max() > 0.01
    with GpuContext(0, "fp32") as ctx:
        ctx.set_projectors(g["projector_data"], p.ori_size, int(g["projector_r_max"][0]))
        o = map3d_estep_pool(ctx, p, checkpoints=True)
        bp = [ctx.get_backprojector(k) for k in range(p.nr_classes)]
    o["bp_data"] = np.stack([b[0] for b in bp])
    o["bp_weight"] = np.stack([b[1] for b in bp])
    return g, p, o


def test_coarse_pass_matches_reference(runscale):
    g, p, o = runscale
    ref = np.full((p.nr_images, p.ncoarse), float(np.iinfo(np.int32).min))
    for i, (idx, v) in enumerate(fine_lists_from_dump(g, "pool0_pass0_diff2_", p.nr_trans, nh=1)):
        ref[i, idx] = v
    ok = ref > -1e9
    assert np.array_equal(ok, o["coarse_diff2"] > -1e9)
    rel = np.abs(o["coarse_diff2"][ok] - ref[ok]) / np.abs(ref[ok])
    assert rel.max() <= DIFF2_TOL, rel.max()
    assert relerr(o["pass_sum_weight0"], g["pool0_pass0_sum_weight"]) < SUM_TOL
    assert (o["Mcoarse_significant"] == g["pool0_pass0_Mcoarse_significant"]).mean() >= 0.999


def test_fine_pass_and_poses_match_reference(runscale):
    g, p, o = runscale
    last = "pool0_pass1_"
    d2 = fine_lists_from_dump(g, last + "diff2_", p.nr_trans)
    mc_same = (o["Mcoarse_significant"] == g["pool0_pass0_Mcoarse_significant"]).all(axis=1)
    q = 0
    for i in range(p.nr_images):
        n = int(o["fine_count"][i])
        idx, dv = o["fine_index"][q:q + n], o["fine_diff2"][q:q + n]
        q += n
        if mc_same[i]:
            assert np.array_equal(idx, d2[i][0])
            assert (np.abs(dv - d2[i][1]) / np.abs(d2[i][1])).max() <= DIFF2_TOL
    assert relerr(o["min_diff2"], g[last + "min_diff2"]) < DIFF2_TOL
    assert relerr(o["sum_weight"], g[last + "sum_weight"]) < SUM_TOL
    same = ((o["cls"] == g[last + "class"]) & (o["rot"] == g[last + "rot"]) & (o["tilt"] == g[last + "tilt"])
            & (o["psi"] == g[last + "psi"]) & (o["xoff"] == g[last + "xoff"]) & (o["yoff"] == g[last + "yoff"]))
    wt = fine_lists_from_dump(g, last + "weight_", p.nr_trans)
    for i in np.nonzero(~same)[0]:
        top = np.sort(wt[i][1])[::-1][:2]
        assert top[1] >= top[0] * (1 - 1e-3), f"particle {i}: pose differs without a near tie"


def test_wsums_scale_spectra_and_backprojection_match_reference(runscale):
    g, p, o = runscale
    assert relerr(o["wsum_norm_correction"], g["pool0_wsum_norm_correction"]) < SUM_TOL
    for k in ["wsum_sigma2_noise", "wsum_pdf_class", "wsum_pdf_direction", "wsum_sigma2_offset", "wsum_sumw_group"]:
        assert relerr(o[k], g["pool0_after_update_" + k]) < SUM_TOL, k
    for k in ("XA", "AA"):
        mine, ref = o["wsum_scale_correction_" + k], g["pool0_wsum_scale_correction_" + k]
        assert np.abs(ref).max() > 0
        assert np.abs(mine - ref).max() <= SUM_TOL * np.abs(ref).max(), k
    # storeWeightedSums (the caller's): XA / scale and AA / scale^2 added to the particle's group
    sc = p.scale_correction[p.group]
    xa = np.zeros_like(g["pool0_after_store_wsum_signal_product_spectra"])
    aa = np.zeros_like(xa)
    np.add.at(xa, p.group, o["wsum_scale_correction_XA"] / sc[:, None])
    np.add.at(aa, p.group, o["wsum_scale_correction_AA"] / (sc * sc)[:, None])
    ref_xa = g["pool0_after_store_wsum_signal_product_spectra"] - g["pool0_after_update_wsum_signal_product_spectra"]
    ref_aa = g["pool0_after_store_wsum_reference_power_spectra"] - g["pool0_after_update_wsum_reference_power_spectra"]
    assert np.abs(xa - ref_xa).max() <= SUM_TOL * np.abs(ref_xa).max()
    assert np.abs(aa - ref_aa).max() <= SUM_TOL * np.abs(ref_aa).max()
    assert relerr(o["bp_data"], g["pool0_after_bp_bp_data"]) < SUM_TOL
    assert relerr(o["bp_weight"], g["pool0_after_bp_bp_weight"]) < SUM_TOL


def test_unscaled_library_differs(golden):
    """The scales matter: the same pool without scale correction moves the
    coarse squared differences far beyond the tolerance."""
    import dataclasses
    g = golden["map3d_scale"]
    p = dataclasses.replace(pool3d_from_dump(g, 0), do_scale_correction=False)
    with GpuContext(0, "fp32") as ctx:
        ctx.set_projectors(g["projector_data"], p.ori_size, int(g["projector_r_max"][0]))
        o = map3d_estep_pool(ctx, p)
    assert relerr(o["min_diff2"], g["pool0_pass1_min_diff2"]) > 10 * DIFF2_TOL
