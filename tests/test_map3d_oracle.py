"""The CPU restatement of the MAP3D E-step (oracle/map3d_oracle.py)
pinned stage by stage against what the reference itself recorded
(tests/golden/map3d_a, map3d_scale, map3d_cc and map3d_norm, the last at a
current size of 30 below the 32-pixel images): the coarse pass (windowing,
Minvsigma2, translated images, MyProjector::project, CTF and intensity scale
on the references, get_diff; the same hypotheses computed, every value
within 1e-10 relative, and in cross-correlation mode the recorded image
norms), the fine pass over the recorded coarse-significant points, the model
sums of updateOtherParams and the class back-projectors, each from the
reference's recorded input of that stage.  No GPU."""
import numpy as np
import pytest

from oracle import map3d_oracle as mo
from oracle import select3d_oracle as so


def recorded_coarse(g, shape):
    out = np.full(shape, np.nan)
    P, K, nd, npsi, ntr = shape
    for i, pl in enumerate(so.lists_from_dump(g, "pool0_pass0_diff2_")):
        flat = out[i].reshape(K * nd * npsi, ntr)
        flat[pl.kdp, pl.ihidden] = pl.value
    return out


@pytest.mark.parametrize("case", ["map3d_a", "map3d_scale", "map3d_cc", "map3d_norm"])
def test_coarse_pass_matches_reference(golden, case):
    g = golden[case]
    cc = bool(int(g["do_cross_correlation"][0])) if "do_cross_correlation" in g else False
    mine, norms = mo.coarse_diff2(g, 0, cc=cc)
    ref = recorded_coarse(g, mine.shape)
    ok = ~np.isnan(ref)
    assert np.array_equal(ok, ~np.isnan(mine)), "different hypotheses computed"
    rel = np.abs(mine[ok] - ref[ok]) / np.abs(ref[ok])
    print(f"{case}: {ok.sum()} coarse hypotheses, max rel diff {rel.max():.2e}")
    assert rel.max() <= 1e-10
    if cc:
        np.testing.assert_allclose(norms, g["pool0_pass0_local_sqrtXi2"], rtol=1e-12)


@pytest.mark.parametrize("case", ["map3d_a", "map3d_scale", "map3d_cc", "map3d_norm"])
def test_fine_pass_matches_reference(golden, case):
    """The fine pass over the coarse points the reference recorded as
    significant: the same list (order and ihidden) and every value within
    1e-10 relative."""
    g = golden[case]
    cc = bool(int(g["do_cross_correlation"][0])) if "do_cross_correlation" in g else False
    mine = mo.fine_diff2(g, 0, cc=cc)
    ref = so.lists_from_dump(g, "pool0_pass1_diff2_")
    worst, n = 0.0, 0
    for (kdp, ih, v), rl in zip(mine, ref):
        assert np.array_equal(kdp, rl.kdp) and np.array_equal(ih, rl.ihidden)
        worst = max(worst, float(np.max(np.abs(v - rl.value) / np.abs(rl.value))) if v.size else 0.0)
        n += v.size
    print(f"{case}: {n} fine hypotheses, max rel diff {worst:.2e}")
    assert worst <= 1e-10


@pytest.mark.parametrize("case", ["map3d_a", "map3d_scale", "map3d_cc", "map3d_norm"])
def test_update_other_params_matches_reference(golden, case):
    """updateOtherParams restated on the recorded fine-pass weights: the
    model sums of the pool, the norm-correction sums and (scale correction)
    the XA/AA spectra, within 1e-11 of each array's largest value."""
    g = golden[case]
    o = mo.update_other_params(g, 0)
    pre = "pool0_after_update_"
    for k in ("wsum_sigma2_noise", "wsum_pdf_class", "wsum_pdf_direction", "wsum_sigma2_offset", "wsum_sumw_group"):
        ref = np.asarray(g[pre + k], np.float64).reshape(np.shape(o[k]))
        err = np.max(np.abs(o[k] - ref)) / max(np.max(np.abs(ref)), 1e-300)
        assert err <= 1e-11, (k, err)
    ref = g["pool0_wsum_norm_correction"]
    assert np.max(np.abs(o["wsum_norm_correction"] - ref)) <= 1e-11 * np.max(np.abs(ref))
    if case == "map3d_scale":
        for k in ("XA", "AA"):
            ref = g["pool0_wsum_scale_correction_" + k]
            assert np.max(np.abs(o[k] - ref)) <= 1e-11 * np.max(np.abs(ref)), k


@pytest.mark.parametrize("case", ["map3d_a", "map3d_scale", "map3d_cc", "map3d_norm"])
def test_back_projection_matches_reference(golden, case):
    """backProjection restated on the recorded fine-pass weights: the
    pool's class back-projectors (data and weight) within 1e-13 of their
    largest recorded value, the same non-zero voxels."""
    g = golden[case]
    data, wt = mo.back_projection(g, 0)
    rd, rw = g["pool0_after_bp_bp_data"], g["pool0_after_bp_bp_weight"]
    ref = rd[..., 0] + 1j * rd[..., 1]
    assert np.max(np.abs(data - ref)) <= 1e-13 * np.max(np.abs(ref))
    assert np.max(np.abs(wt - rw)) <= 1e-13 * np.max(np.abs(rw))
    assert np.array_equal(wt != 0, rw != 0)
