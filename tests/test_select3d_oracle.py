"""The CPU restatement of the MAP3D posterior and significance steps
(oracle/select3d_oracle.py) pinned against the reference's own recorded
lists (tests/golden/map3d_a, map3d_scale, map3d_cc, map3d_norm: oracle/_ref/map3d_dump):
from the recorded diff2 lists it reproduces the recorded weights (1e-13
relative), exp_sum_weight (1e-12), significant_weight and NR_SIGN, the
coarse significance mask, and in cross-correlation mode the single weight-1
entry.  No GPU."""
import numpy as np
import pytest

from oracle import select3d_oracle as so


def _pass_shape(g, p):
    ang = g[f"pool0_pass{p}_angles"]
    otx = g[f"pool0_pass{p}_over_trans_x"]
    return int(ang.shape[2]), int(otx.shape[1])


@pytest.mark.parametrize("case", ["map3d_a", "map3d_scale", "map3d_norm"])
@pytest.mark.parametrize("ipass", [0, 1])
def test_ml_weights_and_significance_match_reference(golden, case, ipass):
    g = golden[case]
    nd, npsi = int(g["nr_dir"][0]), int(g["nr_psi"][0])
    nor, notr = _pass_shape(g, ipass)
    pre = f"pool0_pass{ipass}_"
    d2 = so.lists_from_dump(g, pre + "diff2_")
    wr = so.lists_from_dump(g, pre + "weight_")
    frac = float(g["adaptive_fraction"][0])
    for i, (pl, rw) in enumerate(zip(d2, wr)):
        assert np.array_equal(pl.kdp, rw.kdp) and np.array_equal(pl.ihidden, rw.ihidden)
        w, s, mx = so.weights_ml(pl, float(g[pre + "min_diff2"][i]), g["pdf_direction"], nd, npsi,
                                 g["trans_x"], g["trans_y"], float(g["pool0_old_offsetx"][i]),
                                 float(g["pool0_old_offsety"][i]), g["prior_offsetx_class"],
                                 g["prior_offsety_class"], float(g["sigma2_offset"][0]), nor, notr)
        np.testing.assert_allclose(w, rw.value, rtol=1e-13, atol=0)
        assert s == pytest.approx(float(g[pre + "sum_weight"][i]), rel=1e-12)
        assert mx / s == pytest.approx(float(g[pre + "pmax"][i]), rel=1e-12)
        pose = so.best_pose(pl, w, nd, npsi, nor, notr, g[f"pool0_pass{ipass}_angles"],
                            g[f"pool0_pass{ipass}_over_trans_x"], g[f"pool0_pass{ipass}_over_trans_y"],
                            float(g["pool0_old_offsetx"][i]), float(g["pool0_old_offsety"][i]))
        for k in ("class", "rot", "tilt", "psi", "xoff", "yoff"):
            assert pose[k] == g[pre + k][i], (i, k)
        sig, n = so.significance(rw.value, float(g[pre + "sum_weight"][i]), frac)
        assert sig == float(g[pre + "significant_weight"][i])
        if ipass == 0:
            assert n == int(g[pre + "nr_sign"][i])
            # exp_Mcoarse_significant: the listed coarse points with w >= significant_weight
            ntr = int(g["nr_trans"][0])
            mask = np.zeros(g[pre + "Mcoarse_significant"].shape[1], np.int8)
            keep = rw.value >= sig
            mask[rw.kdp[keep] * ntr + rw.ihidden[keep]] = 1
            assert np.array_equal(mask, g[pre + "Mcoarse_significant"][i]), i


def test_cc_selection_matches_reference(golden):
    g = golden["map3d_cc"]
    frac = float(g["adaptive_fraction"][0])
    checked = 0
    for k in range(6):
        for ipass in (0, 1):
            pre = f"pool{k}_pass{ipass}_"
            d2 = so.lists_from_dump(g, pre + "diff2_")
            wr = so.lists_from_dump(g, pre + "weight_")
            for i, (pl, rw) in enumerate(zip(d2, wr)):
                q, v = so.weights_cc(pl)
                assert rw.value.size == 1 and rw.value[0] == 1.0
                assert pl.kdp[q] == rw.kdp[0] and pl.ihidden[q] == rw.ihidden[0], (k, ipass, i)
                assert v == float(g[pre + "min_diff2"][i])
                assert float(g[pre + "sum_weight"][i]) == 1.0
                sig, n = so.significance(rw.value, 1.0, frac)
                assert sig == float(g[pre + "significant_weight"][i]) == 1.0 and n == 1
                checked += 1
    assert checked == 2 * 24


def test_pdf_offset_restatement():
    # Gaussian of the offset distance, normalised in 2D; the sharp limit below sigma2 1e-4
    v = so.calculate_pdf_offset(np.array([1.0]), np.array([2.0]), np.array([0.0]), np.array([0.0]), 2.0)
    assert v[0] == pytest.approx(np.exp(-5.0 / 4.0) / (4.0 * np.pi), rel=1e-15)
    assert so.calculate_pdf_offset(np.array([0.0, 1.0]), np.zeros(2), np.zeros(2), np.zeros(2), 0.0).tolist() == [1, 0]
