"""storeWeightedSums of MAP3D (src/map3d_optimizer.cpp:1933-2045), the
host-side FP64 step after the E-step, restated in
rome_b200.map3d.store_weighted_sums: fed the reference's own E-step outputs
of the first pool of each golden case (sum_weight, min_diff2 and pmax of the
fine pass, the per-particle norm-correction sums and, with scale correction,
the XA/AA spectra), it must reproduce the model sums the reference holds
after its storeWeightedSums (wsum_sigma2_noise with the power-spectrum fill
beyond the current size, wsum_LL, wsum_ave_Pmax, wsum_avg_norm_correction
and the group spectra of the scale correction) and the per-particle dLL and
NORM it records: maximum likelihood (map3d_a), scale correction
(map3d_scale), cross correlation (map3d_cc) and norm correction with the
current size below the image size (map3d_norm).  CPU only."""
import numpy as np
import pytest

from rome_b200.map3d import pool3d_from_dump, store_weighted_sums
from tests.util import relerr


@pytest.mark.parametrize("case", ["map3d_a", "map3d_scale", "map3d_cc", "map3d_norm"])
def test_store_weighted_sums_3d_matches_reference(golden, case):
    g = golden[case]
    p = pool3d_from_dump(g, 0)
    last = "pool0_pass1_"
    est = {"sum_weight": g[last + "sum_weight"], "min_diff2": g[last + "min_diff2"], "pmax": g[last + "pmax"],
           "wsum_norm_correction": g["pool0_wsum_norm_correction"]}
    names = ["wsum_sigma2_noise", "wsum_avg_norm_correction", "wsum_LL", "wsum_ave_Pmax"]
    if p.do_scale_correction:
        est["wsum_scale_correction_XA"] = g["pool0_wsum_scale_correction_XA"]
        est["wsum_scale_correction_AA"] = g["pool0_wsum_scale_correction_AA"]
        names += ["wsum_signal_product_spectra", "wsum_reference_power_spectra"]
    wsum = {k: np.array(g["pool0_after_update_" + k], np.float64).copy() for k in names}
    for k in ("wsum_LL", "wsum_ave_Pmax", "wsum_avg_norm_correction"):
        wsum[k] = float(wsum[k][0])
    dll, norm = store_weighted_sums(p, est, g["pool0_power_imgs"], g["pool0_norm_in"],
                                    float(g["avg_norm_correction"][0]), bool(g["do_norm_correction"][0]), wsum)
    assert relerr(dll, g["pool0_dLL"]) <= 1e-12
    assert relerr(norm, g["pool0_norm_out"]) <= 1e-12
    for k in names:
        ref = np.asarray(g["pool0_after_store_" + k], np.float64)
        if ref.size == 1:
            assert abs(wsum[k] - float(ref[0])) <= 1e-12 * max(1.0, abs(wsum[k])), k
        else:
            assert relerr(wsum[k], ref.reshape(wsum[k].shape)) <= 1e-12, k
