"""storeWeightedSums (src/map2d_optimizer.cpp:1314-1414), the host-side
FP64 step after the E-step, restated in rome_b200.map2d.store_weighted_sums:
fed the reference's own E-step outputs of the first pool of each golden case
(sum_weight, min_diff2 and pmax of the last pass, the per-particle norm
correction sums, power spectra), it must reproduce the model sums the
reference holds after its storeWeightedSums (wsum_sigma2_noise with the
high-resolution fill, wsum_LL, wsum_ave_Pmax, wsum_avg_norm_correction) and
the per-particle dLL and NORM it records.  CPU only."""
import numpy as np
import pytest

from rome_b200.map2d import pool_from_dump, store_weighted_sums
from tests.util import relerr


@pytest.mark.parametrize("case", ["map2d_a", "map2d_b", "map2d_c", "map2d_norm"])
def test_store_weighted_sums_matches_reference(golden, case):
    g = golden[case]
    p = pool_from_dump(g, 0)
    last = "pool0_pass1_" if int(g["adaptive_oversampling"][0]) > 0 else "pool0_pass0_"
    est = {"sum_weight": g[last + "sum_weight"], "min_diff2": g[last + "min_diff2"], "pmax": g[last + "pmax"],
           "wsum_norm_correction": g["pool0_wsum_norm_correction"]}
    names = ["wsum_sigma2_noise", "wsum_avg_norm_correction", "wsum_LL", "wsum_ave_Pmax"]
    wsum = {k: np.array(g["pool0_after_update_" + k], np.float64).copy() for k in names}
    for k in ("wsum_LL", "wsum_ave_Pmax", "wsum_avg_norm_correction"):
        wsum[k] = float(wsum[k][0])
    dll, norm = store_weighted_sums(p, est, g["pool0_power_imgs"], g["pool0_norm_in"],
                                    float(g["avg_norm_correction"][0]), bool(g["do_norm_correction"][0]),
                                    g["Mresol_fine"], g["sigma2_noise"], wsum)
    assert relerr(dll, g["pool0_dLL"]) <= 1e-12
    assert relerr(norm, g["pool0_norm_out"]) <= 1e-12
    assert relerr(wsum["wsum_sigma2_noise"], g["pool0_after_store_wsum_sigma2_noise"]) <= 1e-12
    for k in ("wsum_LL", "wsum_ave_Pmax", "wsum_avg_norm_correction"):
        assert abs(wsum[k] - float(g["pool0_after_store_" + k][0])) <= 1e-12 * max(1.0, abs(wsum[k])), k
