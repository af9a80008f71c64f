"""maximizationOtherParameters (src/map2d_optimizer.cpp:1984-2045,
src/map3d_optimizer.cpp:2620-2798), the host-side FP64 update of the model
parameters other than the class maps, restated in
rome_b200.map2d / rome_b200.map3d.maximization_other_parameters: fed the
iteration's summed weights the reference recorded before its M-step
(iter_wsum_*), it must leave the model as the reference left it
(pdf_class, pdf_direction, the 2D class prior offsets, sigma2_offset,
sigma2_noise, the group scales of -scale, avg_norm_correction, LL,
ave_Pmax, refs_are_ctf_corrected): maximum likelihood, scale correction,
cross correlation (LL as the mean correlation) and norm correction.  CPU
only."""
import numpy as np
import pytest

from rome_b200 import map2d, map3d
from rome_b200.map2d import RomeError

WSUM = ("wsum_pdf_class", "wsum_pdf_direction", "wsum_sigma2_offset", "wsum_sigma2_noise", "wsum_sumw_group",
        "wsum_avg_norm_correction", "wsum_LL", "wsum_ave_Pmax")


def _scalar(a):
    return float(np.asarray(a).ravel()[0])


def _model_before(g, names):
    m = {k: np.array(g[k], np.float64) for k in names if k in g}
    m["avg_norm_correction"] = _scalar(g["avg_norm_correction"])
    m["refs_are_ctf_corrected"] = bool(int(g["refs_are_ctf_corrected"][0]))
    return m


def _check(m, g, names):
    for k in names:
        ref = np.asarray(g[k + "_after"], np.float64)
        got = np.asarray(m[k], np.float64).reshape(ref.shape)
        np.testing.assert_allclose(got, ref, rtol=1e-14, atol=0, equal_nan=True, err_msg=k)
    assert bool(m["refs_are_ctf_corrected"]) == bool(int(g["refs_are_ctf_corrected_after"][0]))


@pytest.mark.parametrize("case", ["map2d_a", "map2d_b", "map2d_c", "map2d_norm"])
def test_maximization_other_parameters_2d(golden, case):
    g = golden[case]
    wsum = {k: g["iter_" + k] for k in WSUM + ("wsum_prior_offsetx_class", "wsum_prior_offsety_class")}
    m = _model_before(g, ("sigma2_noise", "pdf_class", "prior_offsetx_class", "prior_offsety_class"))
    map2d.maximization_other_parameters(m, wsum, g["Npix_per_shell"], bool(g["do_norm_correction"][0]),
                                        bool(g["do_ctf_correction"][0]))
    _check(m, g, ("sigma2_noise", "pdf_direction", "pdf_class", "prior_offsetx_class", "prior_offsety_class",
                  "sigma2_offset", "avg_norm_correction", "LL", "ave_Pmax"))


@pytest.mark.parametrize("case", ["map3d_a", "map3d_scale", "map3d_cc", "map3d_norm"])
def test_maximization_other_parameters_3d(golden, case):
    g = golden[case]
    scale = bool(g["do_scale_correction"][0])
    names = WSUM + (("wsum_signal_product_spectra", "wsum_reference_power_spectra") if scale else ())
    wsum = {k: g["iter_" + k] for k in names}
    m = _model_before(g, ("sigma2_noise", "pdf_class", "pdf_direction", "scale_correction"))
    map3d.maximization_other_parameters(m, wsum, g["Npix_per_shell"], g["nr_particles_group"],
                                        bool(g["do_norm_correction"][0]), scale, bool(g["do_ctf_correction"][0]),
                                        cross_correlation=bool(g["do_cross_correlation"][0]))
    _check(m, g, ("sigma2_noise", "pdf_direction", "pdf_class", "sigma2_offset", "scale_correction",
                  "avg_norm_correction", "LL", "ave_Pmax"))


def test_first_cc_iteration_is_left_to_the_caller(golden):
    g = golden["map3d_cc"]
    with pytest.raises(RomeError):
        map3d.maximization_other_parameters({}, {k: g["iter_" + k] for k in WSUM}, g["Npix_per_shell"],
                                            g["nr_particles_group"], False, False, True, True,
                                            first_iteration_cc=True)
