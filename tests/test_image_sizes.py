"""The image sizes of an iteration, restated in rome_b200.sampling
(MAPModel::updateCurrentResolution and updateImageSizeAndResolutionPointers,
src/map_model.cpp:375-576): from the data_vs_prior the reference held at
the start of each golden case's dumped iteration, the current and coarse
sizes, the pixel count per shell and both resolution tables the reference
used in that iteration, exactly.  2D (psi-step sampling, keep-safe 1.5)
and 3D (HEALPix sampling, 1.2); single pass and adaptive oversampling;
current size equal to and below the image size.  CPU only."""
import numpy as np
import pytest

from rome_b200 import sampling

CASES = ["map2d_a", "map2d_b", "map2d_c", "map2d_norm", "map3d_a", "map3d_cc", "map3d_scale", "map3d_norm"]


@pytest.mark.parametrize("case", CASES)
def test_image_sizes_match_reference(golden, case):
    g = golden[case]
    i = lambda k: int(np.asarray(g[k]).ravel()[0])  # noqa: E731
    f = lambda k: float(np.asarray(g[k]).ravel()[0])  # noqa: E731
    ori, pixel = i("ori_size"), f("pixel_size")
    if case.startswith("map3d"):
        ref_dim, ang = 3, sampling.angular_sampling(healpix_order=i("healpix_order"))
        diameter = (ori - 5) * pixel          # the default: (ori_size - width_mask_edge) * pixel_size
    else:
        ref_dim, ang = 2, sampling.angular_sampling(psi_step=f("psi_step"))
        diameter = f("prep_particle_diameter")
    res = sampling.current_resolution(g["data_vs_prior_before"], ori, pixel, i("minres_map"), bool(i("do_map")))
    got = sampling.image_sizes(res, ori, pixel, i("adaptive_oversampling"), ang, diameter, ref_dim)
    assert got["current_size"] == i("current_size")
    assert got["coarse_size"] == i("coarse_size")
    for k in ("Npix_per_shell", "Mresol_fine", "Mresol_coarse"):
        assert np.array_equal(got[k], np.asarray(g[k]).ravel()), k


def test_resolution_rules():
    # the shell before the first with data_vs_prior < 1, the largest over classes, at least minres_map
    dvp = np.array([[9, 5, 3, 0.5, 2, 2, 2, 2], [9, 5, 3, 2, 2, 0.9, 2, 2]], float)
    assert sampling.current_resolution(dvp, 16, 2.0, 1) == 4 / 32
    assert sampling.current_resolution(dvp, 16, 2.0, 6) == 6 / 32
    assert sampling.current_resolution(dvp, 16, 2.0, 1, do_map=False) == 8 / 32
    assert sampling.current_resolution(dvp, 16, 2.0, 1, ini_high=8.0, set_by_ini_high=True) == 4 / 32
    # current size 2 * (pixel + incr_size), at most the image size; coarse at most the current size
    s = sampling.image_sizes(4 / 128, 64, 2.0, 1, 30.0, 100.0, 3)
    assert s["current_size"] == 28 and s["coarse_size"] == 2 * int(np.ceil(128 / ((30 / 360) * np.pi * 100 / 1.2)))
    assert sampling.image_sizes(4 / 128, 64, 2.0, 0, 30.0, 100.0, 3)["coarse_size"] == 28
    assert sampling.image_sizes(30 / 128, 64, 2.0, 0, 30.0, 100.0, 3)["current_size"] == 64
    # shells of a 4-pixel image: radius 0 once, 1 four times, 2 five times (corner and x = 0, y < 0 left out)
    assert sampling.npix_per_shell(4).tolist() == [1, 4, 5]
