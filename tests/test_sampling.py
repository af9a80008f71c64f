"""The restated 3D sampler (rome_b200/sampling.py: HEALPix NEST directions,
in-plane angles, adaptive oversampling, random perturbation, translations)
reproduces the reference's tables bit for bit: the coarse and fine angle
tables and the over-translations that oracle/ref_harness/map3d_dump
recorded from HealpixSampler (HEALPix order 1, oversampling 1) in
tests/golden/map3d_a.npz."""
import numpy as np
import pytest

from rome_b200.sampling import (check_direction, euler_matrix, euler_matrix2angles, healpix_directions,
                                nest2xyf, oversampled_orientations_3d, oversampled_translations, pix2ang_z_phi_nest,
                                psi_angles_3d, xyf2nest)


@pytest.fixture(scope="module")
def g(golden):
    return golden["map3d_a"]


def _perturbation(g):
    # over_trans = trans + random_perturbation * offset_step (offset_step 1 in this fixture)
    return float(g["pool0_pass0_over_trans_x"][0, 0] - g["trans_x"][0])


def test_coarse_and_fine_angle_tables_bit_exact(g):
    order = int(g["healpix_order"][0])
    rp = _perturbation(g)
    assert np.array_equal(oversampled_orientations_3d(order, 0, rp), g["pool0_pass0_angles"])
    assert np.array_equal(oversampled_orientations_3d(order, 1, rp), g["pool0_pass1_angles"])


def test_over_translations_bit_exact(g):
    rp = _perturbation(g)
    for o, key in ((0, "pool0_pass0_"), (1, "pool0_pass1_")):
        ox, oy = oversampled_translations(g["trans_x"], g["trans_y"], 1.0, o, rp)
        assert np.array_equal(ox, g[key + "over_trans_x"]) and np.array_equal(oy, g[key + "over_trans_y"])


@pytest.mark.parametrize("order", [0, 1, 2, 3])
def test_healpix_nest_properties(order):
    n = 12 << (2 * order)
    for pix in range(0, n, max(1, n // 97)):
        x, y, f = nest2xyf(pix, order)
        assert xyf2nest(x, y, f, order) == pix
    d = healpix_directions(order)
    assert d.shape == (n, 2)
    # equal-area pixels: mean of z = cos(tilt) is 0, rot in [-180, 180], tilt in [0, 180]
    z = np.array([pix2ang_z_phi_nest(p, order)[0] for p in range(n)])
    assert abs(z.mean()) < 1e-12
    assert (d[:, 0] >= -180).all() and (d[:, 0] <= 180).all() and (d[:, 1] >= 0).all() and (d[:, 1] <= 180).all()
    assert len(psi_angles_3d(order)) == 6 << order


def test_euler_round_trip():
    rng = np.random.default_rng(0)
    for _ in range(200):
        rot, tilt, psi = rng.uniform(-180, 180), rng.uniform(1, 179), rng.uniform(-180, 180)
        A = euler_matrix(rot, tilt, psi)
        np.testing.assert_allclose(A @ A.T, np.eye(3), atol=1e-14)
        r2, t2, p2 = euler_matrix2angles(A)
        np.testing.assert_allclose(euler_matrix(r2, t2, p2), A, atol=1e-12)
    assert check_direction(200.0, -10.0) == (20.0, 10.0)
