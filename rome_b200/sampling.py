"""Orientation and translation sampling of the MAP E-step for synthetic 3D
pools: HEALPix directions (NEST scheme), in-plane angles, translations and
their adaptive oversampling, restated from the reference's HealpixSampler
(src/sampling.cpp) and Healpix_Base (Healpix_2.15a/healpix_base.cc).

The library itself never derives these tables -- it consumes the caller's
(the reference's own sampler output); this module builds them for pools
that do not come from the reference, with the reference's arithmetic
(scalar libm calls through `math`, the reference's operation order), and is
checked against the reference's tables recorded in tests/golden/map3d_a.npz.
It also restates the per-iteration choice of image sizes (the resolution
reached, the current and coarse sizes, the shell counts and resolution
tables: MAPModel::updateCurrentResolution and
updateImageSizeAndResolutionPointers), checked against every golden case.
"""
from __future__ import annotations

import math
from typing import Tuple

import numpy as np

__all__ = ["healpix_directions", "psi_step_3d", "psi_angles_3d", "oversampled_orientations_3d",
           "oversampled_translations", "euler_matrix", "euler_matrix2angles", "check_direction", "angular_sampling",
           "resolution_indices", "npix_per_shell", "current_resolution", "image_sizes"]

ROME_PI = 3.14159265358979323846      # rome_pi, src/math.h:38
HALFPI = 1.570796326794896619231321691639751442099  # Healpix_2.15a/lsconstants.h:43
FLT_EPSILON = 1.1920928955078125e-07
JRLL = (2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4)  # healpix_base.cc ring / phi offsets of the 12 base faces
JPLL = (1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7)


def _compress(v: int) -> int:
    """Every other bit of v (bit 2i -> bit i)."""
    out, b = 0, 0
    while v:
        out |= (v & 1) << b
        v >>= 2
        b += 1
    return out


def _spread(v: int) -> int:
    """Bit i of v -> bit 2i."""
    out, b = 0, 0
    while v:
        out |= (v & 1) << (2 * b)
        v >>= 1
        b += 1
    return out


def nest2xyf(pix: int, order: int) -> Tuple[int, int, int]:
    """Healpix_Base::nest2xyf (healpix_base.cc:127-136)."""
    face = pix >> (2 * order)
    p = pix & ((1 << (2 * order)) - 1)
    return _compress(p), _compress(p >> 1), face


def xyf2nest(x: int, y: int, face: int, order: int) -> int:
    """Healpix_Base::xyf2nest (healpix_base.cc:138-143)."""
    return (face << (2 * order)) + _spread(x) + (_spread(y) << 1)


def pix2ang_z_phi_nest(pix: int, order: int) -> Tuple[float, float]:
    """Healpix_Base::pix2ang_z_phi, NEST scheme (healpix_base.cc:494-528)."""
    nside = 1 << order
    npix = 12 * nside * nside
    fact2 = 4.0 / npix
    fact1 = (nside << 1) * fact2
    nl4 = nside * 4
    ix, iy, face = nest2xyf(pix, order)
    jr = (JRLL[face] << order) - ix - iy - 1
    if jr < nside:
        nr, kshift = jr, 0
        z = 1 - nr * nr * fact2
    elif jr > 3 * nside:
        nr, kshift = nl4 - jr, 0
        z = nr * nr * fact2 - 1
    else:
        nr = nside
        z = (2 * nside - jr) * fact1
        kshift = (jr - nside) & 1
    jp = (JPLL[face] * nr + ix - iy + 1 + kshift) // 2
    if jp > nl4:
        jp -= nl4
    if jp < 1:
        jp += nl4
    phi = (jp - (kshift + 1) * 0.5) * (HALFPI / nr)
    return z, phi


def check_direction(rot: float, tilt: float) -> Tuple[float, float]:
    """HealpixSampler::checkDirection (src/sampling.h:59-76): rot in [-180, 180], tilt >= 0."""
    if tilt < 0.0:
        tilt = -tilt
        rot += 180.0
    while True:
        if rot > 180.0:
            rot -= 360.0
        elif rot < -180.0:
            rot += 360.0
        else:
            return rot, tilt


def _rad2deg(r: float) -> float:
    return r * 180.0 / ROME_PI


def _deg2rad(d: float) -> float:
    return d * ROME_PI / 180.0


def healpix_directions(order: int) -> np.ndarray:
    """(rot, tilt) of every HEALPix pixel in NEST order, C1 symmetry
    (HealpixSampler::initialize, src/sampling.cpp:204-220)."""
    n = 12 * (1 << (2 * order))
    out = np.zeros((n, 2))
    for ipix in range(n):
        z, phi = pix2ang_z_phi_nest(ipix, order)
        out[ipix] = check_direction(_rad2deg(phi), math.acos(z) * 180.0 / ROME_PI)
    return out


def psi_step_3d(order: int) -> float:
    """Default 3D in-plane step 360 / (6 * 2^order) (src/sampling.cpp:70-73)."""
    return 360.0 / (6 * round(2.0 ** order))


def psi_angles_3d(order: int) -> np.ndarray:
    step = psi_step_3d(order)
    n = int(math.ceil(360.0 / step))
    return np.array([i * (360.0 / n) for i in range(n)])


def euler_matrix(rot: float, tilt: float, psi: float) -> np.ndarray:
    """Euler_angles2matrix (src/math.cpp:86-114), degrees."""
    a, b, g = _deg2rad(rot), _deg2rad(tilt), _deg2rad(psi)
    ca, cb, cg = math.cos(a), math.cos(b), math.cos(g)
    sa, sb, sg = math.sin(a), math.sin(b), math.sin(g)
    cc, cs, sc, ss = cb * ca, cb * sa, sb * ca, sb * sa
    return np.array([[cg * cc - sg * sa, cg * cs + sg * ca, -cg * sb],
                     [-sg * cc - cg * sa, -sg * cs + cg * ca, sg * sb],
                     [sc, ss, cb]])


def _sgn(x: float) -> float:
    return 1.0 if x >= 0 else -1.0


def euler_matrix2angles(A: np.ndarray) -> Tuple[float, float, float]:
    """Euler_matrix2angles (src/math.cpp:149-196), degrees."""
    abs_sb = math.sqrt(A[0][2] * A[0][2] + A[1][2] * A[1][2])
    if abs_sb > 16 * FLT_EPSILON:
        gamma = math.atan2(A[1][2], -A[0][2])
        alpha = math.atan2(A[2][1], A[2][0])
        if abs(math.sin(gamma)) < FLT_EPSILON:
            sign_sb = _sgn(-A[0][2] / math.cos(gamma))
        else:
            sign_sb = _sgn(A[1][2]) if math.sin(gamma) > 0 else -_sgn(A[1][2])
        beta = math.atan2(sign_sb * abs_sb, A[2][2])
    elif _sgn(A[2][2]) > 0:
        alpha, beta = 0.0, 0.0
        gamma = math.atan2(-A[1][0], A[0][0])
    else:
        alpha, beta = 0.0, ROME_PI
        gamma = math.atan2(A[1][0], -A[0][0])
    return _rad2deg(alpha), _rad2deg(beta), _rad2deg(gamma)


def _perturb(rot: float, tilt: float, psi: float, p: float) -> Tuple[float, float, float]:
    """HealpixSampler::addPerturbation for one orientation (src/sampling.cpp:509-528)."""
    A = euler_matrix(rot, tilt, psi)
    R = euler_matrix(p, p, p)
    AR = [[A[i][0] * R[0][j] + A[i][1] * R[1][j] + A[i][2] * R[2][j] for j in range(3)] for i in range(3)]
    return euler_matrix2angles(AR)


def oversampled_orientations_3d(order: int, oversampling: int, random_perturbation: float = 0.0) -> np.ndarray:
    """angles[dir][psi][over_rot][(rot, tilt, psi)] of one pass
    (HealpixSampler::getOrientations3D, src/sampling.cpp:530-592): for
    oversampling 0 the coarse grid; for oversampling o the 4^o NEST children
    of each direction x 2^o sub-angles of each psi, over_rot = child * 2^o +
    sub-psi; then the random perturbation composed on the right."""
    dirs = healpix_directions(order)
    psis = psi_angles_3d(order)
    step = psi_step_3d(order)
    ndir, npsi = len(dirs), len(psis)
    nps, nds = 1 << oversampling, 1 << (2 * oversampling)
    myperturb = random_perturbation * (360.0 / (6 * round(2.0 ** order)))
    out = np.zeros((ndir, npsi, nps * nds, 3))
    fact = 1 << oversampling
    for d in range(ndir):
        if oversampling == 0:
            children = [tuple(dirs[d])]
        else:
            x, y, face = nest2xyf(d, order)
            children = []
            for j in range(fact * y, fact * (y + 1)):
                for i in range(fact * x, fact * (x + 1)):
                    z, phi = pix2ang_z_phi_nest(xyf2nest(i, j, face, order + oversampling), order + oversampling)
                    children.append(check_direction(_rad2deg(phi), math.acos(z) * 180.0 / ROME_PI))
        for ps in range(npsi):
            for c, (rot, tilt) in enumerate(children):
                for s in range(nps):
                    psi = psis[ps] if oversampling == 0 else psis[ps] - 0.5 * step + (0.5 + s) * step / nps
                    ang = (rot, tilt, psi)
                    if abs(random_perturbation) > 0.0:
                        ang = _perturb(rot, tilt, psi, myperturb)
                    out[d, ps, c * nps + s] = ang
    return out


def oversampled_translations(tx: np.ndarray, ty: np.ndarray, offset_step: float, oversampling: int,
                             random_perturbation: float = 0.0):
    """over_trans_x/y[trans][over_trans] (HealpixSampler::getTranslations,
    src/sampling.cpp:312-349): 2^o x 2^o sub-steps, over_trans = iy * 2^o + ix."""
    n = 1 << oversampling
    ox = np.zeros((len(tx), n * n))
    oy = np.zeros((len(tx), n * n))
    myperturb = random_perturbation * offset_step
    for t in range(len(tx)):
        for iy in range(n):
            for ix in range(n):
                if oversampling == 0:
                    x, y = tx[t], ty[t]
                else:
                    y = ty[t] - 0.5 * offset_step + (0.5 + iy) * offset_step / n
                    x = tx[t] - 0.5 * offset_step + (0.5 + ix) * offset_step / n
                if abs(random_perturbation) > 0.0:
                    x += myperturb
                    y += myperturb
                ox[t, iy * n + ix] = x
                oy[t, iy * n + ix] = y
    return ox, oy


# ---- image sizes of an iteration (MAPModel::updateCurrentResolution, updateImageSizeAndResolutionPointers) ----

def angular_sampling(healpix_order: int = -1, psi_step: float = 0.0, adaptive_oversampling: int = 0) -> float:
    """HealpixSampler::getAngularSampling (src/sampling.cpp:287-295): 360 /
    (6 * 2^(order + oversampling)) in 3D (healpix_order >= 0), else the psi
    step / 2^oversampling."""
    if healpix_order >= 0:
        return 360.0 / (6 * round(2.0 ** (healpix_order + adaptive_oversampling)))
    return psi_step / 2.0 ** adaptive_oversampling


def resolution_indices(size: int) -> np.ndarray:
    """Mresol_fine / Mresol_coarse of an image of `size` (src/map_model.cpp:540-575):
    the rounded radius of every coefficient of the FFTW half-plane, -1 beyond
    size / 2 and on the negative half of the x = 0 column."""
    Fs = size // 2 + 1
    i = np.arange(size)
    ip = np.where(i < Fs, i, i - size)
    jp = np.arange(Fs)
    ires = np.round(np.sqrt(ip[:, None] ** 2 + jp[None, :] ** 2)).astype(np.int32)
    bad = (ires >= Fs) | ((jp[None, :] == 0) & (ip[:, None] < 0))
    return np.where(bad, -1, ires).astype(np.int32).reshape(-1)


def npix_per_shell(ori_size: int) -> np.ndarray:
    """Npix_per_shell (src/map_model.cpp:523-537): coefficients of the
    ori_size half-plane per rounded radius, the negative half of the x = 0
    column left out."""
    r = resolution_indices(ori_size)
    return np.bincount(r[r >= 0], minlength=ori_size // 2 + 1).astype(np.int32)


def current_resolution(data_vs_prior: np.ndarray, ori_size: int, pixel_size: float, minres_map: int,
                       do_map: bool = True, ini_high: float = 0.0, set_by_ini_high: bool = False) -> float:
    """MAPModel::updateCurrentResolution (src/map_model.cpp:375-424), the
    resolution (1/A) the next iteration works to: with MAP, from ini_high
    when set_by_ini_high, else the shell before the first one (from 1) at
    which any class's data_vs_prior drops below 1, the largest over classes
    and at least minres_map; Nyquist without MAP."""
    if do_map:
        if set_by_ini_high:
            maxres = int(round(ori_size * pixel_size / ini_high))
        else:
            maxres = 0
            for row in np.asarray(data_vs_prior, np.float64):
                ires = 1
                while ires < ori_size // 2 and not row[ires] < 1.0:
                    ires += 1
                maxres = max(maxres, ires - 1)
            maxres = max(maxres, minres_map)
    else:
        maxres = ori_size // 2
    return maxres / (pixel_size * ori_size)


def image_sizes(current_res: float, ori_size: int, pixel_size: float, adaptive_oversampling: int,
                angular_sampling_deg: float, particle_diameter: float, ref_dim: int, incr_size: int = 10,
                ave_pmax: float = 0.0, has_high_fsc_at_limit: bool = False, do_use_all_data: bool = False) -> dict:
    """MAPModel::updateImageSizeAndResolutionPointers (src/map_model.cpp:463-576):
    current_size = 2 * (the resolution's pixel + incr_size) (+ a quarter of
    the image instead with a high FSC at the limit and Pmax > 0.1), at most
    ori_size; with adaptive oversampling coarse_size = 2 * ceil(pixel_size *
    ori_size / coarse_resolution), coarse_resolution the arc the angular
    step sweeps on the particle's diameter divided by 1.2 (3D) or 1.5 (2D),
    at most current_size; the shell counts and resolution tables of those
    sizes."""
    maxres = int(current_res * pixel_size * ori_size + 0.0001)  # getPixelFromResolution, src/map_model.h:102
    if ave_pmax > 0.1 and has_high_fsc_at_limit:
        maxres += int(round(0.25 * ori_size / 2))
    else:
        maxres += incr_size
    cur = ori_size if do_use_all_data else maxres * 2
    cur = min(cur, ori_size)
    if adaptive_oversampling > 0:
        rotated_distance = (angular_sampling_deg / 360.0) * ROME_PI * particle_diameter
        keepsafe = 1.2 if ref_dim == 3 else 1.5
        coarse = 2 * int(math.ceil(pixel_size * ori_size / (rotated_distance / keepsafe)))
        coarse = min(ori_size, coarse)
    else:
        coarse = cur
    coarse = min(cur, coarse)
    return {"current_size": cur, "coarse_size": coarse, "Npix_per_shell": npix_per_shell(ori_size),
            "Mresol_fine": resolution_indices(cur), "Mresol_coarse": resolution_indices(coarse)}
