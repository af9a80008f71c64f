"""Orientation and translation sampling of the MAP E-step for synthetic 3D
pools: HEALPix directions (NEST scheme), in-plane angles, translations and
their adaptive oversampling, restated from the reference's HealpixSampler
(src/sampling.cpp) and Healpix_Base (Healpix_2.15a/healpix_base.cc).

The library itself never derives these tables -- it consumes the caller's
(the reference's own sampler output); this module builds them for pools
that do not come from the reference, with the reference's arithmetic
(scalar libm calls through `math`, the reference's operation order), and is
checked against the reference's tables recorded in tests/golden/map3d_a.npz.
"""
from __future__ import annotations

import math
from typing import Tuple

import numpy as np

__all__ = ["healpix_directions", "psi_step_3d", "psi_angles_3d", "oversampled_orientations_3d",
           "oversampled_translations", "euler_matrix", "euler_matrix2angles", "check_direction"]

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
