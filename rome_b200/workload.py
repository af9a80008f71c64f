"""Synthetic MAP2D pools at the benchmark configurations.

Builds everything ``rome_gpu_map2d_estep_pool`` consumes without touching
disk: class references (random Gaussian-blob templates), their padded
Fourier projector maps, particles in Fourier space (a rotated, shifted,
CTF-modulated projection plus white complex noise at a target SNR), the
sampling tables and the model state.  The numerics follow the reference's
definitions (cited per function) so the hypotheses, layouts and posterior
shapes match a real iteration; values are seeded synthetic data.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np

from .map2d import Map2dPool
from .synthetic import ctf_image


@dataclasses.dataclass
class Map2dWorkload:
    n_particles: int = 1000
    ori_size: int = 64
    current_size: Optional[int] = None  # default: ori_size
    n_classes: int = 10
    n_blobs: int = 20
    blob_sigma: tuple = (2.0, 6.0)
    psi_step: float = 10.0
    offset_range: int = 5
    offset_step: int = 1
    max_shift: float = 4.0
    pixel: float = 2.0
    snr: float = 0.05
    defocus: tuple = (10000.0, 30000.0)
    seed: int = 1
    random_perturbation: float = 0.0  # sampler perturbation in units of the step
    particle_seed: Optional[int] = None  # particles from another seed, same class templates


def grid_templates(rng, ori, K, n_blobs, sig):
    c = np.arange(ori) - ori // 2
    yy, xx = np.meshgrid(c, c, indexing="ij")
    refs = np.zeros((K, ori, ori))
    for k in range(K):
        r = 0.3 * ori * np.sqrt(rng.uniform(0, 1, n_blobs))
        t = rng.uniform(0, 2 * np.pi, n_blobs)
        s = rng.uniform(sig[0], sig[1], n_blobs)
        a = rng.uniform(0.5, 1.0, n_blobs)
        for q in range(n_blobs):
            refs[k] += a[q] * np.exp(-((xx - r[q] * np.cos(t[q])) ** 2 + (yy - r[q] * np.sin(t[q])) ** 2) / (2 * s[q] ** 2))
    return refs


def projector_map_2d(ref: np.ndarray, current_size: int, padding: int = 2):
    """MyProjector::computeFourierTransformMap for a 2D reference
    (src/reconstruct.cpp:106-223): gridding correction, zero padding by 2,
    centred FFT normalised by the padded size, scaled by padding^2 and
    windowed to r_max.  Returns (data [pad][pad/2+1][2], r_max, pad_size)."""
    ori = ref.shape[0]
    r_max = min(current_size // 2, ori // 2)
    pad_size = 2 * (padding * r_max + 1) + 1
    padF = pad_size // 2 + 1
    # griddingCorrect (reconstruct.cpp:61-103): divide by sinc^2
    c = np.arange(ori) - ori // 2
    yy, xx = np.meshgrid(c, c, indexing="ij")
    r = np.sqrt(xx * xx + yy * yy)
    rval = r / (ori * padding)
    sinc = np.where(r > 0, np.sin(np.pi * rval) / np.where(r > 0, np.pi * rval, 1.0), 1.0)
    vol = ref / (sinc * sinc)
    P = padding * ori
    Mpad = np.zeros((P, P))
    o = P // 2 - ori // 2
    Mpad[o:o + ori, o:o + ori] = vol
    F = np.fft.rfft2(np.fft.ifftshift(Mpad)) / (P * P) * (padding * padding)
    data = np.zeros((pad_size, padF, 2))
    hP = P // 2 + 1
    max_r2 = (r_max * padding) ** 2
    for i in range(P):
        ip = i if i < hP else i - P
        jp = np.arange(hP)
        ok = ip * ip + jp * jp <= max_r2
        jj = jp[ok]
        y = ip + pad_size // 2
        data[y, jj, 0] = F[i, jj].real
        data[y, jj, 1] = F[i, jj].imag
    return data, r_max, pad_size


def rotate2d_np(data: np.ndarray, r_max: int, psi_deg: np.ndarray, size: int, padding: int = 2) -> np.ndarray:
    """MyProjector::rotate2D (src/reconstruct.cpp:823-958) for many angles,
    vectorised; returns complex [n][size][size/2+1]."""
    pad = data.shape[0]
    Fs = size // 2 + 1
    my_r = min(r_max, size // 2)
    rows = np.arange(size)
    yv = np.where(rows <= my_r, rows, rows - size)
    rowok = (rows <= my_r) | (rows >= size - my_r)
    yy, xx = np.meshgrid(yv, np.arange(Fs), indexing="ij")
    ok = rowok[:, None] & (xx <= my_r) & (xx * xx + yy * yy <= my_r * my_r)
    ys, xs = yy[ok].astype(np.float64), xx[ok].astype(np.float64)
    psi = np.deg2rad(np.atleast_1d(psi_deg))[:, None]
    cg, sg = np.cos(psi), np.sin(psi)
    xp = (cg * xs + -sg * ys) * padding
    yp = (sg * xs + cg * ys) * padding
    neg = xp < 0
    xp = np.where(neg, -xp, xp)
    yp = np.where(neg, -yp, yp)
    x0 = np.floor(xp).astype(np.int64)
    fx = xp - x0
    y0 = np.floor(yp).astype(np.int64)
    fy = yp - y0
    y0 = y0 + pad // 2
    cplx = data[..., 0] + 1j * data[..., 1]
    d00, d01 = cplx[y0, x0], cplx[y0, x0 + 1]
    d10, d11 = cplx[y0 + 1, x0], cplx[y0 + 1, x0 + 1]
    dx0 = d00 + (d01 - d00) * fx
    dx1 = d10 + (d11 - d10) * fx
    v = dx0 + (dx1 - dx0) * fy
    v = np.where(neg, np.conj(v), v)
    out = np.zeros((psi.shape[0], size, Fs), np.complex128)
    out[:, ok] = v
    return out


def mresol(size: int) -> np.ndarray:
    """Mresol_fine / Mresol_coarse (src/map_model.cpp:540-575)."""
    from .sampling import resolution_indices
    return resolution_indices(size)


def translations(offset_range: int, offset_step: int):
    """HealpixSampler::setTranslations (src/sampling.cpp:121-172)."""
    maxr = math.ceil(offset_range / offset_step)
    tx, ty = [], []
    for ix in range(-maxr, maxr + 1):
        for iy in range(-maxr, maxr + 1):
            x, y = ix * offset_step, iy * offset_step
            if x * x + y * y <= offset_range * offset_range:
                tx.append(float(x))
                ty.append(float(y))
    return np.array(tx), np.array(ty)


def psi_angles(psi_step: float):
    """HealpixSampler::setOrientations, 2D in-plane angles (src/sampling.cpp:174-194)."""
    n = math.ceil(360.0 / psi_step)
    step = 360.0 / n
    return np.arange(n) * step, step


def build_map2d(w: Map2dWorkload):
    """Returns (Map2dPool for all particles, projector data [K][pad][padF][2], r_max, truth dict)."""
    rng = np.random.default_rng(w.seed)
    ori = w.ori_size
    cur = w.current_size or ori
    K = w.n_classes
    refs = grid_templates(rng, ori, K, w.n_blobs, w.blob_sigma)
    proj = []
    for k in range(K):
        d, r_max, pad = projector_map_2d(refs[k], cur)
        proj.append(d)
    proj = np.stack(proj)
    if w.particle_seed is not None:
        rng = np.random.default_rng(w.particle_seed)
    N = w.n_particles
    Fs = cur // 2 + 1
    cls = rng.integers(0, K, N)
    psi = rng.uniform(0, 360, N)
    sx = rng.uniform(-w.max_shift, w.max_shift, N)
    sy = rng.uniform(-w.max_shift, w.max_shift, N)
    du = rng.uniform(*w.defocus, N)
    dv = rng.uniform(*w.defocus, N)
    da = rng.uniform(0, 180, N)
    rows = np.arange(cur)
    ky = np.where(rows < Fs, rows, rows - cur).astype(np.float64)[:, None]
    kx = np.arange(Fs, dtype=np.float64)[None, :]
    Fr = np.zeros((N, cur * Fs))
    Fi = np.zeros((N, cur * Fs))
    ctf = np.zeros((N, cur * Fs))
    mres = mresol(cur)
    sig_all = []
    chunk = 256
    for c0 in range(0, N, chunk):
        c1 = min(N, c0 + chunk)
        for k in np.unique(cls[c0:c1]):
            idx = np.nonzero(cls[c0:c1] == k)[0] + c0
            P = rotate2d_np(proj[k], r_max, psi[idx], cur)
            for q, i in enumerate(idx):
                c = ctf_image(cur, ori, w.pixel, du[i], dv[i], da[i], 300.0, 2.7, 0.1)
                # an image shifted by -s is brought back by the offset s (XOFF/YOFF)
                ph = np.exp(2j * np.pi * (kx * sx[i] + ky * sy[i]) / ori)
                s = P[q] * ph * c
                Fr[i] = s.real.reshape(-1)
                Fi[i] = s.imag.reshape(-1)
                ctf[i] = c.reshape(-1)
                sig_all.append(np.mean(np.abs(s.reshape(-1)[mres > 0]) ** 2))
    # white noise per component at the requested SNR (signal power / noise power)
    sig_pow = float(np.mean(sig_all))
    sigma2 = sig_pow / (2.0 * w.snr)
    Fr += rng.normal(0, math.sqrt(sigma2), Fr.shape)
    Fi += rng.normal(0, math.sqrt(sigma2), Fi.shape)
    Fr[:, 0] = 0.0
    Fi[:, 0] = 0.0
    oriF = ori // 2 + 1
    tx, ty = translations(w.offset_range, w.offset_step)
    pa, pstep = psi_angles(w.psi_step)
    pert = w.random_perturbation
    over_psi = (pa + pert * pstep)[:, None]
    over_tx = (tx + pert * w.offset_step)[:, None]
    over_ty = (ty + pert * w.offset_step)[:, None]
    pool = Map2dPool(
        ori_size=ori, current_size=cur, coarse_size=cur, nr_classes=K, nr_groups=1, adaptive_oversampling=0,
        over_psi=[over_psi], over_trans_x=[over_tx], over_trans_y=[over_ty], trans_x=tx, trans_y=ty,
        Fimg_real=Fr, Fimg_imag=Fi, Fimg_nomask_real=Fr.copy(), Fimg_nomask_imag=Fi.copy(), Fctf=ctf,
        highres_Xi2=np.zeros(N), old_offsetx=np.zeros(N), old_offsety=np.zeros(N), group=np.zeros(N, np.int32),
        sigma2_noise=np.full((1, oriF), sigma2), Mresol_fine=mres, Mresol_coarse=mres.copy(),
        pdf_class=np.full(K, 1.0 / K), pdf_direction=np.full(K, 1.0 / K), prior_offsetx_class=np.zeros(K),
        prior_offsety_class=np.zeros(K), sigma2_offset=float(w.offset_range) ** 2 / 4.0,
    )
    truth = dict(cls=cls, psi=psi, sx=sx, sy=sy, defocus_u=du, defocus_v=dv, defocus_angle=da)
    return pool, proj, r_max, truth


def raw_particles(p: Map2dPool, truth: dict, first_image: int = 0, dtype=np.float32):
    """The pool's particles as read from an MRC stack: real-space images
    (float32) whose centred transform is the pool's unmasked spectra, with
    the metadata the image preparation reads (NORM 1, old offsets 0, the
    CTF parameters the spectra were made with)."""
    from .particles import ParticleImages, images_from_spectra
    N = p.nr_images
    imgs = images_from_spectra(p.Fimg_nomask_real, p.Fimg_nomask_imag, p.current_size, p.ori_size, dtype)
    ctf = np.zeros((N, 7))
    ctf[:, 0], ctf[:, 1], ctf[:, 2] = truth["defocus_u"], truth["defocus_v"], truth["defocus_angle"]
    ctf[:, 3:7] = [300.0, 2.7, 0.1, 0.0]
    return ParticleImages(images=imgs, norm=np.ones(N), xoff=np.zeros(N), yoff=np.zeros(N), ctf=ctf,
                          group=np.asarray(p.group, np.int32), first_image=first_image)


def prep_options(w: Map2dWorkload):
    """Preparation settings of a synthetic workload: a particle diameter of
    0.84 of the box (the templates' blobs lie within 0.3 of it, plus their
    width and the shifts), the reference's 5-pixel soft edge, noise outside."""
    from .particles import PrepOptions
    return PrepOptions(pixel_size=w.pixel, particle_diameter=0.84 * w.ori_size * w.pixel, width_mask_edge=5,
                       random_seed=int(w.seed))


def image_template(p: Map2dPool) -> Map2dPool:
    """The pool without its image arrays (zero-width placeholders): the model,
    sampling and per-particle scalars that prepared pools are made from."""
    from .map2d import DEVICE_FIELDS
    return dataclasses.replace(p, **{f: np.empty((p.nr_images, 0)) for f in DEVICE_FIELDS})


def slice_particles(imgs, lo: int, hi: int):
    """Particles [lo, hi) of a ParticleImages (first_image moves with lo)."""
    import dataclasses as dc
    return dc.replace(imgs, images=imgs.images[lo:hi], norm=imgs.norm[lo:hi], xoff=imgs.xoff[lo:hi],
                      yoff=imgs.yoff[lo:hi], ctf=imgs.ctf[lo:hi], group=imgs.group[lo:hi],
                      first_image=imgs.first_image + lo)


# ---------------------------------------------------------------------------
# 3D: random-blob volumes, Fourier-slice particles, HEALPix sampling


@dataclasses.dataclass
class Map3dWorkload:
    n_particles: int = 1000
    ori_size: int = 32
    current_size: Optional[int] = None  # default: ori_size
    coarse_size: Optional[int] = None   # default: current_size / 2 (even, >= 12)
    n_classes: int = 2
    n_blobs: int = 30
    blob_sigma: tuple = (1.5, 4.0)
    healpix_order: int = 1
    offset_range: int = 2
    offset_step: int = 1
    max_shift: float = 2.0
    pixel: float = 2.0
    snr: float = 0.1
    defocus: tuple = (10000.0, 30000.0)
    seed: int = 1
    random_perturbation: float = 0.0
    particle_seed: Optional[int] = None
    # uneven noise: per-particle SNR log-uniform in snr_range (when set), and noisy_fraction of the
    # particles with noisy_factor (range) times the noise amplitude on top
    snr_range: Optional[tuple] = None
    noisy_fraction: float = 0.0
    noisy_factor: tuple = (2.0, 4.0)
    # distinct particles generated; the rest repeat them in order (0: all distinct)
    unique_particles: int = 0


def blob_volumes(rng, ori, K, n_blobs, sig):
    """K volumes ori^3, each a sum of n_blobs Gaussian blobs inside 0.3 ori of the centre."""
    c = np.arange(ori) - ori // 2
    zz, yy, xx = np.meshgrid(c, c, c, indexing="ij")
    vols = np.zeros((K, ori, ori, ori))
    for k in range(K):
        u = rng.normal(size=(n_blobs, 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        r = 0.3 * ori * np.cbrt(rng.uniform(0, 1, n_blobs))
        ctr = u * r[:, None]
        s = rng.uniform(sig[0], sig[1], n_blobs)
        a = rng.uniform(0.5, 1.0, n_blobs)
        for q in range(n_blobs):
            d2 = (xx - ctr[q, 0]) ** 2 + (yy - ctr[q, 1]) ** 2 + (zz - ctr[q, 2]) ** 2
            vols[k] += a[q] * np.exp(-d2 / (2 * s[q] ** 2))
    return vols


def projector_map_3d(vol: np.ndarray, current_size: int, padding: int = 2):
    """MyProjector::computeFourierTransformMap for a 3D reference
    (src/reconstruct.cpp:106-223), as projector_map_2d: gridding correction,
    zero padding by 2, centred FFT, windowed to r_max.  Returns
    (data [pad][pad][pad/2+1][2], r_max, pad_size)."""
    ori = vol.shape[0]
    r_max = min(current_size // 2, ori // 2)
    pad_size = 2 * (padding * r_max + 1) + 1
    padF = pad_size // 2 + 1
    c = np.arange(ori) - ori // 2
    zz, yy, xx = np.meshgrid(c, c, c, indexing="ij")
    r = np.sqrt(xx * xx + yy * yy + zz * zz)
    rval = r / (ori * padding)
    sinc = np.where(r > 0, np.sin(np.pi * rval) / np.where(r > 0, np.pi * rval, 1.0), 1.0)
    P = padding * ori
    Mpad = np.zeros((P, P, P))
    o = P // 2 - ori // 2
    Mpad[o:o + ori, o:o + ori, o:o + ori] = vol / (sinc * sinc)
    F = np.fft.rfftn(np.fft.ifftshift(Mpad)) / (P * P * P) * padding ** 3
    hP = P // 2 + 1
    ip = np.where(np.arange(P) < hP, np.arange(P), np.arange(P) - P)
    kz, ky, kx = np.meshgrid(ip, ip, np.arange(hP), indexing="ij")
    ok = (kz * kz + ky * ky + kx * kx <= (r_max * padding) ** 2) & (np.abs(kz) <= pad_size // 2) & (
        np.abs(ky) <= pad_size // 2) & (kx < padF)
    data = np.zeros((pad_size, pad_size, padF, 2))
    zi, yi, xi = kz[ok] + pad_size // 2, ky[ok] + pad_size // 2, kx[ok]
    data[zi, yi, xi, 0] = F[ok].real
    data[zi, yi, xi, 1] = F[ok].imag
    return data, r_max, pad_size


def project3d_np(data: np.ndarray, r_max: int, angles: np.ndarray, size: int, padding: int = 2) -> np.ndarray:
    """MyProjector::project, trilinear (src/reconstruct.cpp:226-410), for many
    (rot, tilt, psi) at once; returns complex [n][size][size/2+1]."""
    from .sampling import euler_matrix
    pad = data.shape[0]
    Fs = size // 2 + 1
    my_r = min(r_max, size // 2)
    rows = np.arange(size)
    yv = np.where(rows <= my_r, rows, rows - size)
    rowok = (rows <= my_r) | (rows >= size - my_r)
    yy, xx = np.meshgrid(yv, np.arange(Fs), indexing="ij")
    ok = rowok[:, None] & (xx <= my_r) & (xx * xx + yy * yy <= my_r * my_r)
    ys, xs = yy[ok].astype(np.float64), xx[ok].astype(np.float64)
    A = np.stack([euler_matrix(*a) for a in np.atleast_2d(angles)]) * padding  # [n][3][3]
    xp = A[:, 0, 0, None] * xs + A[:, 1, 0, None] * ys
    yp = A[:, 0, 1, None] * xs + A[:, 1, 1, None] * ys
    zp = A[:, 0, 2, None] * xs + A[:, 1, 2, None] * ys
    neg = xp < 0
    xp, yp, zp = np.where(neg, -xp, xp), np.where(neg, -yp, yp), np.where(neg, -zp, zp)
    x0 = np.floor(xp).astype(np.int64)
    y0 = np.floor(yp).astype(np.int64)
    z0 = np.floor(zp).astype(np.int64)
    fx, fy, fz = xp - x0, yp - y0, zp - z0
    y0 += pad // 2
    z0 += pad // 2
    cplx = data[..., 0] + 1j * data[..., 1]
    lerp = lambda a, lo, hi: lo + (hi - lo) * a  # noqa: E731
    c00 = lerp(fx, cplx[z0, y0, x0], cplx[z0, y0, x0 + 1])
    c01 = lerp(fx, cplx[z0 + 1, y0, x0], cplx[z0 + 1, y0, x0 + 1])
    c10 = lerp(fx, cplx[z0, y0 + 1, x0], cplx[z0, y0 + 1, x0 + 1])
    c11 = lerp(fx, cplx[z0 + 1, y0 + 1, x0], cplx[z0 + 1, y0 + 1, x0 + 1])
    v = lerp(fz, lerp(fy, c00, c10), lerp(fy, c01, c11))
    v = np.where(neg, np.conj(v), v)
    out = np.zeros((A.shape[0], size, Fs), np.complex128)
    out[:, ok] = v
    return out


def build_map3d(w: Map3dWorkload):
    """Returns (Map3dPool for all particles, projector data [K][pad][pad][padF][2],
    r_max, truth dict).  Sampling: HEALPix order w.healpix_order with
    adaptive oversampling 1 (rome_b200.sampling, the reference's sampler)."""
    from .map3d import Map3dPool
    from .sampling import oversampled_orientations_3d, oversampled_translations
    rng = np.random.default_rng(w.seed)
    ori = w.ori_size
    cur = w.current_size or ori
    cs = w.coarse_size or max(12, (cur // 2) // 2 * 2)
    K = w.n_classes
    vols = blob_volumes(rng, ori, K, w.n_blobs, w.blob_sigma)
    proj = []
    for k in range(K):
        d, r_max, pad = projector_map_3d(vols[k], cur)
        proj.append(d)
    proj = np.stack(proj)
    if w.particle_seed is not None:
        rng = np.random.default_rng(w.particle_seed)
    N_all = w.n_particles
    N = min(N_all, w.unique_particles) if w.unique_particles else N_all
    Fs = cur // 2 + 1
    cls = rng.integers(0, K, N)
    rot = rng.uniform(0.0, 360.0, N)
    tilt = np.rad2deg(np.arccos(rng.uniform(-1.0, 1.0, N)))
    psi = rng.uniform(0.0, 360.0, N)
    sx = rng.uniform(-w.max_shift, w.max_shift, N)
    sy = rng.uniform(-w.max_shift, w.max_shift, N)
    du = rng.uniform(*w.defocus, N)
    dv = rng.uniform(*w.defocus, N)
    da = rng.uniform(0, 180, N)
    rows = np.arange(cur)
    ky = np.where(rows < Fs, rows, rows - cur).astype(np.float64)[:, None]
    kx = np.arange(Fs, dtype=np.float64)[None, :]
    Fr = np.zeros((N, cur * Fs))
    Fi = np.zeros((N, cur * Fs))
    ctf = np.zeros((N, cur * Fs))
    mres = mresol(cur)
    sig_all = []
    chunk = 64
    for c0 in range(0, N, chunk):
        c1 = min(N, c0 + chunk)
        for k in np.unique(cls[c0:c1]):
            idx = np.nonzero(cls[c0:c1] == k)[0] + c0
            Pk = project3d_np(proj[k], r_max, np.stack([rot[idx], tilt[idx], psi[idx]], axis=1), cur)
            for q, i in enumerate(idx):
                c = ctf_image(cur, ori, w.pixel, du[i], dv[i], da[i], 300.0, 2.7, 0.1)
                ph = np.exp(2j * np.pi * (kx * sx[i] + ky * sy[i]) / ori)
                s = Pk[q] * ph * c
                Fr[i] = s.real.reshape(-1)
                Fi[i] = s.imag.reshape(-1)
                ctf[i] = c.reshape(-1)
                sig_all.append(np.mean(np.abs(s.reshape(-1)[mres > 0]) ** 2))
    sig_pow = float(np.mean(sig_all))
    sigma2 = sig_pow / (2.0 * w.snr)  # the model's noise power at the configured SNR
    amp = np.ones(N)
    if w.snr_range is not None:
        lo, hi = np.log(w.snr_range[0]), np.log(w.snr_range[1])
        amp *= np.sqrt(w.snr / np.exp(rng.uniform(lo, hi, N)))
    if w.noisy_fraction > 0:
        noisy = rng.uniform(0, 1, N) < w.noisy_fraction
        amp *= np.where(noisy, rng.uniform(w.noisy_factor[0], w.noisy_factor[1], N), 1.0)
    Fr += rng.normal(0, math.sqrt(sigma2), Fr.shape) * amp[:, None]
    Fi += rng.normal(0, math.sqrt(sigma2), Fi.shape) * amp[:, None]
    Fr[:, 0] = 0.0
    Fi[:, 0] = 0.0
    # uneven noise: the particles are grouped by noise level (8 log-spaced bins of the amplitude), each
    # group with its own noise power in the model, as the reference estimates sigma2_noise per group
    if w.snr_range is not None or w.noisy_fraction > 0:
        edges = np.exp(np.linspace(np.log(amp.min()), np.log(amp.max()) + 1e-9, 9))
        group = np.clip(np.searchsorted(edges, amp, side="right") - 1, 0, 7).astype(np.int32)
        gamp = np.array([np.exp(np.mean(np.log(amp[group == g]))) if np.any(group == g) else 1.0 for g in range(8)])
        sigma2_groups = sigma2 * gamp ** 2
    else:
        group = np.zeros(N, np.int32)
        sigma2_groups = np.array([sigma2])
    if N < N_all:
        # the remaining particles repeat the distinct ones in order (the E-step's work per particle
        # does not depend on which particle it is)
        rep = np.arange(N_all) % N
        Fr, Fi, ctf, group = Fr[rep], Fi[rep], ctf[rep], group[rep]
        cls, rot, tilt, psi, sx, sy, du, dv, da = (a[rep] for a in (cls, rot, tilt, psi, sx, sy, du, dv, da))
        N = N_all
    oriF = ori // 2 + 1
    tx, ty = translations(w.offset_range, w.offset_step)
    rp = w.random_perturbation
    angles = [oversampled_orientations_3d(w.healpix_order, o, rp) for o in (0, 1)]
    otr = [oversampled_translations(tx, ty, float(w.offset_step), o, rp) for o in (0, 1)]
    ndir = angles[0].shape[0]
    pool = Map3dPool(
        ori_size=ori, current_size=cur, coarse_size=cs, nr_classes=K, nr_groups=len(sigma2_groups), nr_dir=ndir,
        angles=angles, over_trans_x=[otr[0][0], otr[1][0]], over_trans_y=[otr[0][1], otr[1][1]], trans_x=tx,
        trans_y=ty, Fimg_real=Fr, Fimg_imag=Fi, Fimg_nomask_real=Fr.copy(), Fimg_nomask_imag=Fi.copy(), Fctf=ctf,
        highres_Xi2=np.zeros(N), old_offsetx=np.zeros(N), old_offsety=np.zeros(N), group=group,
        sigma2_noise=np.repeat(sigma2_groups[:, None], oriF, axis=1), Mresol_fine=mres, Mresol_coarse=mresol(cs),
        pdf_class=np.full(K, 1.0 / K), pdf_direction=np.full((K, ndir), 1.0 / ndir),
        prior_offsetx_class=np.zeros(K), prior_offsety_class=np.zeros(K),
        sigma2_offset=float(w.offset_range) ** 2 / 4.0, adaptive_oversampling=1)
    truth = dict(cls=cls, rot=rot, tilt=tilt, psi=psi, sx=sx, sy=sy, defocus_u=du, defocus_v=dv, defocus_angle=da)
    return pool, proj, r_max, truth


def subset3d(p, lo: int, hi: int):
    """The particles [lo, hi) of a 3D pool."""
    q = dataclasses.replace(p)
    for name in ["Fimg_real", "Fimg_imag", "Fimg_nomask_real", "Fimg_nomask_imag", "Fctf", "highres_Xi2",
                 "old_offsetx", "old_offsety", "group"]:
        setattr(q, name, np.ascontiguousarray(getattr(p, name)[lo:hi]))
    if getattr(p, "proposals", None) is not None:
        q.proposals = np.ascontiguousarray(p.proposals[lo:hi])
    return q


def subset(p: Map2dPool, lo: int, hi: int) -> Map2dPool:
    """The particles [lo, hi) of a pool (same model and sampling)."""
    q = dataclasses.replace(p)
    for name in ["Fimg_real", "Fimg_imag", "Fimg_nomask_real", "Fimg_nomask_imag", "Fctf", "highres_Xi2",
                 "old_offsetx", "old_offsety", "group"]:
        setattr(q, name, np.ascontiguousarray(getattr(p, name)[lo:hi]))
    if p.proposals is not None:
        q.proposals = np.ascontiguousarray(p.proposals[lo:hi])
    return q


# the benchmark configurations (BASELINE configs 1 and 2)
CONFIGS = {
    "map2d_cfg1": Map2dWorkload(n_particles=1000, ori_size=64, n_classes=10, n_blobs=20, psi_step=10.0,
                                offset_range=5, offset_step=1, max_shift=4.0, pixel=2.0, snr=0.05, seed=1),
    "map2d_cfg2": Map2dWorkload(n_particles=20000, ori_size=128, n_classes=50, n_blobs=40, psi_step=5.0,
                                offset_range=6, offset_step=2, max_shift=6.0, pixel=1.5, snr=0.03, seed=2),
    # MAP3D: 10,000 particles of 128^2 from K=4 blob volumes (60 blobs, sigma 2-8 voxels), HEALPix order 2
    # (192 directions x 24 coarse psi), +-4 px step 2 (13 translations), adaptive oversampling 1; coarse
    # size 20 as the reference's formula gives for these images (map_model.cpp:505-520)
    # Batched uneven MAP3D: 50,000 particles of 128^2 (10,000 distinct, repeated) from K=8 blob volumes,
    # HEALPix order 3 (768 directions x 48 coarse psi, coarse size 40), +-4 px step 2, oversampling 1;
    # per-particle SNR log-uniform over a decade and 30% of the particles with 2-4x the noise amplitude,
    # noise power per noise-level group, so the number of coarse-significant points varies widely.  The
    # SNR here is per Fourier component of the CTF-modulated projection; the decade [0.01, 0.1] on that
    # scale leaves the noisiest particles nearly uninformative (significant over most of the 3.8 M coarse
    # hypotheses, tens of thousands of coarse orientations for one particle), so the decade is
    # [0.06, 0.6], which puts the largest counts at a few thousand
    "map3d_cfg4": Map3dWorkload(n_particles=50000, ori_size=128, coarse_size=40, n_classes=8, n_blobs=60,
                                blob_sigma=(2.0, 8.0), healpix_order=3, offset_range=4, offset_step=2, max_shift=4.0,
                                pixel=1.5, snr=0.19, seed=4, snr_range=(0.06, 0.6), noisy_fraction=0.3,
                                noisy_factor=(2.0, 4.0), unique_particles=10000),
    "map3d_cfg3": Map3dWorkload(n_particles=10000, ori_size=128, coarse_size=20, n_classes=4, n_blobs=60,
                                blob_sigma=(2.0, 8.0), healpix_order=2, offset_range=4, offset_step=2, max_shift=4.0,
                                pixel=1.5, snr=0.05, seed=3),
}
