"""Seeded synthetic cryo-EM particle stacks for the MAP hot path.

The reference ships no datasets (its ``src/simulatedata.h`` is an empty stub),
so every workload is generated here: class templates built from random 2D or
3D Gaussian blobs, random poses, a CTF per particle and additive white noise
at a target SNR.  Files are written in the layouts the reference reads:

* MRCS stacks: 1024-byte header, float32 images (``src/map2d_optimizer.cpp:150``
  seeks to ``(256 + (index-1) * ori_size^2) * 4``; header fields
  ``src/mrcs.h:50-80``).
* STAR metadata with the ``_rln`` labels ``src/metadata.h:55-107`` parses.

The CTF uses the reference's formula (``src/ctf.cpp:136-171``, ``src/ctf.h:151-204``)
so the generated data is consistent with the model the E-step evaluates.
"""
from __future__ import annotations

import dataclasses
import os
from typing import List, Optional, Sequence

import numpy as np

__all__ = [
    "Map2dSpec",
    "ctf_image",
    "make_templates_2d",
    "make_particles_2d",
    "write_mrcs",
    "write_star",
    "write_dataset_2d",
    "Map3dSpec",
    "euler_matrix",
    "make_volumes_3d",
    "render_volume",
    "make_particles_3d",
    "write_dataset_3d",
]


@dataclasses.dataclass
class Map2dSpec:
    n_particles: int = 1000
    size: int = 64
    n_classes: int = 10
    n_blobs: int = 20
    blob_sigma: Sequence[float] = (2.0, 6.0)
    max_shift: float = 4.0
    defocus: Sequence[float] = (10000.0, 30000.0)  # Angstrom (1.0-3.0 um)
    voltage: float = 300.0
    cs: float = 2.7
    q0: float = 0.1
    pixel: float = 2.0
    snr: float = 0.05
    seed: int = 1


def ctf_image(size: int, ori_size: int, angpix: float, def_u: float, def_v: float, def_angle: float,
              voltage: float, cs: float, q0: float, bfac: float = 0.0) -> np.ndarray:
    """CTF in FFTW half-plane layout ``[size][size//2+1]``.

    Restates ``CTF::initialise`` (ctf.cpp:136-171), ``CTF::getCTF``/``getDeltaF``
    (ctf.h:151-204) and ``CTF::getFftwImage`` (ctf.cpp:173-191) with damping on.
    """
    local_cs = cs * 1e7
    local_kv = voltage * 1e3
    rad_az = np.deg2rad(def_angle)
    defocus_average = -(def_u + def_v) * 0.5
    defocus_deviation = -(def_u - def_v) * 0.5
    lam = 12.2643247 / np.sqrt(local_kv * (1.0 + local_kv * 0.978466e-6))
    k1 = np.pi / 2 * 2 * lam
    k2 = np.pi / 2 * local_cs * lam ** 3
    k3 = np.sqrt(1 - q0 * q0)
    k4 = -bfac / 4.0
    hdim = size // 2 + 1
    i = np.arange(size)
    ip = np.where(i < hdim, i, i - size).astype(np.float64)
    jp = np.arange(hdim, dtype=np.float64)
    xs = ori_size * angpix
    X = jp[None, :] / xs
    Y = ip[:, None] / xs
    u2 = X * X + Y * Y
    u4 = u2 * u2
    ang = np.arctan2(Y, X) - rad_az
    deltaf = defocus_average + defocus_deviation * np.cos(2 * ang)
    deltaf = np.where((np.abs(X) < 1e-8) & (np.abs(Y) < 1e-8), 0.0, deltaf)
    arg = k1 * deltaf * u2 + k2 * u4
    ret = -(k3 * np.sin(arg) - q0 * np.cos(arg))
    ret = ret * np.exp(k4 * u2)
    return ret


def _render_blobs_2d(size: int, centers: np.ndarray, sigmas: np.ndarray, amps: np.ndarray) -> np.ndarray:
    c = np.arange(size) - size // 2
    yy, xx = np.meshgrid(c, c, indexing="ij")
    img = np.zeros((size, size), np.float64)
    for (cx, cy), s, a in zip(centers, sigmas, amps):
        img += a * np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2 * s * s))
    return img


def make_templates_2d(rng: np.random.Generator, spec: Map2dSpec) -> List[dict]:
    """K templates, each a sum of ``n_blobs`` Gaussian blobs inside the particle disc."""
    out = []
    radius = 0.3 * spec.size
    for _ in range(spec.n_classes):
        r = radius * np.sqrt(rng.uniform(0, 1, spec.n_blobs))
        t = rng.uniform(0, 2 * np.pi, spec.n_blobs)
        centers = np.stack([r * np.cos(t), r * np.sin(t)], axis=1)
        sigmas = rng.uniform(spec.blob_sigma[0], spec.blob_sigma[1], spec.n_blobs)
        amps = rng.uniform(0.5, 1.0, spec.n_blobs)
        out.append(dict(centers=centers, sigmas=sigmas, amps=amps))
    return out


def make_particles_2d(spec: Map2dSpec, templates: Optional[List[dict]] = None):
    """Render particles: template class k, rotated by psi, shifted, CTF-modulated, noisy.

    Returns (images float32 [N][S][S], metadata dict of per-particle arrays).
    """
    rng = np.random.default_rng(spec.seed)
    if templates is None:
        templates = make_templates_2d(rng, spec)
    n, s = spec.n_particles, spec.size
    cls = rng.integers(0, spec.n_classes, n)
    psi = rng.uniform(0.0, 360.0, n)
    shx = rng.uniform(-spec.max_shift, spec.max_shift, n)
    shy = rng.uniform(-spec.max_shift, spec.max_shift, n)
    du = rng.uniform(spec.defocus[0], spec.defocus[1], n)
    dv = rng.uniform(spec.defocus[0], spec.defocus[1], n)
    dang = rng.uniform(0.0, 180.0, n)
    imgs = np.empty((n, s, s), np.float32)
    # signal variance is measured inside the particle disc
    c = np.arange(s) - s // 2
    yy, xx = np.meshgrid(c, c, indexing="ij")
    disc = (xx * xx + yy * yy) <= (0.45 * s) ** 2
    for p in range(n):
        t = templates[cls[p]]
        a = np.deg2rad(psi[p])
        rot = np.array([[np.cos(a), -np.sin(a)], [np.sin(a), np.cos(a)]])
        cen = t["centers"] @ rot.T + np.array([shx[p], shy[p]])
        img = _render_blobs_2d(s, cen, t["sigmas"], t["amps"])
        F = np.fft.rfft2(np.fft.ifftshift(img))
        F *= ctf_image(s, s, spec.pixel, du[p], dv[p], dang[p], spec.voltage, spec.cs, spec.q0)
        sig = np.fft.fftshift(np.fft.irfft2(F, s=(s, s)))
        var = float(np.var(sig[disc]))
        sigma = np.sqrt(var / spec.snr) if var > 0 else 1.0
        noisy = sig + rng.normal(0.0, sigma, (s, s))
        # normalise the background like a real extraction (zero mean, unit std)
        noisy = (noisy - noisy[~disc].mean()) / max(noisy[~disc].std(), 1e-12)
        imgs[p] = noisy.astype(np.float32)
    meta = dict(cls=cls, psi=psi, shx=shx, shy=shy, du=du, dv=dv, dang=dang)
    return imgs, meta


def write_mrcs(path: str, stack: np.ndarray, angpix: float = 1.0) -> None:
    """Write a float32 image stack with a 1024-byte MRC header (mode 2)."""
    stack = np.ascontiguousarray(stack, dtype=np.float32)
    n, ny, nx = stack.shape
    hdr = np.zeros(256, np.int32)
    hdr[0], hdr[1], hdr[2], hdr[3] = nx, ny, n, 2
    hdr[7], hdr[8], hdr[9] = nx, ny, n
    fh = hdr.view(np.float32)
    fh[10], fh[11], fh[12] = nx * angpix, ny * angpix, n * angpix
    fh[13] = fh[14] = fh[15] = 90.0
    hdr[16], hdr[17], hdr[18] = 1, 2, 3
    fh[19], fh[20], fh[21] = stack.min(), stack.max(), stack.mean()
    hdr[52] = int.from_bytes(b"MAP ", "little")
    hdr[53] = 0x00004444
    with open(path, "wb") as f:
        f.write(hdr.tobytes())
        f.write(stack.tobytes())


def write_star(path: str, mrcs_path: str, meta: dict, voltage: float, cs: float, q0: float) -> None:
    n = len(meta["du"])
    labels = ["rlnImageName", "rlnMicrographName", "rlnDefocusU", "rlnDefocusV", "rlnDefocusAngle",
              "rlnVoltage", "rlnSphericalAberration", "rlnAmplitudeContrast", "rlnGroupNumber"]
    with open(path, "w") as f:
        f.write("\ndata_\n\nloop_\n")
        for i, lab in enumerate(labels):
            f.write(f"_{lab} #{i + 1}\n")
        for p in range(n):
            f.write(f"{p + 1:06d}@{mrcs_path} mic{p % 7:03d}.mrc {meta['du'][p]:.6f} {meta['dv'][p]:.6f} "
                    f"{meta['dang'][p]:.6f} {voltage:.6f} {cs:.6f} {q0:.6f} 1\n")


def write_dataset_2d(out_dir: str, spec: Map2dSpec, name: str = "particles") -> str:
    """Generate a 2D dataset; returns the STAR path (images referenced by absolute path)."""
    os.makedirs(out_dir, exist_ok=True)
    imgs, meta = make_particles_2d(spec)
    mrcs = os.path.abspath(os.path.join(out_dir, name + ".mrcs"))
    star = os.path.join(out_dir, name + ".star")
    write_mrcs(mrcs, imgs, spec.pixel)
    write_star(star, mrcs, meta, spec.voltage, spec.cs, spec.q0)
    np.savez(os.path.join(out_dir, name + "_truth.npz"), **meta)
    return star


# ---------------------------------------------------------------------------
# 3D: blob volumes, projections at uniform random orientations


@dataclasses.dataclass
class Map3dSpec:
    n_particles: int = 1000
    size: int = 64
    n_classes: int = 4
    n_blobs: int = 60
    blob_sigma: Sequence[float] = (2.0, 8.0)
    max_shift: float = 4.0
    defocus: Sequence[float] = (10000.0, 30000.0)
    voltage: float = 300.0
    cs: float = 2.7
    q0: float = 0.1
    pixel: float = 2.0
    snr: float = 0.05
    seed: int = 1


def euler_matrix(rot: float, tilt: float, psi: float) -> np.ndarray:
    """ZYZ Euler matrix in degrees, the convention of ``Euler_angles2matrix``
    (src/math.cpp:86-115)."""
    a, b, g = np.deg2rad([rot, tilt, psi])
    ca, cb, cg, sa, sb, sg = np.cos(a), np.cos(b), np.cos(g), np.sin(a), np.sin(b), np.sin(g)
    cc, cs, sc, ss = cb * ca, cb * sa, sb * ca, sb * sa
    return np.array([[cg * cc - sg * sa, cg * cs + sg * ca, -cg * sb],
                     [-sg * cc - cg * sa, -sg * cs + cg * ca, sg * sb],
                     [sc, ss, cb]])


def make_volumes_3d(rng: np.random.Generator, spec: Map3dSpec) -> List[dict]:
    """K volumes, each a sum of ``n_blobs`` isotropic Gaussian blobs inside the particle sphere."""
    out = []
    radius = 0.3 * spec.size
    for _ in range(spec.n_classes):
        v = rng.normal(size=(spec.n_blobs, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        r = radius * rng.uniform(0, 1, spec.n_blobs) ** (1.0 / 3.0)
        out.append(dict(centers=v * r[:, None],
                        sigmas=rng.uniform(spec.blob_sigma[0], spec.blob_sigma[1], spec.n_blobs),
                        amps=rng.uniform(0.5, 1.0, spec.n_blobs)))
    return out


def render_volume(size: int, vol: dict) -> np.ndarray:
    """Real-space volume [z][y][x], origin at size//2 (the reference's centre convention)."""
    c = np.arange(size) - size // 2
    zz, yy, xx = np.meshgrid(c, c, c, indexing="ij")
    out = np.zeros((size,) * 3, np.float64)
    for (cx, cy, cz), s, a in zip(vol["centers"], vol["sigmas"], vol["amps"]):
        out += a * np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2 + (zz - cz) ** 2) / (2 * s * s))
    return out


def _uniform_rotations(rng: np.random.Generator, n: int):
    """Orientations uniform on SO(3): rot, psi uniform, cos(tilt) uniform."""
    rot = rng.uniform(0.0, 360.0, n)
    tilt = np.rad2deg(np.arccos(rng.uniform(-1.0, 1.0, n)))
    psi = rng.uniform(0.0, 360.0, n)
    return rot, tilt, psi


def make_particles_3d(spec: Map3dSpec, volumes: Optional[List[dict]] = None):
    """Project class volumes at uniform random orientations, shift, CTF, noise.

    A Gaussian blob of width s projects to a 2D Gaussian of the same width
    with amplitude a*s*sqrt(2 pi) centred at (A c)_xy, which is the real-space
    counterpart of the Fourier slice the reference extracts with A^T
    (src/reconstruct.cpp:226-410), so projections are exact.
    """
    rng = np.random.default_rng(spec.seed)
    if volumes is None:
        volumes = make_volumes_3d(rng, spec)
    n, s = spec.n_particles, spec.size
    cls = rng.integers(0, spec.n_classes, n)
    rot, tilt, psi = _uniform_rotations(rng, n)
    shx = rng.uniform(-spec.max_shift, spec.max_shift, n)
    shy = rng.uniform(-spec.max_shift, spec.max_shift, n)
    du = rng.uniform(spec.defocus[0], spec.defocus[1], n)
    dv = rng.uniform(spec.defocus[0], spec.defocus[1], n)
    dang = rng.uniform(0.0, 180.0, n)
    imgs = np.empty((n, s, s), np.float32)
    c = np.arange(s) - s // 2
    yy, xx = np.meshgrid(c, c, indexing="ij")
    disc = (xx * xx + yy * yy) <= (0.45 * s) ** 2
    for p in range(n):
        v = volumes[cls[p]]
        A = euler_matrix(rot[p], tilt[p], psi[p])
        cen = (v["centers"] @ A.T)[:, :2] + np.array([shx[p], shy[p]])
        img = _render_blobs_2d(s, cen, v["sigmas"], v["amps"] * v["sigmas"] * np.sqrt(2 * np.pi))
        F = np.fft.rfft2(np.fft.ifftshift(img))
        F *= ctf_image(s, s, spec.pixel, du[p], dv[p], dang[p], spec.voltage, spec.cs, spec.q0)
        sig = np.fft.fftshift(np.fft.irfft2(F, s=(s, s)))
        var = float(np.var(sig[disc]))
        sigma = np.sqrt(var / spec.snr) if var > 0 else 1.0
        noisy = sig + rng.normal(0.0, sigma, (s, s))
        noisy = (noisy - noisy[~disc].mean()) / max(noisy[~disc].std(), 1e-12)
        imgs[p] = noisy.astype(np.float32)
    meta = dict(cls=cls, rot=rot, tilt=tilt, psi=psi, shx=shx, shy=shy, du=du, dv=dv, dang=dang)
    return imgs, meta, volumes


def write_dataset_3d(out_dir: str, spec: Map3dSpec, name: str = "particles", ref_lowpass_sigma: float = 2.0):
    """Generate a 3D dataset and a starting reference volume.

    Returns (STAR path, reference MRC path).  The reference is the average of
    the class volumes blurred by a Gaussian of ``ref_lowpass_sigma`` pixels
    (every class starts from it, as ``MAPModel::initializeRef`` does,
    src/map_model.cpp:56-84).
    """
    os.makedirs(out_dir, exist_ok=True)
    imgs, meta, volumes = make_particles_3d(spec)
    mrcs = os.path.abspath(os.path.join(out_dir, name + ".mrcs"))
    star = os.path.join(out_dir, name + ".star")
    write_mrcs(mrcs, imgs, spec.pixel)
    write_star(star, mrcs, meta, spec.voltage, spec.cs, spec.q0)
    blurred = []
    for v in volumes:
        b = dict(v)
        b["sigmas"] = np.sqrt(v["sigmas"] ** 2 + ref_lowpass_sigma ** 2)
        b["amps"] = v["amps"] * (v["sigmas"] / b["sigmas"]) ** 3
        blurred.append(render_volume(spec.size, b))
    ref = np.mean(blurred, axis=0)
    ref_path = os.path.abspath(os.path.join(out_dir, name + "_ref.mrc"))
    write_mrcs(ref_path, ref.astype(np.float32), spec.pixel)
    np.savez(os.path.join(out_dir, name + "_truth.npz"), **meta)
    return star, ref_path
