"""Host-side mirror of the particle image preparation
(ParticleModel::setFourierTransforms, src/exp_model.h:397-640).

`ParticleImages` carries what the reference reads for one pool -- the images
as read and the metadata fields NORM, XOFF/YOFF, the CTF parameters and the
group -- and `PrepOptions` the optimizer settings the preparation uses.
`prepare_particles` runs it on the device through the C ABI
(``rome_gpu_prepare_particles``); `prepared_pool` hands the result to the
E-step without it leaving the device.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Dict, Optional

import numpy as np

from . import abi
from .map2d import DEVICE_FIELDS, GpuContext, Map2dPool, StagedPool, _f64, _i32

__all__ = ["ParticleImages", "PrepOptions", "prepare_particles", "prepared_pool", "images_from_spectra",
           "CTF_FIELDS"]

#: columns of ParticleImages.ctf (MetaDataElem CTF_* fields, src/metadata.h)
CTF_FIELDS = ("defocus_u", "defocus_v", "defocus_angle", "voltage", "cs", "q0", "bfac")


@dataclasses.dataclass
class ParticleImages:
    """One pool of particles as read: exp_images and exp_metadata."""
    images: object             # [P][ori][ori] float32 / float64: numpy (host) or a torch CUDA tensor
    norm: np.ndarray           # NORM [P]
    xoff: np.ndarray           # XOFF, YOFF [P] (old offsets, rounded by the preparation)
    yoff: np.ndarray
    ctf: np.ndarray            # [P][7] in CTF_FIELDS order
    group: np.ndarray          # GROUP_NO - 1 [P]
    first_image: int = 0       # exp_first_image (seeds the noise)

    @property
    def nr_images(self) -> int:
        return int(self.images.shape[0])

    @property
    def ori_size(self) -> int:
        return int(self.images.shape[-1])


@dataclasses.dataclass
class PrepOptions:
    """The settings setFourierTransforms reads from the optimizer and model."""
    pixel_size: float
    particle_diameter: float
    width_mask_edge: int = 5
    sigma2_fudge: float = 1.0
    random_seed: int = 33
    avg_norm_correction: float = 1.0
    do_norm_correction: bool = False
    do_zero_mask: bool = False
    do_ctf_correction: bool = True
    ctf_phase_flipped: bool = False
    only_flip_phases: bool = False
    intact_ctf_first_peak: bool = False


def prepare_particles(ctx: GpuContext, imgs: ParticleImages, opts: PrepOptions, sigma2_noise: np.ndarray,
                      current_size: int, on_device: bool = False, power: bool = True) -> Dict[str, object]:
    """setFourierTransforms of one pool.  Returns Fimg_real/imag,
    Fimg_nomask_real/imag and Fctf ([P][F] numpy arrays, or torch CUDA
    tensors when on_device), highres_Xi2, old_offsetx/y ([P]) and, with
    `power`, power_imgs ([P][ori/2+1])."""
    P, ori = imgs.nr_images, imgs.ori_size
    F = current_size * (current_size // 2 + 1)
    sigma2_noise = _f64(sigma2_noise)
    keep = []

    def d(a):
        a = _f64(a)
        keep.append(a)
        return abi.dptr(a)

    s = abi.RomePrepIn()
    s.nr_images, s.ori_size, s.current_size = P, ori, current_size
    s.nr_groups = int(sigma2_noise.shape[0])
    s.first_image = int(imgs.first_image)
    im = imgs.images
    if hasattr(im, "data_ptr"):  # torch tensor
        import torch
        if not (im.is_cuda and im.is_contiguous() and im.dtype in (torch.float32, torch.float64)):
            raise TypeError("device images: a contiguous float32 or float64 CUDA tensor")
        s.images, s.images_on_device = C.c_void_p(im.data_ptr()), 1
        s.image_type = 1 if im.dtype == torch.float32 else 0
        torch.cuda.current_stream(im.device).synchronize()
    else:
        im = np.ascontiguousarray(im)
        if im.dtype not in (np.float32, np.float64):
            raise TypeError(f"images: float32 or float64, got {im.dtype}")
        keep.append(im)
        s.images, s.images_on_device = C.c_void_p(im.ctypes.data), 0
        s.image_type = 1 if im.dtype == np.float32 else 0
    s.norm, s.xoff, s.yoff = d(imgs.norm), d(imgs.xoff), d(imgs.yoff)
    ctf = _f64(imgs.ctf).reshape(P, len(CTF_FIELDS))
    for k, name in enumerate(CTF_FIELDS):
        setattr(s, "ctf_" + name, d(ctf[:, k]))
    grp = _i32(imgs.group)
    keep.append(grp)
    s.group = abi.iptr(grp)
    s.sigma2_noise = abi.dptr(sigma2_noise)
    for name in ("avg_norm_correction", "pixel_size", "particle_diameter", "sigma2_fudge"):
        setattr(s, name, float(getattr(opts, name)))
    s.width_mask_edge, s.random_seed = int(opts.width_mask_edge), int(opts.random_seed)
    for name in ("do_norm_correction", "do_zero_mask", "do_ctf_correction", "ctf_phase_flipped", "only_flip_phases",
                 "intact_ctf_first_peak"):
        setattr(s, name, int(bool(getattr(opts, name))))

    o: Dict[str, object] = {}
    so = abi.RomePrepOut()
    if on_device:
        import torch
        for name in DEVICE_FIELDS:
            t = torch.empty((P, F), dtype=torch.float64, device=f"cuda:{ctx.device}")
            o[name] = t
            setattr(so, name, C.cast(C.c_void_p(t.data_ptr()), abi._DP))
        so.outputs_on_device = 1
    else:
        for name in DEVICE_FIELDS:
            o[name] = np.zeros((P, F), np.float64)
            setattr(so, name, abi.dptr(o[name]))
    for name in ("highres_Xi2", "old_offsetx", "old_offsety"):
        o[name] = np.zeros(P, np.float64)
        setattr(so, name, abi.dptr(o[name]))
    if power:
        o["power_imgs"] = np.zeros((P, ori // 2 + 1), np.float64)
        so.power_imgs = abi.dptr(o["power_imgs"])
    ctx._check(ctx.lib.rome_gpu_prepare_particles(ctx.h, C.byref(s), C.byref(so)))
    return o


def prepared_pool(ctx: GpuContext, template: Map2dPool, imgs: ParticleImages, opts: PrepOptions,
                  power: bool = False) -> StagedPool:
    """The E-step input of a pool prepared on the device: `template`'s model
    and sampling with this pool's particles, the images left on the device
    (a StagedPool for GpuContext.map2d_estep_pool and the learned E-step, or,
    with a Map3dPool template, for map3d.map3d_estep_pool(ctx, sp.pool,
    dev=sp.dev))."""
    o = prepare_particles(ctx, imgs, opts, template.sigma2_noise, template.current_size, on_device=True, power=power)
    P = imgs.nr_images
    rep = {name: np.empty((P, 0)) for name in DEVICE_FIELDS}
    rep.update(highres_Xi2=o["highres_Xi2"], old_offsetx=o["old_offsetx"], old_offsety=o["old_offsety"],
               group=_i32(imgs.group), proposals=None)
    if hasattr(template, "particle_rows"):  # MAP2D pools only
        rep["particle_rows"] = None
    pool = dataclasses.replace(template, **rep)
    sp = StagedPool(pool, {name: o[name] for name in DEVICE_FIELDS})
    if power:
        sp.power_imgs = o["power_imgs"]
    return sp


def images_from_spectra(F_real: np.ndarray, F_imag: np.ndarray, current_size: int, ori_size: int,
                        dtype=np.float32) -> np.ndarray:
    """Real-space images [P][ori][ori] whose normalised, centred transform
    (before any mask) is the given half-plane spectra [P][cur*(cur/2+1)]
    (cur = current_size <= ori; the frequencies above cur are zero): the
    inverse of the preparation's unmasked path, for synthetic raw images."""
    P, n, cur = F_real.shape[0], ori_size, current_size
    cF, oF = cur // 2 + 1, n // 2 + 1
    full = np.zeros((P, n, oF), np.complex128)
    Fc = (np.asarray(F_real) + 1j * np.asarray(F_imag)).reshape(P, cur, cF)
    for i in range(cur):
        ip = i if i < cF else i - cur
        full[:, ip % n, :cF] = Fc[:, i, :]
    img = np.fft.irfft2(full * (n * n), s=(n, n), axes=(1, 2))
    img = np.roll(img, (-(n // 2), -(n // 2)), axis=(1, 2))
    return np.ascontiguousarray(img.astype(dtype))


def pin_particles(imgs: ParticleImages) -> ParticleImages:
    """The images copied into page-locked host memory (what prepared_stream
    copies to the device asynchronously)."""
    import torch
    t = torch.empty(tuple(imgs.images.shape), dtype=torch.from_numpy(np.asarray(imgs.images[:0])).dtype,
                    pin_memory=True)
    t.numpy()[...] = imgs.images
    return dataclasses.replace(imgs, images=t.numpy())


def prepared_stream(prep_ctx: GpuContext, items, opts: PrepOptions, power: bool = False):
    """Yield a prepared StagedPool for each (template Map2dPool, ParticleImages
    with page-locked host images) of `items`: the images of item k + 1 are
    copied to the device on a side stream while item k is prepared, and the
    preparation runs on `prep_ctx` (a context of its own, so the caller's
    E-step contexts keep computing the previous pools meanwhile)."""
    import torch
    side = getattr(prep_ctx, "_side", None)
    if side is None:
        side = prep_ctx._side = torch.cuda.Stream(device=prep_ctx.device)
    dev = f"cuda:{prep_ctx.device}"

    def upload(imgs):
        with torch.cuda.stream(side):
            t = torch.from_numpy(np.asarray(imgs.images)).to(dev, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(side)
        return t, ev

    items = list(items)
    nxt = upload(items[0][1]) if items else None
    for q, (template, imgs) in enumerate(items):
        t, ev = nxt
        if q + 1 < len(items):
            nxt = upload(items[q + 1][1])
        ev.synchronize()
        yield prepared_pool(prep_ctx, template, dataclasses.replace(imgs, images=t), opts, power=power)
        del t


def h2d_bytes(imgs: ParticleImages) -> int:
    """Bytes a preparation call copies to the device: the images and the
    per-particle metadata (NORM, offsets, 7 CTF parameters, group)."""
    return int(np.asarray(imgs.images).nbytes) + imgs.nr_images * (10 * 8 + 4)
