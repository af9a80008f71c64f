"""Reconstruction at known poses on the GPU: the reference's rome_reconstruct
(apps/rome_reconstruct.cpp:123-409).

    python -m rome_b200.reconstruct_poses -i particles.star -o recon -angpix 1.5 -ctf 1 -iter 10

For every particle of the STAR file (rlnAngleRot/Tilt/Psi and
rlnOriginX/Y required, as the reference asserts, :71-76): the transform of
the centred image (the device image preparation's unmasked transform at
current size = image size, with no old-offset translation and no norm
correction), shifted by the particle's origin with the reference's
tabulated phases, times its CTF image, back-projected with weight CTF^2
(`rome_gpu_backproject_images`); then the gridding-corrected
reconstruction without a prior (`rome_gpu_reconstruct` with do_map 0,
tau2_fudge 1, normalise 1 and `iter` Pipe-Menon iterations, the reference's
`backprojector.reconstruct(vol_out, nr_iters, false, 1., ...)`, :381).
Images stream from disk one pool at a time (`ParticleStack.device_pools`).

Differences from the reference app, all outside its working options:
a particle with an origin of exactly (0, 0) is back-projected unshifted (the
reference's loop skips the shift and back-projects the previous particle's
shifted spectrum, :222-226); `-angular_error`/`-shift_error` (random pose
noise), `-subtract`, `-fsc`, `-NN` and symmetry other than C1 are not
provided (the reference leaves -subtract and -fsc as TODO and asserts
-NN 0); r_max is capped at Nyquist.
"""
from __future__ import annotations

import argparse
import math
from typing import Optional

import numpy as np

from .map2d import GpuContext
from .particles import PrepOptions, prepare_particles
from .star_mrcs import ParticleStack

__all__ = ["reconstruct_from_star", "write_mrc"]

POSE_LABELS = ("rlnAngleRot", "rlnAngleTilt", "rlnAnglePsi", "rlnOriginX", "rlnOriginY")


def reconstruct_from_star(star_path: str, angpix: float, iters: int = 10, do_ctf: bool = False,
                          ctf_phase_flipped: bool = False, only_flip_phases: bool = False,
                          ctf_intact_first_peak: bool = False, maxres: float = -1.0, pool: int = 1000,
                          device: int = 0, ctx: Optional[GpuContext] = None) -> np.ndarray:
    """The reconstructed volume [ori][ori][ori] (FP64) of the particles of
    `star_path` at their recorded poses."""
    stack = ParticleStack(star_path)
    missing = [lab for lab in POSE_LABELS if lab not in stack.columns]
    if missing:
        raise ValueError(f"{star_path}: pose columns {missing} missing")
    poses = np.stack([np.asarray([float(v) for v in stack.columns[lab]]) for lab in POSE_LABELS], axis=1)
    ori = stack.ori_size
    oriF = ori // 2 + 1
    r_max = ori // 2 if maxres < 0 else min(ori // 2, int(math.ceil(ori * angpix / maxres)))
    pad = 2 * (2 * r_max + 1) + 1
    opts = PrepOptions(pixel_size=angpix, particle_diameter=ori * angpix, do_norm_correction=False,
                       do_ctf_correction=do_ctf, ctf_phase_flipped=ctf_phase_flipped,
                       only_flip_phases=only_flip_phases, intact_ctf_first_peak=ctf_intact_first_peak)
    sigma2 = np.ones((max(stack.nr_groups, 1), oriF))
    own = ctx is None
    if own:
        ctx = GpuContext(device, "fp32")
    try:
        ctx.set_projectors(np.zeros((1, pad, pad, pad // 2 + 1, 2)), ori, r_max)  # also zeroes the back-projector
        for imgs in stack.device_pools(ctx.device, pool):
            lo, hi = imgs.first_image, imgs.first_image + imgs.nr_images
            imgs.xoff[:] = 0.0   # the app translates in Fourier space only
            imgs.yoff[:] = 0.0
            out = prepare_particles(ctx, imgs, opts, sigma2, ori, on_device=True, power=False)
            ctx.backproject_images(0, out["Fimg_nomask_real"], out["Fimg_nomask_imag"],
                                   out["Fctf"] if do_ctf else None, poses[lo:hi])
            del out
        r = ctx.reconstruct(0, ori, 3, np.zeros(oriF), 1.0, 1.0, gridding_nr_iter=iters, do_map=False)
        return r["vol"]
    finally:
        if own:
            ctx.close()


def write_mrc(path: str, vol: np.ndarray, angpix: float) -> None:
    """A float32 cubic MRC volume with the header fields the reference sets
    (`Mrcs::setMrcHead`, src/mrcs.cpp:64-74)."""
    from .synthetic import write_mrcs
    write_mrcs(path, np.asarray(vol, np.float32), angpix)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("-i", required=True, help="input STAR file with the images and their poses")
    ap.add_argument("-o", required=True, help="output reconstruction (.mrc)")
    ap.add_argument("-angpix", type=float, required=True)
    ap.add_argument("-iter", type=int, default=10, help="gridding-correction iterations")
    ap.add_argument("-ctf", type=int, default=0)
    ap.add_argument("-ctf_intact_first_peak", type=int, default=0)
    ap.add_argument("-ctf_phase_flipped", type=int, default=0)
    ap.add_argument("-only_flip_phases", type=int, default=0)
    ap.add_argument("-maxres", type=float, default=-1.0)
    ap.add_argument("-pad", type=int, default=2)
    ap.add_argument("-sym", default="c1")
    ap.add_argument("-pool", type=int, default=1000)
    ap.add_argument("-device", type=int, default=0)
    a = ap.parse_args(argv)
    if a.pad != 2 or a.sym.lower() != "c1":
        ap.error("only -pad 2 and -sym c1 are supported")
    star = a.i if a.i.endswith(".star") else a.i + ".star"
    vol = reconstruct_from_star(star, a.angpix, a.iter, bool(a.ctf), bool(a.ctf_phase_flipped),
                                bool(a.only_flip_phases), bool(a.ctf_intact_first_peak), a.maxres, a.pool, a.device)
    out = a.o if a.o.endswith(".mrc") else a.o + ".mrc"
    write_mrc(out, vol, a.angpix)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
