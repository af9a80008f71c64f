"""CPU restatement of the reference's particle-image preparation (TEST
INFRASTRUCTURE: only tests/ may use it, as the checker of the GPU
preparation).

ParticleModel::setFourierTransforms (src/exp_model.h:397-640) for one pool:
norm correction, translation by the rounded old offsets without wrap
(translate / applyGeometry, src/image.h:53-257), CenterFFT (src/image.h:
275-340), the normalised r2c transform (src/fft_base.cpp:52-57), the window
to current_size (windowFourierTransform, src/image.h:496-566), the noise
image outside the particle mask (seeded per image with glibc srand/rand
through Random_generator::rnd_gaus, src/math.cpp:361-480) and the soft mask
(softMaskOutsideMap, src/image.h:571-634), the masked transform, the power
spectrum and highres_Xi2, and the CTF image (CTF::initialise / getCTF /
getFftwImage, src/ctf.cpp:136-191, src/ctf.h:151-204).

Parity is pinned against the reference's own outputs recorded by
oracle/ref_harness/map2d_dump in tests/golden/map2d_*.npz
(tests/test_prep_oracle.py).
"""
from __future__ import annotations

import math

import numpy as np

ROME_PI = 3.14159265358979323846
M31 = 2147483647  # 2^31 - 1: RAND_MAX and the seeding modulus


class GlibcRand:
    """std::srand / std::rand of glibc (random_r.c, TYPE_3: additive feedback
    r[i] = r[i-31] + r[i-3] over a 31-word table seeded by 16807 x mod
    2^31 - 1, 310 outputs discarded, output r >> 1) -- the generator behind
    the reference's Random_generator when MAP3D_OLD_BASELINE is defined
    (src/math.h:35, src/math.cpp:361-388)."""

    def __init__(self, seed: int):
        seed &= 0xFFFFFFFF
        if seed == 0:
            seed = 1
        w = seed if seed < 2 ** 31 else seed - 2 ** 32
        r = [w]
        for _ in range(1, 31):
            hi = int(w / 127773) if abs(w) < 2 ** 52 else w // 127773
            lo = w - hi * 127773
            w = 16807 * lo - 2836 * hi
            if w < 0:
                w += M31
            r.append(w)
        self.r = [v & 0xFFFFFFFF for v in r]
        self.f, self.b = 3, 0
        for _ in range(310):
            self()

    def __call__(self) -> int:
        r = self.r
        r[self.f] = (r[self.f] + r[self.b]) & 0xFFFFFFFF
        out = r[self.f] >> 1
        self.f = (self.f + 1) % 31
        self.b = (self.b + 1) % 31
        return out


def uniform01(eng: GlibcRand) -> np.float32:
    """randUniform01: (float)rand() / (float)RAND_MAX (src/math.cpp:383-385)."""
    return np.float32(np.float32(eng()) / np.float32(M31))


class GaussRng:
    """Random_generator::rnd_gaus (src/math.cpp:443-480): polar Box-Muller on
    float uniforms (W = U1^2 + U2^2 rounded to float, the multiplier in
    double rounded to float), the second value cached."""

    def __init__(self, seed: int):
        self.eng = GlibcRand(seed)
        self.call = 0
        self.x2 = np.float32(0)

    def gaus(self, sigma: float) -> np.float32:
        sigma = np.float32(sigma)
        if sigma == 0:
            return np.float32(0)
        if self.call == 1:
            self.call = 0
            return np.float32(sigma * self.x2)
        while True:
            u1 = np.float32(np.float32(-1) + uniform01(self.eng) * np.float32(2))
            u2 = np.float32(np.float32(-1) + uniform01(self.eng) * np.float32(2))
            w = np.float32(float(u1) * float(u1) + float(u2) * float(u2))
            if not (w >= 1 or w == 0):
                break
        # log and sqrt of the float W are the C library's double functions
        mult = np.float32(math.sqrt((-2 * math.log(float(w))) / float(w)))
        x1 = np.float32(u1 * mult)
        self.x2 = np.float32(u2 * mult)
        self.call = 1
        return np.float32(sigma * x1)


def center_fft(v: np.ndarray) -> np.ndarray:
    """CenterFFT(forward) of an even-sized square image."""
    n = v.shape[0]
    return np.roll(v, (n // 2, n // 2), axis=(0, 1))


def window_ft(F: np.ndarray, out_size: int) -> np.ndarray:
    """windowFourierTransform to a smaller (or equal) size: the low rows / columns."""
    n = F.shape[0]
    if n == out_size:
        return F.copy()
    oF = out_size // 2 + 1
    out = np.zeros((out_size, oF), complex)
    for i in range(out_size):
        ip = i if i < oF else i - out_size
        out[i] = F[ip if ip >= 0 else ip + n, :oF]
    return out


def ctf_image(size: int, ori_size: int, angpix: float, params, do_abs: bool = False, only_flip: bool = False,
              intact_first_peak: bool = False) -> np.ndarray:
    """CTF::getFftwImage(size, ori, ori, angpix, do_abs, only_flip,
    intact_first_peak, damping on) for params = (defocus U, defocus V,
    defocus angle, voltage, Cs, Q0, B-factor); scale 1."""
    du, dv, dang, kv, cs, q0, bfac = (float(v) for v in params)
    local_cs, local_kv = cs * 1e7, kv * 1e3
    rad_az = dang * ROME_PI / 180.0
    avg, dev = -(du + dv) * 0.5, -(du - dv) * 0.5
    lam = 12.2643247 / math.sqrt(local_kv * (1. + local_kv * 0.978466e-6))
    k1 = ROME_PI / 2 * 2 * lam
    k2 = ROME_PI / 2 * local_cs * lam * lam * lam
    k3 = math.sqrt(1 - q0 * q0)
    k4 = -bfac / 4.
    hdim = size // 2 + 1
    xs = ori_size * angpix
    out = np.zeros((size, hdim))
    for i in range(size):
        ip = i if i < hdim else i - size
        for j in range(hdim):
            x, y = j / xs, ip / xs
            u2 = x * x + y * y
            u4 = u2 * u2
            if abs(x) < 1e-6 and abs(y) < 1e-6:  # ROME_EQUAL_ACCURACY (double build)
                df = 0.0
            else:
                df = avg + dev * math.cos(2 * (math.atan2(y, x) - rad_az))
            arg = k1 * df * u2 + k2 * u4
            if intact_first_peak and abs(arg) < ROME_PI / 2.:
                v = 1.
            else:
                v = -(k3 * math.sin(arg) - q0 * math.cos(arg))
            v *= math.exp(k4 * u2)
            if do_abs:
                v = abs(v)
            elif only_flip:
                v = -1. if v < 0. else 1.
            out[i, j] = v
    return out


def prepare_pool(raw: np.ndarray, meta: np.ndarray, group: np.ndarray, sigma2_noise: np.ndarray, current_size: int,
                 first_image: int, o: dict):
    """Returns dict of Fimg (masked) [P][F], Fimg_nomask [P][F] (complex), Fctf
    [P][F], highres_Xi2 [P], power_imgs [P][ori/2+1], old_offsetx/y [P].
    meta rows: NORM, XOFF, YOFF, DEFOCUS_U, DEFOCUS_V, DEFOCUS_ANGLE, VOLTAGE, CS, Q0, BFAC."""
    P, ori = raw.shape[0], raw.shape[1]
    oF = ori // 2 + 1
    fine, fineF = current_size, current_size // 2 + 1
    cen = ori // 2
    out = {k: [] for k in ("Fimg", "Fimg_nomask", "Fctf", "highres_Xi2", "power_imgs", "old_offsetx",
                           "old_offsety")}
    ii, jj = np.meshgrid(np.arange(ori), np.arange(ori), indexing="ij")
    r = np.sqrt(((ii - cen) ** 2 + (jj - cen) ** 2).astype(np.float64))
    radius = o["particle_diameter"] / (2.0 * o["pixel_size"])
    width = float(o["width_mask_edge"])
    radius_p = radius + width
    ip_all = np.where(np.arange(ori) < oF, np.arange(ori), np.arange(ori) - ori)
    ires = np.array([[int(round(math.sqrt(ip * ip + jp * jp))) for jp in range(oF)] for ip in ip_all])
    for i in range(P):
        img = raw[i].astype(np.float64).copy()
        if o["do_norm_correction"]:
            img = img * o["avg_norm_correction"] / meta[i, 0]
        # C round(): half away from zero
        ox = math.copysign(math.floor(abs(meta[i, 1]) + 0.5), meta[i, 1])
        oy = math.copysign(math.floor(abs(meta[i, 2]) + 0.5), meta[i, 2])
        tr = np.zeros_like(img)
        dx, dy = int(ox), int(oy)
        for a in range(ori):
            sa = a - dy
            if 0 <= sa < ori:
                for b in range(ori):
                    sb = b - dx
                    if 0 <= sb < ori:
                        tr[a, b] = img[sa, sb]
        F0 = np.fft.rfft2(center_fft(tr)) / (ori * ori)
        nomask = window_ft(F0, fine)
        if not o["do_zero_mask"]:
            rng = GaussRng(o["random_seed"] + first_image + i)
            Fn = np.zeros((ori, oF), complex)
            s2 = sigma2_noise[group[i]]
            for a in range(ori):
                for b in range(oF):
                    ir = ires[a, b]
                    if 0 <= ir < oF:
                        sig = math.sqrt(o["sigma2_fudge"] * s2[ir])
                        re = float(rng.gaus(sig))
                        im = float(rng.gaus(sig))
                        Fn[a, b] = complex(re, im)
            Mnoise = np.fft.irfft2(Fn, s=(ori, ori)) * (ori * ori)
        else:
            Mnoise = None
        m = tr.copy()
        edge = (r >= radius) & (r <= radius_p)
        rc = 0.5 + 0.5 * np.cos(ROME_PI * (radius_p - r) / width)
        if Mnoise is None:
            w = np.where(r > radius_p, 1.0, np.where(edge, rc, 0.0))
            bg = np.sum(w * tr) / np.sum(w)
            add = np.full_like(tr, bg)
        else:
            add = Mnoise
        m = np.where(edge, (1 - rc) * m + rc * add, m)
        m = np.where(r > radius_p, add, m)
        F1 = np.fft.rfft2(center_fft(m)) / (ori * ori)
        spec = np.zeros(oF)
        xi2 = 0.0
        if fine < ori:
            for a in range(ori):
                ip = ip_all[a]
                for b in range(oF):
                    ir = ires[a, b]
                    if ir > 0 and ir < oF and not (b == 0 and ip < 0):
                        v = F1[a, b].real ** 2 + F1[a, b].imag ** 2
                        spec[ir] += v
                        if ir >= fineF:
                            xi2 += v
        ctf = ctf_image(fine, ori, o["pixel_size"], meta[i, 3:10], o.get("ctf_phase_flipped", False),
                        o.get("only_flip_phases", False), o.get("intact_ctf_first_peak", False)) \
            if o["do_ctf_correction"] else np.ones((fine, fineF))
        out["Fimg"].append(window_ft(F1, fine).reshape(-1))
        out["Fimg_nomask"].append(nomask.reshape(-1))
        out["Fctf"].append(np.asarray(ctf).reshape(-1))
        out["highres_Xi2"].append(xi2)
        out["power_imgs"].append(spec)
        out["old_offsetx"].append(ox)
        out["old_offsety"].append(oy)
    return {k: np.array(v) for k, v in out.items()}


def options_from_golden(g) -> dict:
    sc = lambda k: float(np.asarray(g[k]).ravel()[0])  # noqa: E731
    return dict(avg_norm_correction=sc("prep_avg_norm_correction"), pixel_size=sc("prep_pixel_size"),
                particle_diameter=sc("prep_particle_diameter"), width_mask_edge=int(sc("prep_width_mask_edge")),
                sigma2_fudge=sc("prep_sigma2_fudge"), random_seed=int(sc("prep_random_seed")),
                do_norm_correction=bool(sc("prep_do_norm_correction")), do_zero_mask=bool(sc("prep_do_zero_mask")),
                do_ctf_correction=bool(sc("do_ctf_correction")),
                ctf_phase_flipped=bool(sc("prep_ctf_phase_flipped")), only_flip_phases=bool(sc("prep_only_flip_phases")),
                intact_ctf_first_peak=bool(sc("prep_intact_ctf_first_peak")))
