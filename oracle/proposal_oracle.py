"""CPU restatement of the pose-proposal network (test infrastructure only: the
checker for the CUDA training and inference kernels in
rome_b200/csrc/proposal.cu, never called by the product).

The network has no counterpart in the reference; it is the learned prior of
the E-step.  It sees a particle's Fourier magnitude in polar coordinates,
where an in-plane rotation by psi is a circular shift along the angle axis,
and is equivariant to that shift by construction, so one set of weights
serves every psi:

    x [N][2][R][A]     log(1 + |X|) and |CTF| at radii r_lo..r_hi (R bins)
                       and angles theta_a = a * 180 / A (A = nr_psi / 2)
    conv3x3 (2 -> c0) + ReLU, conv3x3 (c0 -> c1) + ReLU
                       (zero padding along r, circular along theta)
    head: z[n][k][p] = bf[k] + sum_{c,r,d} wf[k][c][r][d] h[n][c][r][(d - p) mod A]
    loss = mean_n sum_{k,p} -t[n][k][p] log softmax(z[n])[k][p]

With P_psi(k) = F_T(R(psi) k) for the reference's rotate2D (Euler(0, 0, psi)
transposed), the magnitude seen at angle theta is the template's at theta +
psi, so the correlation above peaks at p = psi / (180 / A): output p is the
psi index modulo 180 degrees.  All arithmetic here is FP64.
"""
from __future__ import annotations

from typing import Dict, List, Tuple

import numpy as np


def param_shapes(n_r: int, n_theta: int, channels: Tuple[int, int], n_classes: int) -> List[Tuple[str, tuple]]:
    c0, c1 = channels
    return [("w0", (c0, 2, 3, 3)), ("b0", (c0,)), ("w1", (c1, c0, 3, 3)), ("b1", (c1,)),
            ("wf", (n_classes, c1, n_r, n_theta)), ("bf", (n_classes,))]


def _pad(x: np.ndarray) -> np.ndarray:
    """zero padding 1 along r (axis 2), circular padding 1 along theta (axis 3)"""
    x = np.concatenate([x[..., -1:], x, x[..., :1]], axis=3)
    z = np.zeros(x.shape[:2] + (1, x.shape[3]), x.dtype)
    return np.concatenate([z, x, z], axis=2)


def conv(x: np.ndarray, w: np.ndarray, b: np.ndarray) -> np.ndarray:
    N, C, R, A = x.shape
    xp = _pad(x)
    out = np.zeros((N, w.shape[0], R, A))
    for kh in range(3):
        for kw in range(3):
            out += np.einsum("nchw,oc->nohw", xp[:, :, kh:kh + R, kw:kw + A], w[:, :, kh, kw])
    return out + b[None, :, None, None]


def conv_backward(x, w, dy):
    N, C, R, A = x.shape
    xp = _pad(x)
    dxp = np.zeros_like(xp)
    dw = np.zeros_like(w)
    for kh in range(3):
        for kw in range(3):
            dw[:, :, kh, kw] = np.einsum("nohw,nchw->oc", dy, xp[:, :, kh:kh + R, kw:kw + A])
            dxp[:, :, kh:kh + R, kw:kw + A] += np.einsum("nohw,oc->nchw", dy, w[:, :, kh, kw])
    dx = dxp[:, :, 1:R + 1, 1:A + 1].copy()
    dx[:, :, :, 0] += dxp[:, :, 1:R + 1, A + 1]   # circular wrap of the theta padding
    dx[:, :, :, A - 1] += dxp[:, :, 1:R + 1, 0]
    return dx, dw, dy.sum(axis=(0, 2, 3))


def head(h: np.ndarray, wf: np.ndarray, bf: np.ndarray) -> np.ndarray:
    N, C, R, A = h.shape
    z = np.zeros((N, wf.shape[0], A))
    for p in range(A):
        hs = np.roll(h, p, axis=3)  # hs[..., d] = h[..., (d - p) mod A]
        z[:, :, p] = np.einsum("ncrd,kcrd->nk", hs, wf)
    return z + bf[None, :, None]


def head_backward(h, wf, dz):
    N, C, R, A = h.shape
    dwf = np.zeros_like(wf)
    dh = np.zeros_like(h)
    for p in range(A):
        hs = np.roll(h, p, axis=3)
        dwf += np.einsum("nk,ncrd->kcrd", dz[:, :, p], hs)
        dh += np.roll(np.einsum("nk,kcrd->ncrd", dz[:, :, p], wf), -p, axis=3)
    return dh, dwf, dz.sum(axis=(0, 2))


def forward(params: Dict[str, np.ndarray], x: np.ndarray):
    h0 = np.maximum(conv(x, params["w0"], params["b0"]), 0.0)
    h1 = np.maximum(conv(h0, params["w1"], params["b1"]), 0.0)
    z = head(h1, params["wf"], params["bf"]).reshape(x.shape[0], -1)
    return z, (x, h0, h1)


def softmax(z: np.ndarray) -> np.ndarray:
    e = np.exp(z - z.max(axis=1, keepdims=True))
    return e / e.sum(axis=1, keepdims=True)


def loss_and_grads(params: Dict[str, np.ndarray], x: np.ndarray, t: np.ndarray):
    """Mean soft-target cross-entropy over the batch, its gradients, logits."""
    N = x.shape[0]
    z, (x0, h0, h1) = forward(params, x)
    p = softmax(z)
    loss = float(-np.sum(t * np.log(np.maximum(p, 1e-300))) / N)
    dz = ((p - t) / N).reshape(N, params["wf"].shape[0], -1)
    g = {}
    dh1, g["wf"], g["bf"] = head_backward(h1, params["wf"], dz)
    dh1 = dh1 * (h1 > 0)
    dh0, g["w1"], g["b1"] = conv_backward(h0, params["w1"], dh1)
    dh0 = dh0 * (h0 > 0)
    _, g["w0"], g["b0"] = conv_backward(x0, params["w0"], dh0)
    return loss, g, z


def features(Fimg_real: np.ndarray, Fimg_imag: np.ndarray, ctf: np.ndarray, cur: int, n_r: int, n_theta: int,
             r_lo: float, r_hi: float) -> np.ndarray:
    """Network input from a particle's masked Fourier image (FFTW half-plane
    [cur][cur/2+1]): bilinear samples of log(1 + |X|) and |CTF| at radius
    r_i = r_lo + i (r_hi - r_lo) / (n_r - 1) and angle theta_a = a pi / n_theta
    (kx = r cos, ky = r sin; negative kx by Friedel symmetry), each channel
    of each particle normalised to zero mean and unit variance."""
    P = Fimg_real.shape[0]
    cf = cur // 2 + 1
    mag = np.log1p(np.sqrt(Fimg_real ** 2 + Fimg_imag ** 2)).reshape(P, cur, cf)
    c = np.abs(ctf).reshape(P, cur, cf)
    out = np.zeros((P, 2, n_r, n_theta))

    def sample(img, kx, ky):
        # value at integer frequency (x, y) with Friedel symmetry for x < 0
        def at(x, y):
            if x < 0:
                x, y = -x, -y
            row = y if y >= 0 else y + cur
            return img[:, row, x]
        x0, y0 = int(np.floor(kx)), int(np.floor(ky))
        fx, fy = kx - x0, ky - y0
        return ((1 - fy) * ((1 - fx) * at(x0, y0) + fx * at(x0 + 1, y0))
                + fy * ((1 - fx) * at(x0, y0 + 1) + fx * at(x0 + 1, y0 + 1)))

    for i in range(n_r):
        r = r_lo + i * (r_hi - r_lo) / (n_r - 1)
        for a in range(n_theta):
            th = a * np.pi / n_theta
            kx, ky = r * np.cos(th), r * np.sin(th)
            out[:, 0, i, a] = sample(mag, kx, ky)
            out[:, 1, i, a] = sample(c, kx, ky)
    m = out.mean(axis=(2, 3), keepdims=True)
    s = out.std(axis=(2, 3), keepdims=True)
    return (out - m) / np.maximum(s, 1e-12)
