"""CPU restatement of the pose-proposal network (test infrastructure only: the
checker for the CUDA training and inference kernels in
rome_b200/csrc/proposal.cu, never called by the product).

The network has no counterpart in the reference; it is the learned prior of
the E-step (a small CNN over the low-pass Fourier magnitude of a particle that
predicts a distribution over (class, psi mod 180)).  Layers, all FP64 here:

    x [N][2][S][S]
    conv3x3 s1 (2 -> c0) + ReLU
    conv3x3 s2 (c0 -> c1) + ReLU
    conv3x3 s2 (c1 -> c2) + ReLU
    conv3x3 s2 (c2 -> c3) + ReLU          -> [N][c3][S/8][S/8]
    flatten, linear (c3*(S/8)^2 -> O)     -> logits
    loss = mean_n sum_o -t[n][o] * log softmax(z[n])[o]

Convolutions use zero padding 1; a stride-2 output pixel (ho, wo) reads the
input at (2 ho + kh - 1, 2 wo + kw - 1).
"""
from __future__ import annotations

from typing import Dict, List, Tuple

import numpy as np

STRIDES = (1, 2, 2, 2)


def param_shapes(in_ch: int, size: int, channels: Tuple[int, int, int, int], n_out: int) -> List[Tuple[str, tuple]]:
    shapes = []
    c_prev = in_ch
    for li, c in enumerate(channels):
        shapes.append((f"w{li}", (c, c_prev, 3, 3)))
        shapes.append((f"b{li}", (c,)))
        c_prev = c
    flat = channels[-1] * (size // 8) ** 2
    shapes.append(("wf", (n_out, flat)))
    shapes.append(("bf", (n_out,)))
    return shapes


def conv3x3(x: np.ndarray, w: np.ndarray, b: np.ndarray, stride: int) -> np.ndarray:
    N, C, H, W = x.shape
    Co = w.shape[0]
    Ho, Wo = (H - 1) // stride + 1, (W - 1) // stride + 1
    xp = np.zeros((N, C, H + 2, W + 2), x.dtype)
    xp[:, :, 1:H + 1, 1:W + 1] = x
    out = np.zeros((N, Co, Ho, Wo), x.dtype)
    for kh in range(3):
        for kw in range(3):
            patch = xp[:, :, kh:kh + stride * (Ho - 1) + 1:stride, kw:kw + stride * (Wo - 1) + 1:stride]
            out += np.einsum("nchw,oc->nohw", patch, w[:, :, kh, kw])
    return out + b[None, :, None, None]


def conv3x3_backward(x, w, dy, stride):
    N, C, H, W = x.shape
    _, _, Ho, Wo = dy.shape
    xp = np.zeros((N, C, H + 2, W + 2), x.dtype)
    xp[:, :, 1:H + 1, 1:W + 1] = x
    dxp = np.zeros_like(xp)
    dw = np.zeros_like(w)
    for kh in range(3):
        for kw in range(3):
            sl = (slice(None), slice(None), slice(kh, kh + stride * (Ho - 1) + 1, stride),
                  slice(kw, kw + stride * (Wo - 1) + 1, stride))
            dw[:, :, kh, kw] = np.einsum("nohw,nchw->oc", dy, xp[sl])
            dxp[sl] += np.einsum("nohw,oc->nchw", dy, w[:, :, kh, kw])
    db = dy.sum(axis=(0, 2, 3))
    return dxp[:, :, 1:H + 1, 1:W + 1], dw, db


def forward(params: Dict[str, np.ndarray], x: np.ndarray):
    acts = [x]
    h = x
    for li, s in enumerate(STRIDES):
        h = np.maximum(conv3x3(h, params[f"w{li}"], params[f"b{li}"], s), 0.0)
        acts.append(h)
    flat = h.reshape(h.shape[0], -1)
    z = flat @ params["wf"].T + params["bf"]
    return z, acts


def softmax(z: np.ndarray) -> np.ndarray:
    e = np.exp(z - z.max(axis=1, keepdims=True))
    return e / e.sum(axis=1, keepdims=True)


def loss_and_grads(params: Dict[str, np.ndarray], x: np.ndarray, t: np.ndarray):
    """Mean soft-target cross-entropy over the batch and its gradients."""
    N = x.shape[0]
    z, acts = forward(params, x)
    p = softmax(z)
    loss = float(-np.sum(t * np.log(np.maximum(p, 1e-300))) / N)
    dz = (p - t) / N
    g = {}
    flat = acts[-1].reshape(N, -1)
    g["wf"] = dz.T @ flat
    g["bf"] = dz.sum(axis=0)
    dh = (dz @ params["wf"]).reshape(acts[-1].shape)
    for li in reversed(range(len(STRIDES))):
        dh = dh * (acts[li + 1] > 0)
        dx, g[f"w{li}"], g[f"b{li}"] = conv3x3_backward(acts[li], params[f"w{li}"], dh, STRIDES[li])
        dh = dx
    return loss, g, z


def features(Fimg_real: np.ndarray, Fimg_imag: np.ndarray, ctf: np.ndarray, cur: int, size: int) -> np.ndarray:
    """Network input from the particle's masked Fourier image (FFTW half-plane,
    [cur][cur/2+1]): channel 0 log(1 + |X|), channel 1 |CTF|, on the centred
    size x size grid of frequencies (kx, ky) in [-size/2, size/2), the
    negative-kx half filled by Friedel symmetry |X(-k)| = |X(k)|; each channel
    of each particle normalised to zero mean and unit variance."""
    P = Fimg_real.shape[0]
    cf = cur // 2 + 1
    mag = np.sqrt(Fimg_real ** 2 + Fimg_imag ** 2).reshape(P, cur, cf)
    c = np.abs(ctf).reshape(P, cur, cf)
    h = size // 2
    out = np.zeros((P, 2, size, size))
    for iy in range(size):
        ky = iy - h
        for ix in range(size):
            kx = ix - h
            sx, sy = (kx, ky) if kx >= 0 else (-kx, -ky)
            row = sy if sy >= 0 else sy + cur
            out[:, 0, iy, ix] = np.log1p(mag[:, row, sx])
            out[:, 1, iy, ix] = c[:, row, sx]
    m = out.mean(axis=(2, 3), keepdims=True)
    s = out.std(axis=(2, 3), keepdims=True)
    return (out - m) / np.maximum(s, 1e-12)
