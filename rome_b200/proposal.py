"""Learned pose proposals: the Python side of rome_gpu_proposal_* (a small
rotation-equivariant network trained on the GPU on (image, posterior) pairs
of the exhaustive E-step) and the proposal-restricted E-step built on it.

Output index of the network: o = class * (nr_psi / 2) + (psi mod nr_psi / 2);
the Fourier magnitude the network sees cannot tell psi from psi + 180, so a
proposed output expands to the two orientations class * nr_psi + psi and
class * nr_psi + psi + nr_psi / 2.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import abi
from .map2d import PARTICLE_OUTPUTS, GpuContext, Map2dPool, _f64, concat_pools, merge_results, take_pool

__all__ = ["ProposalNet", "param_offsets", "flat_to_dict", "dict_to_flat", "posterior_targets",
           "expand_proposals", "learned_estep", "learned_estep_pools", "DEFAULT_CHANNELS"]

DEFAULT_CHANNELS = (16, 16)
_FP = C.POINTER(C.c_float)


def _fptr(a: np.ndarray):
    abi._need(a, np.float32)
    return a.ctypes.data_as(_FP)


def param_offsets(n_r: int, n_theta: int, channels, n_classes: int) -> List[Tuple[str, tuple, int]]:
    """(name, shape, offset) of every parameter block in the flat array; each
    block starts at a multiple of 4 floats, as the library lays them out."""
    a4 = lambda v: (v + 3) // 4 * 4  # noqa: E731
    c0, c1 = channels
    shapes = [("w0", (c0, 2, 3, 3)), ("b0", (c0,)), ("w1", (c1, c0, 3, 3)), ("b1", (c1,)),
              ("wf", (n_classes, c1, n_r, n_theta)), ("bf", (n_classes,))]
    out, o = [], 0
    for name, shape in shapes:
        out.append((name, shape, o))
        o = a4(o + int(np.prod(shape)))
    return out + [("_total", (), o)]


def flat_to_dict(flat: np.ndarray, n_r: int, n_theta: int, channels, n_classes: int) -> Dict[str, np.ndarray]:
    d = {}
    for name, shape, off in param_offsets(n_r, n_theta, channels, n_classes)[:-1]:
        n = int(np.prod(shape))
        d[name] = np.asarray(flat[off:off + n], np.float64).reshape(shape)
    return d


def dict_to_flat(d: Dict[str, np.ndarray], n_r: int, n_theta: int, channels, n_classes: int) -> np.ndarray:
    offs = param_offsets(n_r, n_theta, channels, n_classes)
    flat = np.zeros(offs[-1][2], np.float32)
    for name, shape, off in offs[:-1]:
        flat[off:off + int(np.prod(shape))] = np.asarray(d[name], np.float32).ravel()
    return flat


def posterior_targets(marg: np.ndarray, nr_classes: int, nr_psi: int) -> np.ndarray:
    """Training targets from the E-step's (class, psi) posterior marginals:
    psi folded modulo 180 degrees, each row normalised to 1."""
    h = nr_psi // 2
    m = marg.reshape(-1, nr_classes, 2, h).sum(axis=2).reshape(-1, nr_classes * h)
    s = m.sum(axis=1, keepdims=True)
    return (m / np.where(s > 0, s, 1.0)).astype(np.float32)


def expand_proposals(idx: np.ndarray, nr_psi: int) -> np.ndarray:
    """Network outputs [n][k] -> ascending orientation lists [n][2k]."""
    h = nr_psi // 2
    cls, pm = idx // h, idx % h
    j = np.concatenate([cls * nr_psi + pm, cls * nr_psi + pm + h], axis=1)
    return np.sort(j, axis=1).astype(np.int32)


class ProposalNet:
    """rome_gpu_proposal_* on one GpuContext: n_classes x n_theta outputs
    (n_theta = nr_psi / 2), polar input of n_r radii in [r_lo, r_hi]."""

    def __init__(self, ctx: GpuContext, n_classes: int, n_theta: int, n_r: int = 16, channels=DEFAULT_CHANNELS,
                 r_lo: float = 2.0, r_hi: float = 24.0, seed: int = 0):
        self.ctx, self.lib = ctx, ctx.lib
        self.n_classes, self.n_theta, self.n_r, self.channels = n_classes, n_theta, n_r, tuple(channels)
        self.r_lo, self.r_hi = r_lo, r_hi
        self.n_out = n_classes * n_theta
        spec = abi.RomeProposalSpec(n_r, n_theta, (C.c_int * 2)(*channels), n_classes, r_lo, r_hi)
        h = C.c_void_p()
        ctx._check(self.lib.rome_gpu_proposal_create(ctx.h, C.byref(spec), seed, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            self.lib.rome_gpu_proposal_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def nparam(self) -> int:
        return int(self.lib.rome_gpu_proposal_num_params(self.h))

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.nparam, np.float32)
        self.ctx._check(self.lib.rome_gpu_proposal_get_params(self.h, _fptr(out)))
        return out

    def set_params(self, flat: np.ndarray):
        flat = np.ascontiguousarray(flat, np.float32)
        if flat.size != self.nparam:
            raise ValueError(f"{flat.size} parameters given, the network has {self.nparam}")
        self.ctx._check(self.lib.rome_gpu_proposal_set_params(self.h, _fptr(flat)))

    def features(self, p) -> np.ndarray:
        """Network input [P][2][n_r][n_theta] of a pool (Map2dPool, or a whole
        StagedPool whose images live on the device)."""
        from .map2d import StagedPool
        base = p.pool if isinstance(p, StagedPool) else p
        x = np.zeros((base.nr_images, 2, self.n_r, self.n_theta), np.float32)
        if isinstance(p, StagedPool):
            import torch
            torch.cuda.current_stream(self.ctx.device).synchronize()
            if base.particle_rows is not None:
                raise ValueError("features takes a whole staged pool, not a particle_rows subset")
            ptrs = [C.c_void_p(p.dev[n].data_ptr()) for n in ("Fimg_real", "Fimg_imag", "Fctf")]
            keep, on_dev = None, 1
        else:
            keep = [_f64(base.Fimg_real), _f64(base.Fimg_imag), _f64(base.Fctf)]
            ptrs = [C.c_void_p(a.ctypes.data) for a in keep]
            on_dev = 0
        self.ctx._check(self.lib.rome_gpu_proposal_features(self.h, base.nr_images, base.current_size, ptrs[0],
                                                            ptrs[1], ptrs[2], on_dev, _fptr(x)))
        del keep
        return x

    def loss_grad(self, x: np.ndarray, t: np.ndarray):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        n = x.shape[0]
        loss = np.zeros(1)
        grad = np.zeros(self.nparam, np.float32)
        logits = np.zeros((n, self.n_out), np.float32)
        self.ctx._check(self.lib.rome_gpu_proposal_loss_grad(self.h, n, _fptr(x), _fptr(t), abi.dptr(loss),
                                                             _fptr(grad), _fptr(logits)))
        return float(loss[0]), grad, logits

    def train(self, x: np.ndarray, t: np.ndarray, epochs: int = 10, batch: int = 256, lr: float = 1e-3,
              seed: int = 1) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        losses = np.zeros(epochs)
        self.ctx._check(self.lib.rome_gpu_proposal_train(self.h, x.shape[0], _fptr(x), _fptr(t), epochs, batch,
                                                         lr, seed, abi.dptr(losses)))
        return losses

    def predict(self, x: np.ndarray, k: int):
        x = np.ascontiguousarray(x, np.float32)
        n = x.shape[0]
        idx = np.zeros((n, k), np.int32)
        prob = np.zeros((n, k), np.float32)
        self.ctx._check(self.lib.rome_gpu_proposal_predict(self.h, n, _fptr(x), k, abi.iptr(idx), _fptr(prob)))
        return idx, prob

    def init_matched_filter(self, templates: np.ndarray, scale: float = 1.0, seed: int = 0):
        """Start from a matched filter instead of random weights: the two
        convolutions pass the log-magnitude channel through (centre tap 1 on
        channel 0, every other weight small), and the head correlates it,
        over all rotations, with each output class's template features
        (templates [n_classes][2][n_r][n_theta], e.g. the features of each
        class/direction's projection; zero mean, unit norm per class).
        Training then refines it.  The physics supplies what few training
        particles per class cannot (e.g. one class per 3D direction)."""
        rng = np.random.default_rng(seed)
        d = flat_to_dict(self.get_params(), self.n_r, self.n_theta, self.channels, self.n_classes)
        for name in d:
            d[name] = d[name] * 0.01
        d["w0"][0, 0, 1, 1] = 1.0
        d["w1"][0, 0, 1, 1] = 1.0
        d["b0"][:] = 0.0
        d["b1"][:] = 0.0
        t = np.asarray(templates, np.float64)[:, 0]  # the log-magnitude channel
        t = t - t.mean(axis=(1, 2), keepdims=True)
        t = t / np.maximum(np.linalg.norm(t.reshape(len(t), -1), axis=1), 1e-30)[:, None, None]
        d["wf"][:, 0] = scale * t
        d["bf"][:] = 0.0
        self.set_params(dict_to_flat(d, self.n_r, self.n_theta, self.channels, self.n_classes))
        del rng

    def propose(self, p, k: int):
        """Top-k network outputs of every particle of a pool (a Map2dPool, or
        a StagedPool whose images live on the device), expanded to ascending
        orientation lists [P][2k], and the probability mass they cover."""
        from .map2d import StagedPool
        base = p.pool if isinstance(p, StagedPool) else p
        P = base.nr_images
        prop = np.zeros((P, 2 * k), np.int32)
        mass = np.zeros(P, np.float32)
        keep = None
        if isinstance(p, StagedPool):
            import torch
            torch.cuda.current_stream(self.ctx.device).synchronize()
            if base.particle_rows is not None:
                raise ValueError("propose takes a whole staged pool, not a particle_rows subset")
            ptrs = [C.c_void_p(p.dev[n].data_ptr()) for n in ("Fimg_real", "Fimg_imag", "Fctf")]
            on_dev = 1
        else:
            keep = [_f64(base.Fimg_real), _f64(base.Fimg_imag), _f64(base.Fctf)]
            ptrs = [C.c_void_p(a.ctypes.data) for a in keep]
            on_dev = 0
        self.ctx._check(self.lib.rome_gpu_proposal_propose(self.h, P, base.current_size, ptrs[0], ptrs[1], ptrs[2],
                                                           on_dev, k, abi.iptr(prop), _fptr(mass)))
        del keep
        return prop, mass


def learned_estep(ctx: GpuContext, net: ProposalNet, pool, k: int, min_mass: float = 0.0, marginals: bool = False):
    """E-step of one pool (Map2dPool or StagedPool) with learned proposals:
    every particle is searched over the 2k orientations of its top-k network
    outputs, except those whose top-k outputs hold less than `min_mass` of the
    network's probability, which are searched exhaustively.  Returns (the
    E-step outputs in pool order, proposals [P][2k], mass [P], the indices of
    the exhaustively searched particles)."""
    props, mass = net.propose(pool, k)
    n = pool.nr_images
    low = np.flatnonzero(mass < min_mass)
    if low.size == 0:
        return ctx.map2d_estep_pool(pool, marginals=marginals, proposals=props), props, mass, low
    high = np.flatnonzero(mass >= min_mass)
    parts = []
    if high.size:
        parts.append((high, ctx.map2d_estep_pool(take_pool(pool, high), marginals=marginals, proposals=props[high])))
    parts.append((low, ctx.map2d_estep_pool(take_pool(pool, low), marginals=marginals)))
    return merge_results(parts, n), props, mass, low


def learned_estep_pools(ctx: GpuContext, net: ProposalNet, pools, k: int, min_mass: float = 0.0,
                        marginals: bool = False, workers=None):
    """learned_estep over several pools of one iteration (a list, or any
    iterable such as GpuContext.staged(host_pools) whose pools are worked on
    as they arrive), with the particles that fall back to the exhaustive
    search gathered from every pool into a single exhaustive E-step (one call
    instead of one per pool, after the pools).

    workers: optional further (GpuContext, ProposalNet) pairs on the same
    device with the same model; pools are dealt round-robin to one host
    thread per pair, so that one context's host-side work overlaps another's
    kernels, and their back-projectors are added into `ctx`'s at the end.

    Returns one (outputs, proposals, mass, fallback indices) per pool; the
    fallback call's pool sums (wsum_*) are added to the first pool's, so the
    sums over all pools are those of the whole set."""
    lanes = [(ctx, net)] + list(workers or [])
    if len(lanes) == 1:
        return _learned_stream(lanes, None, pools, k, min_mass, marginals)
    from concurrent.futures import ThreadPoolExecutor
    execs = [ThreadPoolExecutor(max_workers=1) for _ in lanes]
    try:
        return _learned_stream(lanes, execs, pools, k, min_mass, marginals)
    finally:
        for e in execs:
            e.shutdown(wait=True)
        for c, _ in lanes[1:]:
            ctx.add_backprojectors(c, clear=True)


def learned_estep3d(ctx: GpuContext, net: ProposalNet, pool, k: int, min_mass: float = 0.0,
                    marginals: bool = False):
    """MAP3D E-step of one pool (Map3dPool) with learned proposals: the
    network (one output per (class, direction), psi mod 180) proposes the 2k
    coarse orientations (class * nr_dir + dir) * nr_psi + psi of each
    particle's top-k outputs and the coarse pass searches only those, with
    every translation (the fine pass refines the coarse-significant points
    among them as usual); particles whose top-k outputs hold less than
    `min_mass` of the network's probability are searched exhaustively
    (map3d_estep_pools_adaptive, which splits a pool whose fine pass would
    not fit).  Both calls back-project into the context's back-projectors.
    Returns (the E-step outputs in pool order, proposals [P][2k], mass [P],
    the indices of the exhaustively searched particles)."""
    props, mass = net.propose(pool, k)
    out, low = _restricted_or_exhaustive3d(ctx, pool, props, mass, min_mass, marginals)
    return out, props, mass, low


def lowres_proposals3d(aux: GpuContext, pool, k: int, coarse_size: int = 12, dev: Optional[dict] = None):
    """Coarse-pass proposals for a MAP3D pool from an exhaustive coarse pass
    at a small coarse size: every orientation and translation compared over
    the shells below coarse_size / 2 only, with the pool's priors.  The
    library's 3D E-step runs on `aux`, a second context with the same
    projectors, whose weighted sums and back-projectors are not used; its
    significance fraction is set so small that the fine pass refines one
    coarse point per particle.  `dev`: the pool's images already on the
    device (as for map3d_estep_pool).  Returns (the k most probable coarse
    orientations of each particle, ascending [P][k], and the
    low-resolution posterior mass they hold [P])."""
    from .map3d import map3d_estep_pool
    from .workload import mresol
    q = dataclasses.replace(pool, coarse_size=coarse_size, Mresol_coarse=mresol(coarse_size),
                            adaptive_fraction=1e-12, proposals=None)
    post = map3d_estep_pool(aux, q, marginals=True, dev=dev)["post_coarse"]
    k = min(k, post.shape[1])  # k at or above the orientation count proposes them all
    top = np.argpartition(-post, k - 1, axis=1)[:, :k]
    mass = np.take_along_axis(post, top, axis=1).sum(axis=1)
    return np.sort(top, axis=1).astype(np.int32), mass


def lowres_estep3d(ctx: GpuContext, aux: GpuContext, pool, k: int, coarse_size: int = 12, min_mass: float = 0.0,
                   marginals: bool = False, dev: Optional[dict] = None):
    """MAP3D E-step of one pool with proposals from a low-resolution
    exhaustive coarse pass (lowres_proposals3d on `aux`): each particle's
    coarse pass at the pool's own coarse size searches only its k proposed
    orientations, with every translation; particles whose proposals hold
    less than `min_mass` of the low-resolution posterior are searched
    exhaustively.  Returns (outputs in pool order, proposals [P][k], mass
    [P], the indices of the exhaustively searched particles)."""
    props, mass = lowres_proposals3d(aux, pool, k, coarse_size, dev=dev)
    out, low = _restricted_or_exhaustive3d(ctx, pool, props, mass, min_mass, marginals, dev=dev)
    return out, props, mass, low


def _rows3d(pool, dev: Optional[dict], idx: np.ndarray):
    """The particles idx of a pool and of its device images (None: host images only)."""
    from .map3d import take_pool3d
    if dev is None:
        return take_pool3d(pool, idx), None
    import torch
    t = next(iter(dev.values()))
    ix = torch.as_tensor(np.asarray(idx, np.int64), device=t.device)
    return take_pool3d(pool, idx), {name: v.index_select(0, ix) for name, v in dev.items()}


def _restricted_or_exhaustive3d(ctx: GpuContext, pool, props: np.ndarray, mass: np.ndarray, min_mass: float,
                                marginals: bool, dev: Optional[dict] = None):
    """The restricted coarse pass for the particles whose proposals hold at
    least min_mass, the exhaustive one for the rest; outputs merged back to
    pool order, sums added.  Returns (outputs, the exhaustive particles)."""
    from .map3d import map3d_estep_pool, map3d_estep_pools_adaptive, merge_results3d
    n = pool.nr_images
    low = np.flatnonzero(mass < min_mass)
    high = np.flatnonzero(mass >= min_mass)
    parts = []
    if high.size:
        sub, sdev = (pool, dev) if low.size == 0 else _rows3d(pool, dev, high)
        parts.append((high, map3d_estep_pool(ctx, sub, marginals=marginals, proposals=props[high], dev=sdev)))
    if low.size:
        sub, sdev = _rows3d(pool, dev, low)
        if marginals:
            parts.append((low, map3d_estep_pool(ctx, sub, marginals=True, dev=sdev)))
        else:
            parts.append((low, map3d_estep_pools_adaptive(ctx, sub, dev=sdev)))
    return merge_results3d(parts, n), low


def _pool_part(ctx: GpuContext, net: ProposalNet, pool, k: int, min_mass: float, marginals: bool):
    """propose + restricted E-step of one pool's confident particles; the rest
    are returned as a view for the exhaustive fallback."""
    props, mass = net.propose(pool, k)
    low = np.flatnonzero(mass < min_mass)
    high = np.flatnonzero(mass >= min_mass)
    parts = []
    if high.size:
        sub = pool if low.size == 0 else take_pool(pool, high)
        parts.append((high, ctx.map2d_estep_pool(sub, marginals=marginals, proposals=props[high])))
    return pool.nr_images, parts, props, mass, low, (take_pool(pool, low) if low.size else None)


def _learned_stream(lanes, execs, pools, k, min_mass, marginals):
    """learned_estep_pools over an iterator of pools (e.g. pools still being
    copied in): each pool is worked on as it arrives, the exhaustive call for
    all fallback particles comes last."""
    ctx = lanes[0][0]
    if execs is None:
        staged = [_pool_part(*lanes[0], pool, k, min_mass, marginals) for pool in pools]
    else:
        futs = [execs[q % len(lanes)].submit(_pool_part, *lanes[q % len(lanes)], pool, k, min_mass, marginals)
                for q, pool in enumerate(pools)]
        staged = [f.result() for f in futs]
    fallback = [f for *_, f in staged if f is not None]
    sums = {}
    if fallback:
        r = ctx.map2d_estep_pool(concat_pools(fallback), marginals=marginals)
        off = 0
        for _, parts, _, _, low, _ in staged:
            if low.size:
                parts.append((low, {name: a[off:off + low.size] for name, a in r.items() if name in PARTICLE_OUTPUTS}))
                off += low.size
        sums = {name: a for name, a in r.items() if name not in PARTICLE_OUTPUTS}
    out = []
    for q, (n, parts, props, mass, low, _) in enumerate(staged):
        res = merge_results(parts, n)
        for name, a in sums.items():
            if q == 0:
                res[name] = res[name] + a if name in res else a.copy()
            elif name not in res:
                res[name] = np.zeros_like(a)
        out.append((res, props, mass, low))
    return out
