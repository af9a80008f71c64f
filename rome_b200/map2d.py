"""Host-side mirror of the MAP2D E-step interface (Map2dOptimizer_old).

`Map2dPool` carries the arrays that ``expectationSomeParticles()``
(src/map2d_optimizer.cpp:802-854) reads from the optimizer's globals;
`GpuContext.map2d_estep_pool` sends them through the C ABI
(``rome_gpu_map2d_estep_pool``) and returns the reference's outputs under the
reference's names.  `store_weighted_sums` is the host-side remainder
(src/map2d_optimizer.cpp:1314-1414).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Dict, Optional

import numpy as np

from . import abi


@dataclasses.dataclass
class Map2dPool:
    ori_size: int
    current_size: int
    coarse_size: int
    nr_classes: int
    nr_groups: int
    adaptive_oversampling: int
    over_psi: list            # per pass [nr_psi][nr_over_rot]
    over_trans_x: list        # per pass [nr_trans][nr_over_trans]
    over_trans_y: list
    trans_x: np.ndarray       # [nr_trans]
    trans_y: np.ndarray
    Fimg_real: np.ndarray     # [P][F(current)]
    Fimg_imag: np.ndarray
    Fimg_nomask_real: np.ndarray
    Fimg_nomask_imag: np.ndarray
    Fctf: np.ndarray
    highres_Xi2: np.ndarray
    old_offsetx: np.ndarray
    old_offsety: np.ndarray
    group: np.ndarray         # int32, 0-based
    sigma2_noise: np.ndarray  # [G][ori/2+1]
    Mresol_fine: np.ndarray   # int32
    Mresol_coarse: np.ndarray
    pdf_class: np.ndarray
    pdf_direction: np.ndarray
    prior_offsetx_class: np.ndarray
    prior_offsety_class: np.ndarray
    sigma2_offset: float
    sigma2_fudge: float = 1.0
    adaptive_fraction: float = 0.999
    do_ctf_correction: int = 1
    refs_are_ctf_corrected: int = 1
    do_map: int = 1
    iclass_min: int = 0
    iclass_max: int = -1
    # optional restricted search: [P][nr_proposals] orientations (class * nr_psi + psi), ascending
    proposals: Optional[np.ndarray] = None
    # optional, staged pools only: device image row of each particle (a subset without a copy)
    particle_rows: Optional[np.ndarray] = None

    @property
    def nr_images(self) -> int:
        return int(self.Fimg_real.shape[0])

    @property
    def nr_psi(self) -> int:
        return int(np.asarray(self.over_psi[0]).shape[0])

    @property
    def nr_trans(self) -> int:
        return int(np.asarray(self.trans_x).shape[0])

    def npass(self) -> int:
        return 2 if self.adaptive_oversampling > 0 else 1

    def xsize(self, ipass: int) -> int:
        nor = np.asarray(self.over_psi[ipass]).shape[1]
        notr = np.asarray(self.over_trans_x[ipass]).shape[1]
        return self.nr_classes * self.nr_psi * nor * self.nr_trans * notr


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def pack_pool(p: Map2dPool):
    """Build the RomeMap2dPool struct; returns (struct, keepalive list)."""
    keep = []

    def d(a):
        a = _f64(a)
        keep.append(a)
        return abi.dptr(a)

    def i(a):
        a = _i32(a)
        keep.append(a)
        return abi.iptr(a)

    s = abi.RomeMap2dPool()
    s.nr_images = p.nr_images
    s.ori_size, s.current_size, s.coarse_size = p.ori_size, p.current_size, p.coarse_size
    s.nr_classes, s.nr_groups = p.nr_classes, p.nr_groups
    s.iclass_min = p.iclass_min
    s.iclass_max = p.iclass_max if p.iclass_max >= 0 else p.nr_classes - 1
    s.adaptive_oversampling = p.adaptive_oversampling
    s.nr_psi, s.nr_trans = p.nr_psi, p.nr_trans
    for ip in range(p.npass()):
        s.over_psi[ip] = d(p.over_psi[ip])
        s.over_trans_x[ip] = d(p.over_trans_x[ip])
        s.over_trans_y[ip] = d(p.over_trans_y[ip])
    s.trans_x, s.trans_y = d(p.trans_x), d(p.trans_y)
    s.Fimg_real, s.Fimg_imag = d(p.Fimg_real), d(p.Fimg_imag)
    s.Fimg_nomask_real, s.Fimg_nomask_imag = d(p.Fimg_nomask_real), d(p.Fimg_nomask_imag)
    s.Fctf = d(p.Fctf)
    s.highres_Xi2 = d(p.highres_Xi2)
    s.old_offsetx, s.old_offsety = d(p.old_offsetx), d(p.old_offsety)
    s.group = i(p.group)
    s.sigma2_noise = d(p.sigma2_noise)
    s.Mresol_fine, s.Mresol_coarse = i(p.Mresol_fine), i(p.Mresol_coarse)
    s.pdf_class, s.pdf_direction = d(p.pdf_class), d(p.pdf_direction)
    s.prior_offsetx_class, s.prior_offsety_class = d(p.prior_offsetx_class), d(p.prior_offsety_class)
    s.sigma2_offset, s.sigma2_fudge, s.adaptive_fraction = p.sigma2_offset, p.sigma2_fudge, p.adaptive_fraction
    s.do_ctf_correction, s.refs_are_ctf_corrected, s.do_map = p.do_ctf_correction, p.refs_are_ctf_corrected, p.do_map
    if p.proposals is not None:
        pr = _i32(p.proposals)
        keep.append(pr)
        s.proposals = abi.iptr(pr)
        s.nr_proposals = int(pr.shape[1])
    if p.particle_rows is not None:
        s.particle_rows = i(p.particle_rows)
    return s, keep


def alloc_outputs(p: Map2dPool, checkpoints: bool = False, marginals: bool = False):
    """Zeroed output arrays + the RomeMap2dPoolOut struct pointing at them."""
    P, K, G, oF = p.nr_images, p.nr_classes, p.nr_groups, p.ori_size // 2 + 1
    o: Dict[str, np.ndarray] = {}
    for name in ["min_diff2", "sum_weight", "significant_weight", "wsum_norm_correction", "pmax", "psi", "xoff",
                 "yoff", "nr_sign"]:
        o[name] = np.zeros(P, np.float64)
    o["cls"] = np.zeros(P, np.int32)
    o["wsum_sigma2_noise"] = np.zeros((G, oF), np.float64)
    for name in ["wsum_pdf_class", "wsum_pdf_direction", "wsum_prior_offsetx_class", "wsum_prior_offsety_class"]:
        o[name] = np.zeros(K, np.float64)
    o["wsum_sigma2_offset"] = np.zeros(1, np.float64)
    o["wsum_sumw_group"] = np.zeros(G, np.float64)
    s = abi.RomeMap2dPoolOut()
    for name, arr in o.items():
        setattr(s, name, abi.iptr(arr) if arr.dtype == np.int32 else abi.dptr(arr))
    if checkpoints:
        for ip in range(p.npass()):
            o[f"diff2_{ip}"] = np.zeros((P, p.xsize(ip)), np.float64)
            o[f"weight_{ip}"] = np.zeros((P, p.xsize(ip)), np.float64)
            s.diff2[ip] = abi.dptr(o[f"diff2_{ip}"])
            s.weight[ip] = abi.dptr(o[f"weight_{ip}"])
        o["Mcoarse_significant"] = np.zeros((P, p.nr_classes * p.nr_psi * p.nr_trans), np.int8)
        s.Mcoarse_significant = abi.cptr(o["Mcoarse_significant"])
    if marginals:
        o["post_class_psi"] = np.zeros((P, p.nr_classes * p.nr_psi), np.float64)
        s.post_class_psi = abi.dptr(o["post_class_psi"])
    return s, o


DEVICE_FIELDS = ["Fimg_real", "Fimg_imag", "Fimg_nomask_real", "Fimg_nomask_imag", "Fctf"]
# fields with one entry (row) per particle
PARTICLE_FIELDS = DEVICE_FIELDS + ["highres_Xi2", "old_offsetx", "old_offsety", "group"]
# outputs with one entry per particle (the rest are sums over the pool)
PARTICLE_OUTPUTS = ["min_diff2", "sum_weight", "significant_weight", "wsum_norm_correction", "pmax", "psi", "xoff",
                    "yoff", "nr_sign", "cls", "post_class_psi"]


def pin_pool(p: Map2dPool) -> Map2dPool:
    """The pool with its image arrays copied into page-locked host memory
    (what GpuContext.staged / stage_pool_async read from)."""
    import torch
    rep = {}
    for name in DEVICE_FIELDS:
        a = _f64(getattr(p, name))
        t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[...] = a
        rep[name] = t.numpy()  # keeps the pinned tensor alive
    return dataclasses.replace(p, **rep)


def _device_index(idx: np.ndarray, device):
    """An int64 index array on the device, copied by a kernel from page-locked
    memory (rome_gpu_copy_from_host) rather than by a copy engine that may be
    busy with a large transfer of the next pool."""
    import torch
    n = len(idx)
    npad = n + (n & 1)  # 16-byte multiple
    h = torch.zeros(npad, dtype=torch.int64, pin_memory=True)
    h.numpy()[:n] = idx
    d = torch.empty(npad, dtype=torch.int64, device=device)
    lib = abi.load_library()
    ctx = _index_ctx(device)
    rc = lib.rome_gpu_copy_from_host(ctx.h, C.c_void_p(d.data_ptr()), C.c_void_p(h.data_ptr()), 8 * npad,
                                     C.c_void_p(torch.cuda.current_stream(device).cuda_stream))
    if rc != abi.ROME_OK:
        raise RomeError(rc, lib.rome_gpu_last_error(ctx.h).decode())
    torch.cuda.current_stream(device).synchronize()  # h is released on return
    return d[:n]


_INDEX_CTX = {}


def _index_ctx(device):
    """A context per device for the small index copies (error reporting only)."""
    dev = device.index if hasattr(device, "index") and device.index is not None else 0
    if dev not in _INDEX_CTX:
        _INDEX_CTX[dev] = GpuContext(dev)
    return _INDEX_CTX[dev]


def take_pool(p, idx: np.ndarray):
    """The particles `idx` of a pool, in that order: a Map2dPool, or a
    StagedPool whose images are gathered on the device (its host image
    fields become zero-width placeholders: only the device copies are read)."""
    idx = np.asarray(idx, np.int64)
    if isinstance(p, StagedPool):
        # no copy: the subset reads its rows of the staged images (particle_rows)
        base = dataclasses.replace(p.pool)
        for name in PARTICLE_FIELDS:
            a = getattr(p.pool, name)
            setattr(base, name, np.empty((len(idx), 0)) if name in DEVICE_FIELDS else np.ascontiguousarray(a[idx]))
        if p.pool.proposals is not None:
            base.proposals = np.ascontiguousarray(p.pool.proposals[idx])
        rows = idx if p.pool.particle_rows is None else np.asarray(p.pool.particle_rows)[idx]
        base.particle_rows = np.ascontiguousarray(rows, np.int32)
        return StagedPool(base, p.dev)
    q = dataclasses.replace(p)
    for name in PARTICLE_FIELDS:
        setattr(q, name, np.ascontiguousarray(getattr(p, name)[idx]))
    if p.proposals is not None:
        q.proposals = np.ascontiguousarray(p.proposals[idx])
    return q


def concat_pools(pools):
    """One pool holding the particles of several pools of the same model and
    sampling, in order (StagedPools: device images concatenated on the device)."""
    if isinstance(pools[0], StagedPool):
        import torch

        dev0 = next(iter(pools[0].dev.values())).device
        idx = [None if q.pool.particle_rows is None
               else _device_index(np.asarray(q.pool.particle_rows, np.int64), dev0) for q in pools]

        def rows(q, ix, name):
            return q.dev[name] if ix is None else q.dev[name].index_select(0, ix)

        base = concat_pools([dataclasses.replace(q.pool, particle_rows=None) for q in pools])
        out = StagedPool(base, {name: torch.cat([rows(q, ix, name) for q, ix in zip(pools, idx)])
                                for name in pools[0].dev})
        torch.cuda.current_stream(next(iter(out.dev.values())).device).synchronize()
        return out
    q = dataclasses.replace(pools[0])
    for name in PARTICLE_FIELDS:
        setattr(q, name, np.concatenate([getattr(x, name) for x in pools]))
    if pools[0].proposals is not None:
        q.proposals = np.concatenate([x.proposals for x in pools])
    return q


def merge_results(parts, n: int) -> Dict[str, np.ndarray]:
    """Outputs of E-steps over disjoint particle subsets [(idx, result)] of one
    pool of n particles: per-particle outputs scattered back to pool order,
    pool sums added."""
    out: Dict[str, np.ndarray] = {}
    for idx, r in parts:
        for name, a in r.items():
            if name in PARTICLE_OUTPUTS:
                if name not in out:
                    out[name] = np.zeros((n,) + a.shape[1:], a.dtype)
                out[name][idx] = a
            else:
                out[name] = out[name] + a if name in out else a.copy()
    return out


@dataclasses.dataclass
class StagedPool:
    """A pool whose particle images were copied to the device (GpuContext.stage_pool)."""
    pool: Map2dPool
    dev: dict

    @property
    def nr_images(self) -> int:
        return self.pool.nr_images


class RomeError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"rome_gpu error {code}: {msg}")
        self.code = code


class GpuContext:
    """One device context of librome_b200 (``rome_gpu_create``)."""

    def __init__(self, device: int = 0, precision: str = "fp32", deterministic: bool = False, profile: bool = False,
                 workspace_limit: int = 0):
        self.lib = abi.load_library()
        self.device = device
        cfg = abi.RomeGpuConfig(abi.PRECISIONS[precision], int(deterministic), int(workspace_limit), int(profile))
        h = C.c_void_p()
        rc = self.lib.rome_gpu_create(device, C.byref(cfg), C.byref(h))
        if rc != 0:
            raise RomeError(rc, "rome_gpu_create failed")
        self.h = h

    def _check(self, rc: int):
        if rc != abi.ROME_OK:
            msg = self.lib.rome_gpu_last_error(self.h)
            raise RomeError(rc, msg.decode() if msg else "")

    def close(self):
        if self.h:
            self.lib.rome_gpu_destroy(self.h)
            self.h = None

    def invalidate_projections(self) -> None:
        """rome_gpu_invalidate_projections: the next pool recomputes the orientation projections."""
        self._check(self.lib.rome_gpu_invalidate_projections(self.h))

    @property
    def torch_device(self) -> str:
        return f"cuda:{self.device}"

    def backprojector_doubles(self) -> int:
        """Doubles of all classes' back-projectors (data [K][vox][2], then weight [K][vox])."""
        n = C.c_size_t()
        self._check(self.lib.rome_gpu_backprojector_size(self.h, C.byref(n)))
        return int(n.value)

    def copy_backprojectors_to(self, buf) -> None:
        """Library back-projectors -> a flat FP64 torch tensor on this device (device to device)."""
        self._bp_copy(0, buf)

    def copy_backprojectors_from(self, buf) -> None:
        """A flat FP64 torch tensor on this device -> the library's back-projectors."""
        self._bp_copy(1, buf)

    def _bp_copy(self, to_library: int, buf) -> None:
        import torch
        if not (buf.dtype == torch.float64 and buf.is_contiguous() and buf.numel() == self.backprojector_doubles()):
            raise ValueError("back-projector buffer: a contiguous float64 tensor of backprojector_doubles() elements")
        if not (buf.is_cuda and buf.device.index == self.device):
            raise ValueError(f"back-projector buffer must live on cuda:{self.device}")
        stream = torch.cuda.current_stream(self.device)
        self._check(self.lib.rome_gpu_backprojector_device_copy(self.h, to_library, C.c_void_p(buf.data_ptr()),
                                                                C.c_void_p(stream.cuda_stream)))

    def wait_selftest(self, limit_seconds: float) -> float:
        """rome_gpu_wait_selftest: a bounded device wait that nothing ends;
        raises RomeError(ROME_ERR_TIMEOUT) after about limit_seconds and
        records the measured wait in self.last_wait_seconds."""
        w = np.zeros(1)
        self.last_wait_seconds = None
        rc = self.lib.rome_gpu_wait_selftest(self.h, float(limit_seconds), abi.dptr(w))
        self.last_wait_seconds = float(w[0])
        self._check(rc)
        return self.last_wait_seconds

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_precision(self, precision: str):
        self._check(self.lib.rome_gpu_set_precision(self.h, abi.PRECISIONS[precision]))

    def set_projectors(self, data: np.ndarray, ori_size: int, r_max: int, padding_factor: int = 2):
        """data: [K][pad][pad/2+1][2] (2D) or [K][pad][pad][pad/2+1][2] (3D)."""
        data = _f64(data)
        ref_dim = 3 if data.ndim == 5 else 2
        K, pad = data.shape[0], data.shape[-3]
        self._check(self.lib.rome_gpu_set_projectors(self.h, ref_dim, K, ori_size, pad, r_max, padding_factor,
                                                     abi.dptr(data)))
        self.proj_shape = data.shape

    def get_backprojector(self, iclass: int):
        shp = self.proj_shape[1:]
        data = np.zeros(shp, np.float64)
        weight = np.zeros(shp[:-1], np.float64)
        self._check(self.lib.rome_gpu_get_backprojector(self.h, iclass, abi.dptr(data), abi.dptr(weight)))
        return data, weight

    def add_backprojectors(self, src: "GpuContext", clear: bool = True):
        """This context's back-projectors += src's (same device), src zeroed when clear."""
        self._check(self.lib.rome_gpu_add_backprojectors(self.h, src.h, int(clear)))

    def backproject_images(self, iclass: int, Fimg_real, Fimg_imag, Fctf, poses: np.ndarray):
        """rome_gpu_backproject_images: images [n][F] at poses [n][5] (rot,
        tilt, psi, xoff, yoff) into class iclass's 3D back-projector.  The
        spectra (and Fctf, or None) are numpy arrays or torch CUDA tensors
        (float64, contiguous) on this context's device."""
        poses = _f64(poses).reshape(-1, 5)
        n = poses.shape[0]
        on_dev = not isinstance(Fimg_real, np.ndarray)
        if on_dev:
            arrs = [Fimg_real, Fimg_imag] + ([Fctf] if Fctf is not None else [])
            for a in arrs:
                if not (a.is_cuda and a.is_contiguous() and str(a.dtype) == "torch.float64"
                        and a.device.index == self.device and a.shape[0] == n):
                    raise ValueError("device spectra must be contiguous float64 CUDA tensors of n rows on this device")
            ptr = [a.data_ptr() for a in arrs] + ([None] if Fctf is None else [])
        else:
            arrs = [_f64(Fimg_real), _f64(Fimg_imag)] + ([_f64(Fctf)] if Fctf is not None else [])
            for a in arrs:
                if a.shape[0] != n:
                    raise ValueError("spectra and poses disagree on the number of images")
            ptr = [a.ctypes.data for a in arrs] + ([None] if Fctf is None else [])
        F = int(arrs[0].shape[1])
        size = int(round((1 + 2 * F) ** 0.5)) - 1       # F = size * (size / 2 + 1)
        if size * (size // 2 + 1) != F or any(int(a.shape[1]) != F for a in arrs):
            raise ValueError(f"{F} coefficients per image is not a half-plane transform of a square image")
        self._check(self.lib.rome_gpu_backproject_images(self.h, iclass, n, size, ptr[0], ptr[1], ptr[2],
                                                         abi.dptr(poses), int(on_dev)))

    def set_backprojector(self, iclass: int, data: np.ndarray, weight: np.ndarray):
        self._check(self.lib.rome_gpu_set_backprojector(self.h, iclass, abi.dptr(_f64(data)), abi.dptr(_f64(weight))))

    def map2d_estep_pool(self, p, checkpoints: bool = False, marginals: bool = False,
                         proposals: Optional[np.ndarray] = None) -> Dict[str, np.ndarray]:
        """E-step of one pool.  `p` is a Map2dPool (host arrays) or a
        StagedPool whose particle images already live on the device.
        `proposals` ([P][k] orientation indices, ascending) restricts the
        search; `marginals` returns the posterior summed per (class, psi)."""
        base = p.pool if isinstance(p, StagedPool) else p
        if proposals is not None:
            base = dataclasses.replace(base, proposals=proposals)
        s, keep = pack_pool(base)
        if isinstance(p, StagedPool):
            import torch
            # the library's stream does not wait for torch's: tensors made on it must be complete
            torch.cuda.current_stream(self.device).synchronize()
            for name, t in p.dev.items():
                setattr(s, name, C.cast(C.c_void_p(t.data_ptr()), abi._DP))
            s.inputs_on_device = 1
        so, o = alloc_outputs(base, checkpoints, marginals)
        self._check(self.lib.rome_gpu_map2d_estep_pool(self.h, C.byref(s), C.byref(so)))
        return o

    def stage_pool(self, p: Map2dPool) -> "StagedPool":
        """Copy the pool's particle images to the device once (torch owns the memory)."""
        import torch
        dev = {}
        for name in DEVICE_FIELDS:
            dev[name] = torch.from_numpy(_f64(getattr(p, name))).to(f"cuda:{self.device}")
        torch.cuda.synchronize(self.device)
        return StagedPool(p, dev)

    def stage_pool_async(self, p: Map2dPool, stream):
        """Start copying the pool's images (page-locked host arrays) to the
        device on a side stream (a torch.cuda.Stream); returns the StagedPool
        and a torch event to wait on before it is used.  The copy runs while
        the context computes an earlier pool."""
        import torch
        dev = {}
        with torch.cuda.stream(stream):
            for name in DEVICE_FIELDS:
                dev[name] = torch.from_numpy(_f64(getattr(p, name))).to(f"cuda:{self.device}", non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(stream)
        return StagedPool(p, dev), ev

    def staged(self, pools):
        """Yield the host pools as StagedPools, copying pool k + 1 to the
        device while the caller works on pool k."""
        import torch
        # one side stream per context: device blocks the caching allocator
        # hands out on it are reused by the next call's copies
        side = getattr(self, "_side", None)
        if side is None:
            side = self._side = torch.cuda.Stream(device=self.device)
        nxt = self.stage_pool_async(pools[0], side) if len(pools) else None
        for k in range(len(pools)):
            cur, ev = nxt
            if k + 1 < len(pools):
                nxt = self.stage_pool_async(pools[k + 1], side)
            ev.synchronize()
            yield cur

    def map2d_estep_pools(self, pools, run=None):
        """E-steps of a sequence of host pools with the copy of pool k + 1
        overlapping the E-step of pool k.  `run(staged_pool)` performs one
        E-step (default: map2d_estep_pool); returns the list of its results."""
        run = run or self.map2d_estep_pool
        return [run(q) for q in self.staged(pools)]

    @staticmethod
    def h2d_bytes(p: Map2dPool) -> int:
        return sum(int(_f64(getattr(p, n)).nbytes) for n in DEVICE_FIELDS) + p.nr_images * (3 * 8 + 4)

    @staticmethod
    def d2h_bytes(p: Map2dPool) -> int:
        P, K, G = p.nr_images, p.nr_classes, p.nr_groups
        return P * (9 * 8 + 4) + 8 * (G * (p.ori_size // 2 + 1) + 4 * K + G + 1)

    def get_timings(self) -> Dict[str, dict]:
        t = abi.RomeGpuTimings()
        self._check(self.lib.rome_gpu_get_timings(self.h, C.byref(t)))
        out = {name: {"ms": t.ms[q], "launches": t.launches[q], "flops": t.flops[q], "bytes": t.bytes[q]}
               for q, name in enumerate(abi.PHASES)}
        out["total_launches"] = t.total_launches
        return out

    def reset_timings(self):
        self._check(self.lib.rome_gpu_reset_timings(self.h))

    def select_significant(self, weights: np.ndarray, sum_weight: np.ndarray, adaptive_fraction: float):
        w = _f64(weights)
        n, ln = w.shape
        sw = np.zeros(n, np.float64)
        ns = np.zeros(n, np.float64)
        self._check(self.lib.rome_gpu_select_significant(self.h, n, ln, abi.dptr(w), abi.dptr(_f64(sum_weight)),
                                                          adaptive_fraction, abi.dptr(sw), abi.dptr(ns)))
        return sw, ns

    def reconstruct(self, iclass: int, ori_size: int, ref_dim: int, tau2: np.ndarray, tau2_fudge: float,
                    normalise: float, gridding_nr_iter: int = 10, do_map: bool = True, minres_map: int = 5):
        oF = ori_size // 2 + 1
        rin = abi.RomeReconIn(iclass, gridding_nr_iter, int(do_map), minres_map, tau2_fudge, normalise,
                              abi.dptr(_f64(tau2)))
        keep_tau = _f64(tau2)
        rin.tau2_in = abi.dptr(keep_tau)
        vol = np.zeros((ori_size,) * ref_dim, np.float64)
        o = {"vol": vol, "tau2": np.zeros(oF), "sigma2": np.zeros(oF), "data_vs_prior": np.zeros(oF)}
        rout = abi.RomeReconOut(abi.dptr(vol), abi.dptr(o["tau2"]), abi.dptr(o["sigma2"]),
                                abi.dptr(o["data_vs_prior"]))
        self._check(self.lib.rome_gpu_reconstruct(self.h, C.byref(rin), C.byref(rout)))
        return o


def store_weighted_sums(p: Map2dPool, est: Dict[str, np.ndarray], power_imgs: np.ndarray, norm_in: np.ndarray,
                        avg_norm_correction: float, do_norm_correction: bool, Mresol_fine: np.ndarray,
                        sigma2_noise: np.ndarray, wsum: Dict[str, np.ndarray]):
    """storeWeightedSums (src/map2d_optimizer.cpp:1314-1414), host side, FP64.

    Returns per-particle (dLL, NORM) and accumulates into ``wsum`` (keys
    wsum_sigma2_noise, wsum_avg_norm_correction, wsum_LL, wsum_ave_Pmax).
    """
    cur_F = p.current_size // 2 + 1
    ori_F = p.ori_size // 2 + 1
    P = p.nr_images
    dll = np.zeros(P)
    norm = np.array(norm_in, np.float64).copy()
    wnc = est["wsum_norm_correction"].copy()
    for i in range(P):
        g = int(p.group[i])
        for ires in range(cur_F, ori_F):
            wsum["wsum_sigma2_noise"][g, ires] += power_imgs[i, ires]
            wnc[i] += power_imgs[i, ires]
        if do_norm_correction:
            old = norm[i] / avg_norm_correction
            norm[i] = old * np.sqrt(wnc[i] * 2.)
            wsum["wsum_avg_norm_correction"] += old * np.sqrt(wnc[i] * 2.)
        ires = Mresol_fine
        sel = ires > 0
        logsigma2 = float(np.sum(np.log(2. * np.pi * sigma2_noise[g][ires[sel]])))
        if est["sum_weight"][i] == 0:
            raise RomeError(abi.ROME_ERR_NUMERIC, "exp_sum_weight[ipart]==0")
        dll[i] = np.log(est["sum_weight"][i]) - est["min_diff2"][i] - logsigma2
        wsum["wsum_LL"] += dll[i]
        wsum["wsum_ave_Pmax"] += est["pmax"][i]
    return dll, norm



def _scalar(v) -> float:
    """A model scalar given as a number or a one-element array."""
    return float(np.asarray(v, np.float64).ravel()[0])


def _running_sum(v) -> float:
    """Sum in index order (the reference's sequential FP64 loops)."""
    t = 0.0
    for x in np.asarray(v, np.float64).ravel():
        t += float(x)
    return t


def maximization_other_parameters(model: Dict, wsum: Dict, Npix_per_shell: np.ndarray, do_norm_correction: bool,
                                  do_ctf_correction: bool) -> Dict:
    """maximizationOtherParameters of MAP2D (src/map2d_optimizer.cpp:1984-2045),
    host side, FP64: the model parameters other than the class maps, from the
    iteration's summed weights.  ``model`` (updated in place and returned):
    pdf_class [K], pdf_direction [K], prior_offsetx_class / prior_offsety_class
    [K], sigma2_offset, sigma2_noise [G][ori/2+1], avg_norm_correction, LL,
    ave_Pmax, refs_are_ctf_corrected.  ``wsum``: the wsum_* sums of every pool
    of the iteration (wsum_pdf_class, wsum_pdf_direction,
    wsum_prior_offsetx_class / y, wsum_sigma2_offset, wsum_sigma2_noise,
    wsum_sumw_group, wsum_avg_norm_correction, wsum_LL, wsum_ave_Pmax).

    With W the sum of wsum_pdf_class: pdf_class and pdf_direction are their
    sums over W, a class's prior offset is its weighted offset sum over its
    weight (0 for a class without weight), sigma2_offset = wsum_sigma2_offset
    / 2W, sigma2_noise[g][n] = wsum_sigma2_noise[g][n] / (2 wsum_sumw_group[g]
    Npix_per_shell[n]), avg_norm_correction (with norm correction) =
    wsum_avg_norm_correction / W, LL = wsum_LL, ave_Pmax = wsum_ave_Pmax / W;
    with CTF correction the references count as CTF-corrected from now on."""
    wpc = np.asarray(wsum["wsum_pdf_class"], np.float64).ravel()
    K = wpc.size
    W = _running_sum(wpc)
    if do_norm_correction:
        model["avg_norm_correction"] = _scalar(wsum["wsum_avg_norm_correction"]) / W
    model["pdf_class"] = wpc / W
    px = np.asarray(wsum["wsum_prior_offsetx_class"], np.float64).ravel()
    py = np.asarray(wsum["wsum_prior_offsety_class"], np.float64).ravel()
    model["prior_offsetx_class"] = np.array([px[k] / wpc[k] if wpc[k] > 0. else 0. for k in range(K)])
    model["prior_offsety_class"] = np.array([py[k] / wpc[k] if wpc[k] > 0. else 0. for k in range(K)])
    model["pdf_direction"] = np.asarray(wsum["wsum_pdf_direction"], np.float64).reshape(K) / W
    model["sigma2_offset"] = _scalar(wsum["wsum_sigma2_offset"]) / (2. * W)
    sumw = np.asarray(wsum["wsum_sumw_group"], np.float64).ravel()
    npix = np.asarray(Npix_per_shell, np.float64).ravel()
    with np.errstate(divide="ignore", invalid="ignore"):  # an empty group or shell divides by 0, as in C
        model["sigma2_noise"] = np.asarray(wsum["wsum_sigma2_noise"], np.float64) / (2. * sumw[:, None] * npix[None, :])
    if do_ctf_correction:
        model["refs_are_ctf_corrected"] = True
    model["LL"] = _scalar(wsum["wsum_LL"])
    model["ave_Pmax"] = _scalar(wsum["wsum_ave_Pmax"]) / W
    return model


def load_dump(path: str) -> Dict[str, np.ndarray]:
    """Read a reference-harness dump directory (manifest.txt + *.bin)."""
    import os
    out = {}
    with open(os.path.join(path, "manifest.txt")) as f:
        for line in f:
            parts = line.split()
            if not parts:
                continue
            name, dt, shape = parts[0], parts[1], tuple(int(x) for x in parts[2:])
            arr = np.fromfile(os.path.join(path, name + ".bin"), dtype=np.dtype(dt))
            out[name] = arr.reshape(shape)
    return out


def pool_from_dump(d: Dict[str, np.ndarray], pool: int = 0) -> Map2dPool:
    """Map2dPool with the inputs the reference harness recorded for one pool."""
    pp = f"pool{pool}_"
    os_ = int(d["adaptive_oversampling"][0])
    npass = 2 if os_ > 0 else 1
    return Map2dPool(
        ori_size=int(d["ori_size"][0]), current_size=int(d["current_size"][0]),
        coarse_size=int(d["coarse_size"][0]), nr_classes=int(d["nr_classes"][0]),
        nr_groups=int(d["nr_groups"][0]), adaptive_oversampling=os_,
        over_psi=[d[f"pass{ip}_over_psi"] for ip in range(npass)],
        over_trans_x=[d[f"pass{ip}_over_trans_x"] for ip in range(npass)],
        over_trans_y=[d[f"pass{ip}_over_trans_y"] for ip in range(npass)],
        trans_x=d["trans_x"], trans_y=d["trans_y"],
        Fimg_real=d[pp + "Fimg_real"], Fimg_imag=d[pp + "Fimg_imag"],
        Fimg_nomask_real=d[pp + "Fimg_nomask_real"], Fimg_nomask_imag=d[pp + "Fimg_nomask_imag"],
        Fctf=d[pp + "Fctf"], highres_Xi2=d[pp + "highres_Xi2"],
        old_offsetx=d[pp + "old_offsetx"], old_offsety=d[pp + "old_offsety"], group=d[pp + "group"],
        sigma2_noise=d["sigma2_noise"], Mresol_fine=d["Mresol_fine"], Mresol_coarse=d["Mresol_coarse"],
        pdf_class=d["pdf_class"], pdf_direction=d["pdf_direction"],
        prior_offsetx_class=d["prior_offsetx_class"], prior_offsety_class=d["prior_offsety_class"],
        sigma2_offset=float(d["sigma2_offset"][0]), sigma2_fudge=float(d["sigma2_fudge"][0]),
        adaptive_fraction=float(d["adaptive_fraction"][0]),
        do_ctf_correction=int(d["do_ctf_correction"][0]),
        refs_are_ctf_corrected=int(d["refs_are_ctf_corrected"][0]), do_map=int(d["do_map"][0]),
    )
