"""Host side of the MAP3D E-step: the pool description that mirrors
``Map3dOptimizer_old``'s expectation state (src/map3d_optimizer.cpp:615-727)
and the call into ``rome_gpu_map3d_estep_pool``.

The sampling tables are the caller's: ``angles[p][dir][psi][over_rot]`` is
what ``SamplingGrid::setOrientation`` returns for pass p
(src/sampling.cpp), ``over_trans_x/y[p]`` are ``exp_over_trans_x/y``.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Dict, Optional

import numpy as np

from . import abi
from .map2d import GpuContext, RomeError, _f64, _i32, _running_sum, _scalar

__all__ = ["Map3dPool", "map3d_estep_pool", "take_pool3d", "merge_results3d", "store_weighted_sums",
           "maximization_other_parameters", "pool3d_from_dump", "fine_lists_from_dump"]


@dataclasses.dataclass
class Map3dPool:
    ori_size: int
    current_size: int
    coarse_size: int
    nr_classes: int
    nr_groups: int
    nr_dir: int
    angles: list            # [2] arrays [ndir][npsi][nor][3]
    over_trans_x: list      # [2] arrays [ntr][notr]
    over_trans_y: list
    trans_x: np.ndarray
    trans_y: np.ndarray
    Fimg_real: np.ndarray   # [P][F(current_size)]
    Fimg_imag: np.ndarray
    Fimg_nomask_real: np.ndarray
    Fimg_nomask_imag: np.ndarray
    Fctf: np.ndarray
    highres_Xi2: np.ndarray
    old_offsetx: np.ndarray
    old_offsety: np.ndarray
    group: np.ndarray
    sigma2_noise: np.ndarray      # [G][ori/2+1]
    Mresol_fine: np.ndarray
    Mresol_coarse: np.ndarray
    pdf_class: np.ndarray         # [K]
    pdf_direction: np.ndarray     # [K][ndir]
    prior_offsetx_class: np.ndarray
    prior_offsety_class: np.ndarray
    sigma2_offset: float
    sigma2_fudge: float = 1.0
    adaptive_fraction: float = 0.999
    do_ctf_correction: bool = True
    refs_are_ctf_corrected: bool = True
    do_map: bool = True
    iclass_min: int = 0
    iclass_max: int = -1
    adaptive_oversampling: int = 1
    # cross-correlation mode ((iter == 1 && do_firstiter_cc) || do_always_cc, src/map3d_optimizer.cpp:907)
    do_cross_correlation: bool = False
    # intensity-scale correction: mlModel.scale_correction [G] and data_vs_prior_class [K][ori/2+1]
    do_scale_correction: bool = False
    scale_correction: Optional[np.ndarray] = None
    data_vs_prior_class: Optional[np.ndarray] = None
    # optional restricted coarse search: [P][nr_proposals] coarse orientations (class * nr_dir + dir) * nr_psi + psi
    proposals: Optional[np.ndarray] = None

    @property
    def nr_images(self) -> int:
        return int(self.Fimg_real.shape[0])

    @property
    def nr_psi(self) -> int:
        return int(self.angles[0].shape[1])

    @property
    def nr_trans(self) -> int:
        return int(self.over_trans_x[0].shape[0])

    @property
    def ncoarse(self) -> int:
        return self.nr_classes * self.nr_dir * self.nr_psi * self.nr_trans


def _pack(p: Map3dPool):
    keep = []

    def d(a):
        a = _f64(a)
        keep.append(a)
        return abi.dptr(a)

    def i(a):
        a = _i32(a)
        keep.append(a)
        return abi.iptr(a)

    s = abi.RomeMap3dPool()
    s.nr_images, s.ori_size, s.current_size, s.coarse_size = p.nr_images, p.ori_size, p.current_size, p.coarse_size
    s.nr_classes, s.nr_groups = p.nr_classes, p.nr_groups
    s.iclass_min = p.iclass_min
    s.iclass_max = p.iclass_max if p.iclass_max >= 0 else p.nr_classes - 1
    s.adaptive_oversampling = p.adaptive_oversampling
    s.nr_dir, s.nr_psi, s.nr_trans = p.nr_dir, p.nr_psi, p.nr_trans
    for q in range(2):
        s.angles[q] = d(p.angles[q])
        s.over_trans_x[q] = d(p.over_trans_x[q])
        s.over_trans_y[q] = d(p.over_trans_y[q])
    s.trans_x, s.trans_y = d(p.trans_x), d(p.trans_y)
    s.Fimg_real, s.Fimg_imag = d(p.Fimg_real), d(p.Fimg_imag)
    s.Fimg_nomask_real, s.Fimg_nomask_imag = d(p.Fimg_nomask_real), d(p.Fimg_nomask_imag)
    s.Fctf, s.highres_Xi2 = d(p.Fctf), d(p.highres_Xi2)
    s.old_offsetx, s.old_offsety, s.group = d(p.old_offsetx), d(p.old_offsety), i(p.group)
    s.sigma2_noise, s.Mresol_fine, s.Mresol_coarse = d(p.sigma2_noise), i(p.Mresol_fine), i(p.Mresol_coarse)
    s.pdf_class, s.pdf_direction = d(p.pdf_class), d(p.pdf_direction)
    s.prior_offsetx_class, s.prior_offsety_class = d(p.prior_offsetx_class), d(p.prior_offsety_class)
    s.sigma2_offset, s.sigma2_fudge, s.adaptive_fraction = p.sigma2_offset, p.sigma2_fudge, p.adaptive_fraction
    s.do_ctf_correction, s.refs_are_ctf_corrected = int(p.do_ctf_correction), int(p.refs_are_ctf_corrected)
    s.do_map = int(p.do_map)
    s.do_scale_correction = int(p.do_scale_correction)
    if p.do_scale_correction:
        s.scale_correction, s.data_vs_prior_class = d(p.scale_correction), d(p.data_vs_prior_class)
    s.do_cross_correlation = int(p.do_cross_correlation)
    s.inputs_on_device = 0
    if p.proposals is not None:
        pr = _i32(p.proposals)
        keep.append(pr)
        s.proposals = abi.iptr(pr)
        s.nr_proposals = int(pr.shape[1])
    return s, keep


def map3d_estep_pool(ctx: GpuContext, p: Map3dPool, checkpoints: bool = False,
                     fine_capacity: Optional[int] = None, marginals: bool = False,
                     proposals: Optional[np.ndarray] = None, dev: Optional[dict] = None) -> Dict[str, np.ndarray]:
    """One pool through ``rome_gpu_map3d_estep_pool``; returns the per-particle
    results, the model sums of this pool, and (with ``checkpoints``) the coarse
    diff2 array, Mcoarse_significant and the fine-pass lists.  ``proposals``
    ([P][k] coarse orientations, ascending) restricts the coarse pass;
    ``marginals`` returns the coarse posterior per coarse orientation
    (``post_coarse`` [P][K * nr_dir * nr_psi])."""
    if proposals is not None:
        p = dataclasses.replace(p, proposals=proposals)
    P, K, G, oF = p.nr_images, p.nr_classes, p.nr_groups, p.ori_size // 2 + 1
    s, keep = _pack(p)
    if dev is not None:
        # images already on the device (torch tensors named like the pool fields)
        import torch
        torch.cuda.current_stream(ctx.device).synchronize()
        for name, t in dev.items():
            setattr(s, name, C.cast(C.c_void_p(t.data_ptr()), abi._DP))
        s.inputs_on_device = 1
    o: Dict[str, np.ndarray] = {}
    so = abi.RomeMap3dPoolOut()
    for name in ("min_diff2", "sum_weight", "significant_weight", "wsum_norm_correction", "pmax", "rot", "tilt",
                 "psi", "xoff", "yoff", "nr_sign"):
        o[name] = np.zeros(P)
        setattr(so, name, abi.dptr(o[name]))
    o["cls"] = np.zeros(P, np.int32)
    so.cls = abi.iptr(o["cls"])
    o["wsum_sigma2_noise"] = np.zeros((G, oF))
    o["wsum_pdf_class"] = np.zeros(K)
    o["wsum_pdf_direction"] = np.zeros((K, p.nr_dir))
    o["wsum_sigma2_offset"] = np.zeros(1)
    o["wsum_sumw_group"] = np.zeros(G)
    for name in ("wsum_sigma2_noise", "wsum_pdf_class", "wsum_pdf_direction", "wsum_sigma2_offset",
                 "wsum_sumw_group"):
        setattr(so, name, abi.dptr(o[name]))
    if checkpoints:
        for q in range(2):
            for name in ("pass_min_diff2", "pass_sum_weight", "pass_significant_weight"):
                o[f"{name}{q}"] = np.zeros(P)
                getattr(so, name)[q] = abi.dptr(o[f"{name}{q}"])
        o["coarse_diff2"] = np.zeros((P, p.ncoarse))
        so.coarse_diff2 = abi.dptr(o["coarse_diff2"])
        o["Mcoarse_significant"] = np.zeros((P, p.ncoarse), np.int8)
        so.Mcoarse_significant = abi.cptr(o["Mcoarse_significant"])
        cap = fine_capacity if fine_capacity is not None else P * p.ncoarse * 32
        o["fine_count"] = np.zeros(P, np.int32)
        o["fine_index"] = np.zeros(cap, np.int64)
        o["fine_diff2"] = np.zeros(cap)
        o["fine_weight"] = np.zeros(cap)
        so.fine_capacity = cap
        so.fine_count = abi.iptr(o["fine_count"])
        so.fine_index = o["fine_index"].ctypes.data_as(C.POINTER(C.c_long))
        so.fine_diff2 = abi.dptr(o["fine_diff2"])
        so.fine_weight = abi.dptr(o["fine_weight"])
    if marginals:
        o["post_coarse"] = np.zeros((P, K * p.nr_dir * p.nr_psi))
        so.post_coarse = abi.dptr(o["post_coarse"])
    if p.do_scale_correction:
        for name in ("wsum_scale_correction_XA", "wsum_scale_correction_AA"):
            o[name] = np.zeros((P, oF))
            setattr(so, name, abi.dptr(o[name]))
    ctx._check(ctx.lib.rome_gpu_map3d_estep_pool(ctx.h, C.byref(s), C.byref(so)))
    del keep
    if checkpoints:
        n = int(o["fine_count"].sum())
        for name in ("fine_index", "fine_diff2", "fine_weight"):
            o[name] = o[name][:n]
    return o


def store_weighted_sums(p: Map3dPool, est: Dict[str, np.ndarray], power_imgs: np.ndarray, norm_in: np.ndarray,
                        avg_norm_correction: float, do_norm_correction: bool, wsum: Dict[str, np.ndarray]):
    """storeWeightedSums (src/map3d_optimizer.cpp:1933-2045), host side, FP64,
    on the outputs of map3d_estep_pool (``est``: sum_weight, min_diff2, pmax,
    wsum_norm_correction and, with scale correction, the
    wsum_scale_correction_XA/AA spectra).

    Per particle, in order: the power spectrum beyond the current size is
    added to the group's wsum_sigma2_noise and to the norm-correction sum;
    with norm correction NORM = NORM / avg_norm_correction * sqrt(2 sum)
    and that value is added to wsum_avg_norm_correction; with scale
    correction XA / scale and AA / scale^2 (the scale as stored, without the
    clamp the E-step applies) are added to the group's
    wsum_signal_product_spectra / wsum_reference_power_spectra; dLL is
    -min_diff2 in cross-correlation mode, else log(sum_weight) - min_diff2 -
    the sum over the current-size pixels with ires > 0 of log(2 pi sigma2).
    Returns per-particle (dLL, NORM) and accumulates into ``wsum`` (keys
    wsum_sigma2_noise, wsum_avg_norm_correction, wsum_LL, wsum_ave_Pmax and,
    with scale correction, wsum_signal_product_spectra and
    wsum_reference_power_spectra [G][ori/2+1])."""
    cur_F = p.current_size // 2 + 1
    ori_F = p.ori_size // 2 + 1
    P = p.nr_images
    dll = np.zeros(P)
    norm = np.array(norm_in, np.float64).copy()
    wnc = np.array(est["wsum_norm_correction"], np.float64).copy()
    ires = np.asarray(p.Mresol_fine).ravel()
    ires = ires[ires > 0]
    # the sum over the pixels of log(2 pi sigma2), one per group
    logsigma2 = np.log(2. * np.pi * np.asarray(p.sigma2_noise)[:, ires]).sum(axis=1)
    for i in range(P):
        g = int(p.group[i])
        for r in range(cur_F, ori_F):
            wsum["wsum_sigma2_noise"][g, r] += power_imgs[i, r]
            wnc[i] += power_imgs[i, r]
        if do_norm_correction:
            old = norm[i] / avg_norm_correction
            norm[i] = old * np.sqrt(wnc[i] * 2.)
            wsum["wsum_avg_norm_correction"] += old * np.sqrt(wnc[i] * 2.)
        if p.do_scale_correction:
            s = float(p.scale_correction[g])
            wsum["wsum_signal_product_spectra"][g] += est["wsum_scale_correction_XA"][i] / s
            wsum["wsum_reference_power_spectra"][g] += est["wsum_scale_correction_AA"][i] / (s * s)
        if est["sum_weight"][i] == 0:
            raise RomeError(abi.ROME_ERR_NUMERIC, "exp_sum_weight[ipart]==0")
        if p.do_cross_correlation:
            dll[i] = -est["min_diff2"][i]
        else:
            dll[i] = np.log(est["sum_weight"][i]) - est["min_diff2"][i] - logsigma2[g]
        wsum["wsum_LL"] += dll[i]
        wsum["wsum_ave_Pmax"] += est["pmax"][i]
    return dll, norm



def maximization_other_parameters(model: Dict, wsum: Dict, Npix_per_shell: np.ndarray,
                                  nr_particles_group: np.ndarray, do_norm_correction: bool,
                                  do_scale_correction: bool, do_ctf_correction: bool,
                                  cross_correlation: bool = False, first_iteration_cc: bool = False) -> Dict:
    """maximizationOtherParameters of MAP3D (src/map3d_optimizer.cpp:2620-2798),
    host side, FP64: the model parameters other than the class maps, from the
    iteration's summed weights.  ``model`` (updated in place and returned):
    pdf_class [K], pdf_direction [K][ndir], sigma2_offset, sigma2_noise
    [G][ori/2+1], scale_correction [G], avg_norm_correction, LL, ave_Pmax,
    refs_are_ctf_corrected.  ``wsum``: the wsum_* sums of every pool of the
    iteration (with scale correction also wsum_signal_product_spectra and
    wsum_reference_power_spectra [G][ori/2+1]).

    With W the sum of wsum_pdf_class: avg_norm_correction (with norm
    correction) = wsum_avg_norm_correction / W; with scale correction each
    group's scale is sum(XA) / sum(AA) (1 without reference power), held
    within [median / 5, 5 median] of the groups (the median is element G / 2
    of the sorted scales), then divided by the particle-weighted mean scale;
    pdf_class and pdf_direction are their sums over W, sigma2_offset =
    wsum_sigma2_offset / 2W, sigma2_noise[g][n] = wsum_sigma2_noise[g][n] /
    (2 wsum_sumw_group[g] Npix_per_shell[n]); LL = wsum_LL (over W in
    cross-correlation mode: the mean correlation), ave_Pmax = wsum_ave_Pmax /
    W; with CTF correction the references count as CTF-corrected from now
    on.  The first iteration of -firstiter_cc also low-pass filters the
    class maps and seeds every class from the first; that step stays with
    the caller (ROME_ERR_UNSUPPORTED here)."""
    if first_iteration_cc:
        raise RomeError(abi.ROME_ERR_UNSUPPORTED,
                        "the first -firstiter_cc iteration filters the class maps: the caller's own step")
    wpc = np.asarray(wsum["wsum_pdf_class"], np.float64).ravel()
    K = wpc.size
    W = _running_sum(wpc)
    if do_norm_correction:
        model["avg_norm_correction"] = _scalar(wsum["wsum_avg_norm_correction"]) / W
    if do_scale_correction:
        xa = np.asarray(wsum["wsum_signal_product_spectra"], np.float64)
        aa = np.asarray(wsum["wsum_reference_power_spectra"], np.float64)
        G = xa.shape[0]
        sc = np.empty(G)
        for g in range(G):
            sxa, saa = _running_sum(xa[g]), _running_sum(aa[g])
            sc[g] = sxa / saa if saa > 0. else 1.
        median = float(np.sort(sc)[G // 2])
        avg, nr = 0.0, 0.0
        npg = np.asarray(nr_particles_group).ravel()
        for g in range(G):
            if sc[g] > 5. * median:
                sc[g] = 5. * median
            elif sc[g] < median / 5.:
                sc[g] = median / 5.
            avg += float(npg[g]) * sc[g]
            nr += float(npg[g])
        model["scale_correction"] = sc / (avg / nr)
    model["pdf_class"] = wpc / W
    model["pdf_direction"] = np.asarray(wsum["wsum_pdf_direction"], np.float64).reshape(K, -1) / W
    model["sigma2_offset"] = _scalar(wsum["wsum_sigma2_offset"]) / (2. * W)
    sumw = np.asarray(wsum["wsum_sumw_group"], np.float64).ravel()
    npix = np.asarray(Npix_per_shell, np.float64).ravel()
    with np.errstate(divide="ignore", invalid="ignore"):  # an empty group or shell divides by 0, as in C
        model["sigma2_noise"] = np.asarray(wsum["wsum_sigma2_noise"], np.float64) / (2. * sumw[:, None] * npix[None, :])
    if do_ctf_correction:
        model["refs_are_ctf_corrected"] = True
    model["LL"] = _scalar(wsum["wsum_LL"]) / W if cross_correlation else _scalar(wsum["wsum_LL"])
    model["ave_Pmax"] = _scalar(wsum["wsum_ave_Pmax"]) / W
    return model


# per-particle outputs of map3d_estep_pool (the rest are the pool's model sums)
_PER_PARTICLE = ("min_diff2", "sum_weight", "significant_weight", "wsum_norm_correction", "pmax", "rot", "tilt",
                 "psi", "xoff", "yoff", "nr_sign", "cls", "wsum_scale_correction_XA", "wsum_scale_correction_AA",
                 "post_coarse")
# the per-particle inputs of a Map3dPool
_PARTICLE_FIELDS = ("Fimg_real", "Fimg_imag", "Fimg_nomask_real", "Fimg_nomask_imag", "Fctf", "highres_Xi2",
                    "old_offsetx", "old_offsety", "group")


def take_pool3d(p: Map3dPool, idx) -> Map3dPool:
    """The particles `idx` of a 3D pool, in that order (same model and sampling)."""
    idx = np.asarray(idx, np.int64)
    q = dataclasses.replace(p)
    for name in _PARTICLE_FIELDS:
        setattr(q, name, np.ascontiguousarray(np.asarray(getattr(p, name))[idx]))
    if p.proposals is not None:
        q.proposals = np.ascontiguousarray(p.proposals[idx])
    return q


def merge_results3d(parts, n: int) -> Dict[str, np.ndarray]:
    """Outputs of 3D E-steps over disjoint particle subsets [(idx, result)] of
    one pool of n particles: per-particle outputs scattered back to pool
    order, the pool's model sums added."""
    out: Dict[str, np.ndarray] = {}
    for idx, r in parts:
        for name, a in r.items():
            if name in _PER_PARTICLE:
                if name not in out:
                    out[name] = np.zeros((n,) + a.shape[1:], a.dtype)
                out[name][idx] = a
            else:
                out[name] = out[name] + a if name in out else np.array(a, copy=True)
    return out


def map3d_estep_pools_adaptive(ctx: GpuContext, p: Map3dPool, dev: Optional[dict] = None,
                               min_pool: int = 1) -> Dict[str, np.ndarray]:
    """map3d_estep_pool for a pool whose fine pass may not fit: when the
    union of the pool's coarse-significant orientations needs more device
    memory for its fine projections than is free (the library refuses such a
    pool with ROME_ERR_OOM before any output is written or back-projected),
    the pool is split in halves, recursively, and the halves' results joined:
    per-particle outputs concatenated, model sums added.  Broad posteriors
    (noisy particles searched at HEALPix order 3) are what make this happen;
    the reference runs such particles in the same pools, one at a time."""
    from .map2d import RomeError
    try:
        return map3d_estep_pool(ctx, p, dev=dev)
    except RomeError as e:
        if e.code != abi.ROME_ERR_OOM or "fine pass" not in str(e) or p.nr_images <= max(1, min_pool):
            raise
    h = p.nr_images // 2
    parts = []
    for lo, hi in ((0, h), (h, p.nr_images)):
        q = dataclasses.replace(p)
        for name in ("Fimg_real", "Fimg_imag", "Fimg_nomask_real", "Fimg_nomask_imag", "Fctf", "highres_Xi2",
                     "old_offsetx", "old_offsety", "group"):
            setattr(q, name, np.ascontiguousarray(getattr(p, name)[lo:hi]))
        d = None if dev is None else {k: v[lo:hi] for k, v in dev.items()}
        parts.append(map3d_estep_pools_adaptive(ctx, q, d, min_pool))
    out = {}
    for k in parts[0]:
        if k in _PER_PARTICLE:
            out[k] = np.concatenate([r[k] for r in parts])
        else:
            out[k] = sum(r[k] for r in parts)
    return out


def pool3d_from_dump(d: Dict[str, np.ndarray], pool: int = 0) -> Map3dPool:
    """The E-step inputs of one pool recorded by oracle/ref_harness/map3d_dump."""
    pp = f"pool{pool}_"
    # the sampling tables of an iteration are recorded with its first pool only
    g = lambda k: d[k] if k in d or not k.startswith(pp) else d["pool0_" + k[len(pp):]]  # noqa: E731
    sc = lambda k: float(np.asarray(d[k]).ravel()[0])  # noqa: E731
    ic = lambda k: int(np.asarray(d[k]).ravel()[0])  # noqa: E731
    return Map3dPool(
        ori_size=ic("ori_size"), current_size=ic("current_size"), coarse_size=ic("coarse_size"),
        nr_classes=ic("nr_classes"), nr_groups=ic("nr_groups"), nr_dir=ic("nr_dir"),
        angles=[g(f"{pp}pass0_angles"), g(f"{pp}pass1_angles")],
        over_trans_x=[g(f"{pp}pass0_over_trans_x"), g(f"{pp}pass1_over_trans_x")],
        over_trans_y=[g(f"{pp}pass0_over_trans_y"), g(f"{pp}pass1_over_trans_y")],
        trans_x=g("trans_x"), trans_y=g("trans_y"),
        Fimg_real=g(pp + "Fimg_real"), Fimg_imag=g(pp + "Fimg_imag"),
        Fimg_nomask_real=g(pp + "Fimg_nomask_real"), Fimg_nomask_imag=g(pp + "Fimg_nomask_imag"),
        Fctf=g(pp + "Fctf"), highres_Xi2=g(pp + "highres_Xi2"),
        old_offsetx=g(pp + "old_offsetx"), old_offsety=g(pp + "old_offsety"), group=g(pp + "group"),
        sigma2_noise=g("sigma2_noise"), Mresol_fine=g("Mresol_fine"), Mresol_coarse=g("Mresol_coarse"),
        pdf_class=g("pdf_class"), pdf_direction=g("pdf_direction"),
        prior_offsetx_class=g("prior_offsetx_class"), prior_offsety_class=g("prior_offsety_class"),
        sigma2_offset=sc("sigma2_offset"), sigma2_fudge=sc("sigma2_fudge"),
        adaptive_fraction=sc("adaptive_fraction"), do_ctf_correction=bool(ic("do_ctf_correction")),
        refs_are_ctf_corrected=bool(ic("refs_are_ctf_corrected")), do_map=bool(ic("do_map")),
        adaptive_oversampling=ic("adaptive_oversampling"),
        do_cross_correlation=bool(ic("do_cross_correlation")) if "do_cross_correlation" in d else False,
        do_scale_correction=bool(ic("do_scale_correction")), scale_correction=g("scale_correction"),
        data_vs_prior_class=g("data_vs_prior_before"))


def fine_lists_from_dump(d: Dict[str, np.ndarray], prefix: str, nr_trans: int, nh: int = 32):
    """Exp_Mweight_old lists of a dump (count[P][K][ndir][npsi], ihidden, value)
    re-indexed like the library's fine_index: coarse index (k, dir, psi, trans)
    * nh + over_rot * nr_over_trans + over_trans, with nh = nr_over_rot *
    nr_over_trans (32 in the fine pass, 1 in the coarse pass, where the index
    is the coarse index itself).  Returns per-particle (index, value)."""
    cnt = d[prefix + "count"]
    ih = d[prefix + "ihidden"].astype(np.int64)
    val = d[prefix + "value"]
    P = cnt.shape[0]
    flat = cnt.reshape(P, -1)
    out = []
    q = 0
    for i in range(P):
        idx, v = [], []
        for kdp, n in enumerate(flat[i]):
            if n == 0:
                continue
            h = ih[q:q + n]
            itr = h // nh
            rest = h - itr * nh  # over_rot * nr_over_trans + over_trans
            idx.append((kdp * nr_trans + itr) * nh + rest)
            v.append(val[q:q + n])
            q += n
        out.append((np.concatenate(idx) if idx else np.zeros(0, np.int64),
                     np.concatenate(v) if v else np.zeros(0)))
    return out


def direction_templates(net, projector_data: np.ndarray, r_max: int, p: Map3dPool) -> np.ndarray:
    """Network-input features of every coarse (class, direction) projection at
    psi = 0 without CTF ([K * nr_dir][2][n_r][n_theta]), the templates of
    ProposalNet.init_matched_filter for 3D proposals."""
    from .workload import project3d_np
    K, cur = p.nr_classes, p.current_size
    dirs = np.asarray(p.angles[0])[:, 0, 0, :2]  # (rot, tilt) of each coarse direction
    ang = np.concatenate([dirs, np.zeros((len(dirs), 1))], axis=1)
    slices = np.concatenate([project3d_np(projector_data[k], r_max, ang, cur) for k in range(K)])
    fake = dataclasses.replace(p, Fimg_real=slices.real.reshape(len(slices), -1),
                               Fimg_imag=slices.imag.reshape(len(slices), -1),
                               Fctf=np.ones((len(slices), cur * (cur // 2 + 1))))
    return net.features(fake)
