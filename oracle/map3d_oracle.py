"""CPU restatement of the MAP3D squared differences, coarse and fine pass
(numpy; the translation phases through the C oracle's restatement of the
5000-entry table).

Test infrastructure only: imported by tests/, never by the product package.

For one pool it restates
* the windowing of the fine-size masked image and CTF to the pass size
  (windowFourierTransform / windowTransform, ParticleModel::
  preShiftedImagesCtfsAndInvSigma2s, src/exp_model.cpp:1015-1049) and
  Minvsigma2 = 1 / (sigma2_fudge * sigma2_noise[group][ires]), 0 at
  ires <= 0 (:1078-1092);
* the image norm of the cross-correlation mode (exp_local_sqrtXi2, :1037-1045);
* the translated images (shiftImageInFourierTransform, src/image.h:1478-1575,
  via oracle/estep_oracle.c);
* MyProjector::project, trilinear branch (src/reconstruct.cpp:226-410);
* applyCtfToClass (src/map3d_optimizer.cpp:1040-1067, CTF and the group's
  intensity scale) and get_diff (:1079-1123), maximum-likelihood and
  cross-correlation forms, over every (class, direction) the coarse pass
  visits (pdf_class > 0 and pdf_direction > 0, :1205-1206), and over the
  over-sampled neighbours of the coarse-significant points in the fine pass
  (:1261-1372);
* from the recorded fine-pass weights, updateOtherParams with get_wdiff2
  (:1426-1602, :2059-2236): the model sums, the norm-correction sums and the
  scale-correction spectra;
* backProjection (:2242-2466) with MyBackProjector::backproject
  (src/reconstruct.cpp:977-1164): the pool's class back-projectors.
"""
from __future__ import annotations

import numpy as np

from oracle import oracle_py


def window_half(F: np.ndarray, cur: int, cs: int) -> np.ndarray:
    """[cur][cur/2+1] half-plane -> [cs][cs/2+1] (rows wrap negative)."""
    csF = cs // 2 + 1
    out = np.zeros((cs, csF), F.dtype)
    F = F.reshape(cur, cur // 2 + 1)
    for i in range(cs):
        ip = i if i < csF else i - cs
        out[i] = F[ip if ip >= 0 else ip + cur, :csF]
    return out


def euler_matrix(rot: float, tilt: float, psi: float) -> np.ndarray:
    return np.asarray(oracle_py.euler_matrix(rot, tilt, psi)).reshape(3, 3)


def _lin(a, lo, hi):
    return lo + (hi - lo) * a


def project3d(data: np.ndarray, r_max: int, padding: int, A: np.ndarray, cs: int) -> np.ndarray:
    """MyProjector::project (trilinear): the [cs][cs/2+1] slice of the
    [pad][pad][pad/2+1] complex volume `data` at orientation A."""
    pad = data.shape[0]
    csF = cs // 2 + 1
    my_r_max = min(r_max, cs // 2)
    shift = -int(np.float32(pad) / np.float32(2.0))
    Ainv = A.T * float(padding)
    out = np.zeros((cs, csF), np.complex128)
    rows, xs = [], []
    for i in range(cs):
        if i <= my_r_max:
            y = i
        elif i >= cs - my_r_max:
            y = i - cs
        else:
            continue
        for x in range(my_r_max + 1):
            if x * x + y * y <= my_r_max * my_r_max:
                rows.append((i, x, y))
    i_, x_, y_ = (np.array(v) for v in zip(*rows))
    xd, yd = x_.astype(np.float64), y_.astype(np.float64)
    xp = Ainv[0, 0] * xd + Ainv[0, 1] * yd
    yp = Ainv[1, 0] * xd + Ainv[1, 1] * yd
    zp = Ainv[2, 0] * xd + Ainv[2, 1] * yd
    neg = xp < 0
    xp, yp, zp = np.where(neg, -xp, xp), np.where(neg, -yp, yp), np.where(neg, -zp, zp)
    x0 = np.floor(xp).astype(np.int64)
    fx = xp - x0
    y0f = np.floor(yp).astype(np.int64)
    fy = yp - y0f
    y0 = y0f - shift
    z0f = np.floor(zp).astype(np.int64)
    fz = zp - z0f
    z0 = z0f - shift
    d = lambda z, y, x: data[z, y, x]  # noqa: E731
    d000, d001 = d(z0, y0, x0), d(z0, y0, x0 + 1)
    d010, d011 = d(z0, y0 + 1, x0), d(z0, y0 + 1, x0 + 1)
    d100, d101 = d(z0 + 1, y0, x0), d(z0 + 1, y0, x0 + 1)
    d110, d111 = d(z0 + 1, y0 + 1, x0), d(z0 + 1, y0 + 1, x0 + 1)
    vals = []
    for part in (np.real, np.imag):
        dx00, dx01 = _lin(fx, part(d000), part(d001)), _lin(fx, part(d100), part(d101))
        dx10, dx11 = _lin(fx, part(d010), part(d011)), _lin(fx, part(d110), part(d111))
        dxy0, dxy1 = _lin(fy, dx00, dx10), _lin(fy, dx01, dx11)
        vals.append(_lin(fz, dxy0, dxy1))
    re, im = vals
    im = np.where(neg, -1.0 * im, im)
    out[i_, x_] = re + 1j * im
    return out


def coarse_diff2(d: dict, pool: int = 0, cc: bool = False):
    """The coarse pass of pool `pool` of a MAP3D dump (the arrays
    oracle/ref_harness/map3d_dump records): diff2 [P][K][ndir][npsi][ntr]
    (NaN where the reference computes nothing), and in cross-correlation
    mode the image norms [P].  The shifted images are the coarse
    translations around each particle's rounded old offset."""
    pp = f"pool{pool}_"
    g = lambda k: d[k] if k in d or not k.startswith(pp) else d["pool0_" + k[len(pp):]]  # noqa: E731
    ic = lambda k: int(np.asarray(d[k]).ravel()[0])  # noqa: E731
    ori, cur, cs = ic("ori_size"), ic("current_size"), ic("coarse_size")
    K, ndir, npsi, ntr = ic("nr_classes"), ic("nr_dir"), ic("nr_psi"), ic("nr_trans")
    r_max, padding = ic("projector_r_max"), ic("projector_padding_factor")
    apply_ctf = ic("do_ctf_correction") and ic("refs_are_ctf_corrected")
    scale = ic("do_scale_correction")
    fudge = float(np.asarray(d["sigma2_fudge"]).ravel()[0])
    P = int(np.asarray(d[pp + "nr_images"]).ravel()[0])
    csF = cs // 2 + 1
    angles = g(pp + "pass0_angles")            # [ndir][npsi][1][3]
    otx, oty = g(pp + "pass0_over_trans_x"), g(pp + "pass0_over_trans_y")  # [ntr][1]
    vol = d["projector_data"][..., 0] + 1j * d["projector_data"][..., 1]
    mres = np.asarray(d["Mresol_coarse"]).reshape(cs, csF)
    s2 = np.asarray(d["sigma2_noise"])
    group = np.asarray(g(pp + "group")).astype(int)
    xi2 = np.asarray(g(pp + "highres_Xi2"))
    pdir, pcls = np.asarray(d["pdf_direction"]).reshape(K, ndir), np.asarray(d["pdf_class"])
    sc = np.asarray(d["scale_correction"]) if scale else None
    # projections of every visited (class, direction, psi)
    proj = {}
    for k in range(K):
        for j in range(ndir):
            if not (pcls[k] > 0 and pdir[k, j] > 0):
                continue
            for p in range(npsi):
                proj[(k, j, p)] = project3d(vol[k], r_max, padding, euler_matrix(*angles[j, p, 0]), cs)
    out = np.full((P, K, ndir, npsi, ntr), np.nan)
    norms = np.zeros(P)
    for i in range(P):
        X = window_half(g(pp + "Fimg_real")[i] + 1j * g(pp + "Fimg_imag")[i], cur, cs)
        ctf = window_half(np.asarray(g(pp + "Fctf")[i]), cur, cs)
        minv = np.where(mres > 0, 1.0 / (fudge * s2[group[i]][np.maximum(mres, 0)]), 0.0)
        norms[i] = np.sqrt(np.sum(X.real * X.real + X.imag * X.imag))
        shifted = []
        for t in range(ntr):
            sr, si = oracle_py.shift_image(X.real.ravel(), X.imag.ravel(), cs, float(otx[t, 0]), float(oty[t, 0]),
                                           ori)
            shifted.append((sr + 1j * si).reshape(cs, csF))
        for (k, j, p), P3 in proj.items():
            Pc = P3 * ctf if apply_ctf else P3.copy()
            if scale:  # check_scale raises a scale below 0.001 to 0.001 (:1000-1018)
                Pc = Pc * max(float(sc[group[i]]), 0.001)
            for t in range(ntr):
                Xt = shifted[t]
                if cc:
                    num = -np.sum(Pc.real * Xt.real + Pc.imag * Xt.imag)
                    out[i, k, j, p, t] = num / (np.sqrt(np.sum(Pc.real ** 2 + Pc.imag ** 2)) * norms[i])
                else:
                    dr, di = Pc.real - Xt.real, Pc.imag - Xt.imag
                    out[i, k, j, p, t] = (np.sum((dr * dr + di * di) * minv) + xi2[i]) / 2
    return out, norms


def fine_diff2(d: dict, pool: int = 0, cc: bool = False):
    """The fine pass of pool `pool` of a MAP3D dump at the current size: for
    every coarse point the reference recorded as significant
    (exp_Mcoarse_significant, coarse index ((class * ndir + dir) * npsi +
    psi) * ntr + itrans), the 8 over-rotations x 4 over-translations in the
    reference's list order (getAllSquaredDifferencesFine,
    src/map3d_optimizer.cpp:1261-1372: class, dir, psi, then ihidden =
    (itrans * nor + iover_rot) * notr + iover_trans).  Returns per particle
    (kdp [n], ihidden [n], diff2 [n])."""
    pp = f"pool{pool}_"
    g = lambda k: d[k] if k in d or not k.startswith(pp) else d["pool0_" + k[len(pp):]]  # noqa: E731
    ic = lambda k: int(np.asarray(d[k]).ravel()[0])  # noqa: E731
    ori, cur = ic("ori_size"), ic("current_size")
    K, ndir, npsi, ntr = ic("nr_classes"), ic("nr_dir"), ic("nr_psi"), ic("nr_trans")
    r_max, padding = ic("projector_r_max"), ic("projector_padding_factor")
    apply_ctf = ic("do_ctf_correction") and ic("refs_are_ctf_corrected")
    scale = ic("do_scale_correction")
    fudge = float(np.asarray(d["sigma2_fudge"]).ravel()[0])
    P = int(np.asarray(d[pp + "nr_images"]).ravel()[0])
    curF = cur // 2 + 1
    angles = g(pp + "pass1_angles")                                        # [ndir][npsi][nor][3]
    otx, oty = g(pp + "pass1_over_trans_x"), g(pp + "pass1_over_trans_y")  # [ntr][notr]
    nor, notr = angles.shape[2], otx.shape[1]
    vol = d["projector_data"][..., 0] + 1j * d["projector_data"][..., 1]
    mres = np.asarray(d["Mresol_fine"]).reshape(cur, curF)
    s2 = np.asarray(d["sigma2_noise"])
    group = np.asarray(g(pp + "group")).astype(int)
    xi2 = np.asarray(g(pp + "highres_Xi2"))
    mc = np.asarray(d[pp + "pass0_Mcoarse_significant"])
    sc = np.asarray(d["scale_correction"]) if scale else None
    cache = {}
    out = []
    for i in range(P):
        X = (g(pp + "Fimg_real")[i] + 1j * g(pp + "Fimg_imag")[i]).reshape(cur, curF)
        ctf = np.asarray(g(pp + "Fctf")[i]).reshape(cur, curF)
        minv = np.where(mres > 0, 1.0 / (fudge * s2[group[i]][np.maximum(mres, 0)]), 0.0)
        norm = np.sqrt(np.sum(X.real * X.real + X.imag * X.imag))
        shifted = {}
        kdp, ih, val = [], [], []
        for q in np.flatnonzero(mc[i]):
            kd_p, itr = divmod(int(q), ntr)
            kd, p = divmod(kd_p, npsi)
            k, j = divmod(kd, ndir)
            for o in range(nor):
                key = (k, j, p, o)
                if key not in cache:
                    cache[key] = project3d(vol[k], r_max, padding, euler_matrix(*angles[j, p, o]), cur)
                Pc = cache[key] * ctf if apply_ctf else cache[key].copy()
                if scale:  # check_scale raises a scale below 0.001 to 0.001 (:1000-1018)
                    Pc = Pc * max(float(sc[group[i]]), 0.001)
                for t in range(notr):
                    if (itr, t) not in shifted:
                        sr, si = oracle_py.shift_image(X.real.ravel(), X.imag.ravel(), cur, float(otx[itr, t]),
                                                       float(oty[itr, t]), ori)
                        shifted[(itr, t)] = (sr + 1j * si).reshape(cur, curF)
                    Xt = shifted[(itr, t)]
                    if cc:
                        v = -np.sum(Pc.real * Xt.real + Pc.imag * Xt.imag) / (
                            np.sqrt(np.sum(Pc.real ** 2 + Pc.imag ** 2)) * norm)
                    else:
                        dr, di = Pc.real - Xt.real, Pc.imag - Xt.imag
                        v = (np.sum((dr * dr + di * di) * minv) + xi2[i]) / 2
                    kdp.append(kd_p)
                    ih.append((itr * nor + o) * notr + t)
                    val.append(v)
        # the reference's order: by (class, dir, psi), then ihidden ascending within it
        order = np.lexsort((np.array(ih), np.array(kdp))) if kdp else np.zeros(0, int)
        out.append((np.array(kdp)[order], np.array(ih)[order], np.array(val)[order]))
    return out


def update_other_params(d: dict, pool: int = 0):
    """updateOtherParams of one pool (src/map3d_optimizer.cpp:2059-2236 and
    CoarseAndFineSearch::updateModel :1484-1602) from the fine-pass weights,
    exp_significant_weight and exp_sum_weight the reference recorded: every
    fine hypothesis with w >= significant_weight, normalised by the sum,
    adds w |Frefctf - X_t|^2 per pixel of resolution shell ires > -1 to
    wsum_sigma2_noise[group][ires] and to the particle's norm-correction sum,
    w to wsum_pdf_class, wsum_pdf_direction and wsum_sumw_group, and
    w |prior - old offset - translation|^2 to wsum_sigma2_offset; with scale
    correction, at the shells whose data_vs_prior exceeds 3 for the class,
    w Re(Frefctf conj X_t) and w |Frefctf|^2 to the particle's XA/AA spectra
    (get_wdiff2 :1426-1482, binned :2090-2112)."""
    from oracle.select3d_oracle import lists_from_dump
    pp = f"pool{pool}_"
    g = lambda k: d[k] if k in d or not k.startswith(pp) else d["pool0_" + k[len(pp):]]  # noqa: E731
    ic = lambda k: int(np.asarray(d[k]).ravel()[0])  # noqa: E731
    ori, cur = ic("ori_size"), ic("current_size")
    K, ndir, npsi, G = ic("nr_classes"), ic("nr_dir"), ic("nr_psi"), ic("nr_groups")
    r_max, padding = ic("projector_r_max"), ic("projector_padding_factor")
    apply_ctf = ic("do_ctf_correction") and ic("refs_are_ctf_corrected")
    scale = ic("do_scale_correction")
    oF, curF = ori // 2 + 1, cur // 2 + 1
    angles = g(pp + "pass1_angles")
    otx, oty = g(pp + "pass1_over_trans_x"), g(pp + "pass1_over_trans_y")
    nor, notr = angles.shape[2], otx.shape[1]
    vol = d["projector_data"][..., 0] + 1j * d["projector_data"][..., 1]
    mres = np.asarray(d["Mresol_fine"]).reshape(cur, curF)
    group = np.asarray(g(pp + "group")).astype(int)
    sc = np.asarray(d["scale_correction"]) if scale else None
    dvp = np.asarray(d["data_vs_prior_before"]).reshape(K, oF)
    prx, pry = np.asarray(d["prior_offsetx_class"]), np.asarray(d["prior_offsety_class"])
    sig, sumw = g(pp + "pass1_significant_weight"), g(pp + "pass1_sum_weight")
    lists = lists_from_dump(d, pp + "pass1_weight_")
    P = len(lists)
    out = {"wsum_sigma2_noise": np.zeros((G, oF)), "wsum_pdf_class": np.zeros(K),
           "wsum_pdf_direction": np.zeros((K, ndir)), "wsum_sigma2_offset": 0.0, "wsum_sumw_group": np.zeros(G),
           "wsum_norm_correction": np.zeros(P), "XA": np.zeros((P, oF)), "AA": np.zeros((P, oF))}
    sel = mres > -1
    ires_sel = mres[sel]
    for i, pl in enumerate(lists):
        X = (g(pp + "Fimg_real")[i] + 1j * g(pp + "Fimg_imag")[i]).reshape(cur, curF)
        ctf = np.asarray(g(pp + "Fctf")[i]).reshape(cur, curF)
        gi = group[i]
        for kdp, h, w in zip(pl.kdp, pl.ihidden, pl.value):
            if w < sig[i]:
                continue
            w = w / sumw[i]
            kd, p = divmod(int(kdp), npsi)
            k, j = divmod(kd, ndir)
            itr, rest = divmod(int(h), nor * notr)
            o, t = divmod(rest, notr)
            Pc = project3d(vol[k], r_max, padding, euler_matrix(*angles[j, p, o]), cur)
            if apply_ctf:
                Pc = Pc * ctf
            if scale:
                Pc = Pc * max(float(sc[gi]), 0.001)
            sr, si = oracle_py.shift_image(X.real.ravel(), X.imag.ravel(), cur, float(otx[itr, t]), float(oty[itr, t]),
                                           ori)
            Xt = (sr + 1j * si).reshape(cur, curF)
            dr, di = Pc.real - Xt.real, Pc.imag - Xt.imag
            wd = (w * (dr * dr + di * di))[sel]
            np.add.at(out["wsum_sigma2_noise"][gi], ires_sel, wd)
            out["wsum_norm_correction"][i] += wd.sum()
            out["wsum_pdf_class"][k] += w
            out["wsum_pdf_direction"][k, j] += w
            out["wsum_sumw_group"][gi] += w
            ox = prx[k] - float(g(pp + "old_offsetx")[i]) - float(otx[itr, t])
            oy = pry[k] - float(g(pp + "old_offsety")[i]) - float(oty[itr, t])
            out["wsum_sigma2_offset"] += w * (ox * ox + oy * oy)
            if scale:
                s_pix = sel & (dvp[k][np.maximum(mres, 0)] > 3.0)
                ir = mres[s_pix]
                np.add.at(out["XA"][i], ir, (w * (Pc.real * Xt.real + Pc.imag * Xt.imag))[s_pix])
                np.add.at(out["AA"][i], ir, (w * (Pc.real * Pc.real + Pc.imag * Pc.imag))[s_pix])
    return out


def backproject3d(data: np.ndarray, weight: np.ndarray, f2d: np.ndarray, fw: np.ndarray, r_max: int, padding: int,
                  A: np.ndarray) -> None:
    """MyBackProjector::backproject, trilinear branch, A not inverted
    (src/reconstruct.cpp:977-1164): adds the [f][f/2+1] slice `f2d` and its
    weights `fw` (only where fw > 0) into the [pad][pad][pad/2+1] complex
    `data` and real `weight` at orientation A, in place.  Rows past r_max
    from the top and the x = 0 column of negative rows are skipped (the
    FFTW layout stores that column twice)."""
    pad = data.shape[0]
    f = f2d.shape[0]
    shift = -int(float(pad) / 2.0)
    Ainv = A.T * float(padding)
    rows = []
    for i in range(f):
        if i <= r_max:
            y, first_x = i, 0
        elif i >= f - r_max:
            y, first_x = i - f, 1
        else:
            continue
        for x in range(first_x, r_max + 1):
            if x * x + y * y <= r_max * r_max and fw[i, x] > 0.0:
                rows.append((i, x, y))
    if not rows:
        return
    i_, x_, y_ = (np.array(v) for v in zip(*rows))
    val, wgt = f2d[i_, x_], fw[i_, x_]
    xd, yd = x_.astype(np.float64), y_.astype(np.float64)
    xp = Ainv[0, 0] * xd + Ainv[0, 1] * yd
    yp = Ainv[1, 0] * xd + Ainv[1, 1] * yd
    zp = Ainv[2, 0] * xd + Ainv[2, 1] * yd
    neg = xp < 0
    xp, yp, zp = np.where(neg, -xp, xp), np.where(neg, -yp, yp), np.where(neg, -zp, zp)
    val = np.where(neg, np.conj(val), val)
    x0 = np.floor(xp).astype(np.int64)
    fx = xp - x0
    y0f = np.floor(yp).astype(np.int64)
    fy = yp - y0f
    z0f = np.floor(zp).astype(np.int64)
    fz = zp - z0f
    y0, z0 = y0f - shift, z0f - shift
    mfx, mfy, mfz = 1.0 - fx, 1.0 - fy, 1.0 - fz
    for dz, dy, dx, c in ((0, 0, 0, mfz * mfy * mfx), (0, 0, 1, mfz * mfy * fx), (0, 1, 0, mfz * fy * mfx),
                          (0, 1, 1, mfz * fy * fx), (1, 0, 0, fz * mfy * mfx), (1, 0, 1, fz * mfy * fx),
                          (1, 1, 0, fz * fy * mfx), (1, 1, 1, fz * fy * fx)):
        idx = (z0 + dz, y0 + dy, x0 + dx)
        np.add.at(data, idx, c * val)
        np.add.at(weight, idx, c * wgt)


def back_projection(d: dict, pool: int = 0):
    """backProjection of one pool (doBackProjectionNew and
    prepareNomaskImageAndMinvsigma2s, src/map3d_optimizer.cpp:2242-2466):
    the unmasked image times Minvsigma2 * CTF (the fine pass's Minvsigma2,
    its origin put back to 1 / (sigma2_fudge * sigma2_noise[group][0]); 1
    without MAP, CTF 1 without CTF correction, CTF times the group's clamped
    scale with scale correction), translated by each significant fine
    hypothesis (w >= significant_weight) and summed with weight w / sum per
    (class, direction, psi, over-rotation), the weights summing
    Minvsigma2 * CTF^2 * w / sum; each sum then back-projected into its
    class at the over-rotation's orientation.  Returns (data [K][pad][pad]
    [pad/2+1] complex, weight [K][pad][pad][pad/2+1])."""
    from oracle.select3d_oracle import lists_from_dump
    pp = f"pool{pool}_"
    g = lambda k: d[k] if k in d or not k.startswith(pp) else d["pool0_" + k[len(pp):]]  # noqa: E731
    ic = lambda k: int(np.asarray(d[k]).ravel()[0])  # noqa: E731
    ori, cur = ic("ori_size"), ic("current_size")
    K, ndir, npsi = ic("nr_classes"), ic("nr_dir"), ic("nr_psi")
    r_max, padding = ic("projector_r_max"), ic("projector_padding_factor")
    do_map, do_ctf, scale = ic("do_map"), ic("do_ctf_correction"), ic("do_scale_correction")
    fudge = float(np.asarray(d["sigma2_fudge"]).ravel()[0])
    curF = cur // 2 + 1
    angles = g(pp + "pass1_angles")
    otx, oty = g(pp + "pass1_over_trans_x"), g(pp + "pass1_over_trans_y")
    nor, notr = angles.shape[2], otx.shape[1]
    mres = np.asarray(d["Mresol_fine"]).reshape(cur, curF)
    s2 = np.asarray(d["sigma2_noise"])
    group = np.asarray(g(pp + "group")).astype(int)
    sc = np.asarray(d["scale_correction"])
    sig, sumw = g(pp + "pass1_significant_weight"), g(pp + "pass1_sum_weight")
    pad = d["projector_data"].shape[1]
    data = np.zeros((K, pad, pad, pad // 2 + 1), np.complex128)
    weight = np.zeros((K, pad, pad, pad // 2 + 1))
    for i, pl in enumerate(lists_from_dump(d, pp + "pass1_weight_")):
        gi = group[i]
        if do_map:
            minv = np.where(mres > 0, 1.0 / (fudge * s2[gi][np.maximum(mres, 0)]), 0.0)
            minv[0, 0] = 1.0 / (fudge * s2[gi][0])
        else:
            minv = np.ones((cur, curF))
        ctf = np.asarray(g(pp + "Fctf")[i]).reshape(cur, curF) if do_ctf else np.ones((cur, curF))
        if scale:
            ctf = ctf * max(float(sc[gi]), 0.001)
        mc = minv * ctf
        Xn = (g(pp + "Fimg_nomask_real")[i] * mc.ravel()) + 1j * (g(pp + "Fimg_nomask_imag")[i] * mc.ravel())
        w2 = mc * ctf
        sums = {}
        for kdp, h, w in zip(pl.kdp, pl.ihidden, pl.value):
            if w < sig[i]:
                continue
            w = w / sumw[i]
            itr, rest = divmod(int(h), nor * notr)
            o, t = divmod(rest, notr)
            sr, si = oracle_py.shift_image(Xn.real, Xn.imag, cur, float(otx[itr, t]), float(oty[itr, t]), ori)
            key = (int(kdp), o)
            if key not in sums:
                sums[key] = [np.zeros((cur, curF), np.complex128), np.zeros((cur, curF))]
            sums[key][0] += (sr + 1j * si).reshape(cur, curF) * w
            sums[key][1] += w2 * w
        for (kdp, o), (fr, fw) in sums.items():
            kd, p = divmod(kdp, npsi)
            k, j = divmod(kd, ndir)
            backproject3d(data[k], weight[k], fr, fw, r_max, padding, euler_matrix(*angles[j, p, o]))
    return data, weight
