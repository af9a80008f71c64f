"""CPU restatement of the MAP3D posterior and significance steps (numpy).

Test infrastructure only: imported by tests/, never by the product package.

Restates, on the sparse per-(particle, class, direction, psi) lists the
reference keeps in Exp_Mweight_old (the layout oracle/ref_harness/map3d_dump
records: count[P][K][ndir][npsi], then (ihidden, value) in that loop order):

* MLModel::calculatePdfOffset (src/ml_model.h:231-242);
* Map3dOptimizer_old::convertSquaredDifferencesToWeights
  (src/map3d_optimizer.cpp:1610-1810), maximum-likelihood and
  cross-correlation branches;
* Map3dOptimizer_old::findAllSignificantPoints (:1812-1931): the ascending
  sort of every listed weight (zeros included) and the walk from the largest;
* the metadata of the largest weight (class, rot, tilt, psi, offsets,
  :1787-1804).

decodeOverRotTrans: ihidden = (itrans * nr_over_rot + iover_rot) *
nr_over_trans + iover_trans (src/map3d_optimizer.cpp:1247-1249).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List

import numpy as np

CC_NOT_COMPUTED = -999.123456789  # the reference's marker of a hypothesis it did not score (:1647)


@dataclass
class ParticleList:
    """One particle's hypotheses in the reference's loop order."""
    kdp: np.ndarray      # (class * ndir + dir) * npsi + psi of every entry
    ihidden: np.ndarray  # ihidden of every entry
    value: np.ndarray    # diff2 (or weight) of every entry


def lists_from_dump(d: dict, prefix: str) -> List[ParticleList]:
    """The Exp_Mweight_old lists of a dump (prefix ends in 'diff2_' or 'weight_')."""
    cnt = d[prefix + "count"]
    ih = d[prefix + "ihidden"].astype(np.int64)
    val = d[prefix + "value"]
    P = cnt.shape[0]
    flat = cnt.reshape(P, -1)
    out, q = [], 0
    for i in range(P):
        n = int(flat[i].sum())
        kdp = np.repeat(np.arange(flat.shape[1]), flat[i])
        out.append(ParticleList(kdp, ih[q:q + n], val[q:q + n]))
        q += n
    return out


def calculate_pdf_offset(offset_x, offset_y, prior_x, prior_y, sigma2_offset: float):
    """MLModel::calculatePdfOffset: the Gaussian prior of an offset around
    the class's prior offset (1 or 0 when sigma2_offset is below 1e-4)."""
    tdiff2 = (offset_x - prior_x) * (offset_x - prior_x) + (offset_y - prior_y) * (offset_y - prior_y)
    if sigma2_offset < 0.0001:
        return np.where(tdiff2 > 0.0, 0.0, 1.0)
    return np.exp(tdiff2 / (-2.0 * sigma2_offset)) / (2.0 * np.pi * sigma2_offset)


def weights_ml(pl: ParticleList, min_diff2: float, pdf_direction: np.ndarray, nr_dir: int, nr_psi: int,
               trans_x, trans_y, old_offx: float, old_offy: float, prior_x, prior_y, sigma2_offset: float,
               nr_over_rot: int, nr_over_trans: int):
    """Maximum-likelihood weights of one particle's list: pdf_direction[class][dir]
    * pdf_offset(coarse translation) * exp(-(diff2 - min_diff2)), 0 beyond 700.
    Returns (weights, sum, max weight)."""
    kd = pl.kdp // nr_psi
    cls, idir = kd // nr_dir, kd % nr_dir
    itrans = pl.ihidden // (nr_over_rot * nr_over_trans)
    ox = np.asarray(trans_x)[itrans] + old_offx
    oy = np.asarray(trans_y)[itrans] + old_offy
    pdf_off = calculate_pdf_offset(ox, oy, np.asarray(prior_x)[cls], np.asarray(prior_y)[cls], sigma2_offset)
    w = pdf_direction.reshape(-1)[cls * nr_dir + idir] * pdf_off
    diff = pl.value - min_diff2
    w = np.where(diff > 700.0, 0.0, w * np.exp(-np.minimum(diff, 700.0)))
    s = 0.0
    for x in w:  # the reference's FP64 running sum (one thread's order)
        s += x
    return w, s, float(w.max()) if w.size else np.finfo(float).tiny


def weights_cc(pl: ParticleList):
    """Cross-correlation branch: the computed entry with the smallest value
    (first in loop order at a tie) gets weight 1, the list keeps only it.
    Returns (position in the list, its value)."""
    ok = pl.value != CC_NOT_COMPUTED
    v = np.where(ok, pl.value, np.inf)
    q = int(np.argmin(v))
    return q, float(pl.value[q])


def significance(weights: np.ndarray, sum_weight: float, adaptive_fraction: float):
    """findAllSignificantPoints for one particle: sort every listed weight
    ascending and walk from the largest, summing, until the sum exceeds
    adaptive_fraction * sum_weight.  Returns (significant weight, number
    walked)."""
    sw = np.sort(np.asarray(weights, dtype=np.float64))
    frac, sig, n = 0.0, 0.0, 0
    for x in sw[::-1]:
        n += 1
        sig = float(x)
        frac += sig
        if frac > adaptive_fraction * sum_weight:
            break
    return sig, n


def best_pose(pl: ParticleList, weights: np.ndarray, nr_dir: int, nr_psi: int, nr_over_rot: int,
              nr_over_trans: int, angles: np.ndarray, over_trans_x: np.ndarray, over_trans_y: np.ndarray,
              old_offx: float, old_offy: float):
    """The metadata convertSquaredDifferencesToWeights writes for the largest
    weight (:1787-1804): class (1-based), rot, tilt, psi of the over-rotation
    (SamplingGrid::setOrientation, `angles` [ndir][npsi][nor][3]) and the
    offsets old_offset + exp_over_trans (over_trans_x/y [ntr][notr]).  The
    first largest weight in loop order wins."""
    q = int(np.argmax(weights))
    kd, ipsi = divmod(int(pl.kdp[q]), nr_psi)
    cls, idir = divmod(kd, nr_dir)
    h = int(pl.ihidden[q])
    itrans, rest = divmod(h, nr_over_rot * nr_over_trans)
    iover_rot, iover_trans = divmod(rest, nr_over_trans)
    rot, tilt, psi = (float(x) for x in angles[idir, ipsi, iover_rot])
    return {"class": cls + 1, "rot": rot, "tilt": tilt, "psi": psi,
            "xoff": old_offx + float(over_trans_x[itrans, iover_trans]),
            "yoff": old_offy + float(over_trans_y[itrans, iover_trans])}
