"""3D learned proposals on the GPU.

* The restricted coarse pass with every coarse orientation proposed gives
  the exhaustive 3D E-step's results (reference fixture pool, all precisions).
* The native synthetic 3D workload (rome_b200.workload.build_map3d: HEALPix
  sampling restated from the reference, Fourier-slice particles) is
  consistent with the library's projector: the exhaustive E-step recovers
  the generating class and orientation.
* Training gain in 3D: the proposal network over (class x direction, psi mod
  180) trained on the coarse posterior marginals finds the exhaustive coarse
  mode in its top k far more often than untrained, and the proposal-
  restricted 3D E-step agrees with the exhaustive one on held-out particles.
"""
import numpy as np
import pytest

from rome_b200.map2d import GpuContext
from rome_b200.map3d import map3d_estep_pool, pool3d_from_dump
from rome_b200.proposal import ProposalNet, expand_proposals, posterior_targets
from rome_b200.sampling import euler_matrix
from rome_b200.workload import Map3dWorkload, build_map3d, subset3d
from tests.util import relerr

pytestmark = pytest.mark.gpu

POSE = ("cls", "rot", "tilt", "psi", "xoff", "yoff")


@pytest.mark.parametrize("prec", ["fp32", "bf16x3", "bf16"])
def test_restricted_coarse_pass_with_every_orientation_equals_exhaustive(golden, prec):
    g = golden["map3d_a"]
    p = pool3d_from_dump(g, 0)
    Jc = p.nr_classes * p.nr_dir * p.nr_psi
    allj = np.tile(np.arange(Jc, dtype=np.int32), (p.nr_images, 1))
    out = []
    for props in (None, allj):
        with GpuContext(0, prec) as ctx:
            ctx.set_projectors(g["projector_data"], p.ori_size, int(g["projector_r_max"][0]))
            out.append(map3d_estep_pool(ctx, p, marginals=True, proposals=props))
    a, b = out
    for k in POSE:
        assert np.array_equal(a[k], b[k]), k
    # the two contractions round differently: FP32 sums in another order; plain BF16 rounds the
    # product xw * conj(P) once instead of the shifted image and P separately
    tol = {"fp32": 1e-4, "bf16x3": 1e-3, "bf16": 1e-2}[prec]
    for k in ("min_diff2", "sum_weight", "significant_weight", "wsum_pdf_direction"):
        assert relerr(b[k], a[k]) <= tol, (k, relerr(b[k], a[k]))
    # the marginals collect the small weights too (up to exp(-diff2) of the BF16 rounding)
    assert relerr(b["post_coarse"], a["post_coarse"]) <= (5e-2 if prec == "bf16" else tol)
    if prec != "bf16":  # a broad coarse posterior (particle 3 of the fixture) has near-ties under BF16
        assert np.array_equal(b["post_coarse"].argmax(axis=1), a["post_coarse"].argmax(axis=1))
    m = a["post_coarse"].sum(axis=1)
    assert (m > 0.99).all() and (m <= 1 + 1e-9).all()


def _angle_between(a, b):
    """Rotation angle (degrees) between two sets of Euler angles."""
    out = []
    for x, y in zip(a, b):
        R = euler_matrix(*x) @ euler_matrix(*y).T
        out.append(np.degrees(np.arccos(np.clip((np.trace(R) - 1) / 2, -1, 1))))
    return np.array(out)


def test_synthetic_3d_workload_recovers_truth():
    w = Map3dWorkload(n_particles=120, ori_size=32, n_classes=2, healpix_order=1, snr=1.0, seed=4)
    p, proj, r_max, truth = build_map3d(w)
    with GpuContext(0, "bf16") as ctx:
        ctx.set_projectors(proj, p.ori_size, r_max)
        o = map3d_estep_pool(ctx, p)
    cls_ok = np.mean(o["cls"] - 1 == truth["cls"])
    err = _angle_between(np.stack([o["rot"], o["tilt"], o["psi"]], 1),
                         np.stack([truth["rot"], truth["tilt"], truth["psi"]], 1))
    print(f"class {cls_ok:.3f}, median angular error {np.median(err):.1f} deg")
    assert cls_ok >= 0.9
    assert np.median(err) <= 12.0  # fine sampling 15 deg at HEALPix order 2 (order 1 oversampled)


def test_3d_training_gain_and_restricted_coarse_pass():
    """3D is harder for the network than 2D: nearby directions have similar
    Fourier magnitudes.  Started from the matched filter of the direction
    projections (init_matched_filter) and trained on the coarse posteriors,
    its top 32 (class x direction, psi mod 180) outputs hold the exhaustive
    coarse mode for most held-out particles, far more often than untrained,
    and the restricted coarse pass (64 of 1,152 coarse orientations) gives
    the exhaustive pose for most of them."""
    from rome_b200.map3d import direction_templates
    w = Map3dWorkload(n_particles=4400, ori_size=32, n_classes=2, healpix_order=1, snr=0.3, seed=8)
    p, proj, r_max, _ = build_map3d(w)
    KD, npsi = p.nr_classes * p.nr_dir, p.nr_psi
    k = 32
    with GpuContext(0, "bf16") as ctx:
        ctx.set_projectors(proj, p.ori_size, r_max)
        train, test = subset3d(p, 0, 4000), subset3d(p, 4000, 4400)
        tr = map3d_estep_pool(ctx, train, marginals=True)
        ex = map3d_estep_pool(ctx, test, marginals=True)
        best = posterior_targets(ex["post_coarse"], KD, npsi).argmax(axis=1)
        with ProposalNet(ctx, KD, npsi // 2, 12, (16, 16), r_lo=1.5, r_hi=13.0, seed=5) as net:
            xtr, xte = net.features(train), net.features(test)
            idx0, _ = net.predict(xte, k)
            recall0 = np.mean([best[i] in idx0[i] for i in range(len(best))])
            net.init_matched_filter(direction_templates(net, proj, r_max, p), scale=10.0)
            losses = net.train(xtr, posterior_targets(tr["post_coarse"], KD, npsi), epochs=15, batch=128, lr=1e-3)
            idx1, _ = net.predict(xte, k)
            recall1 = np.mean([best[i] in idx1[i] for i in range(len(best))])
            props, mass = net.propose(test, k)
        assert np.array_equal(props, expand_proposals(idx1, npsi))
        r = map3d_estep_pool(ctx, test, proposals=props)
    agree = np.mean((r["cls"] == ex["cls"]) & (r["rot"] == ex["rot"]) & (r["tilt"] == ex["tilt"])
                    & (r["psi"] == ex["psi"]))
    print(f"3D: loss {losses[0]:.3f} -> {losses[-1]:.3f}; top-{k} recall {recall0:.3f} -> {recall1:.3f}; "
          f"restricted pose agreement {agree:.3f} searching {props.shape[1]} of {KD * npsi} coarse orientations")
    assert losses[-1] < losses[0]
    assert recall1 >= recall0 + 0.3
    assert recall1 >= 0.65
    assert agree >= 0.6
