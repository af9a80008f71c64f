"""Learned pose proposals on the GPU.

* The hand-written CUDA forward/backward of the proposal network matches the
  CPU oracle (oracle/proposal_oracle.py, FP64, itself checked against finite
  differences): loss and logits to 1e-4 relative, every gradient block to
  2e-3 of its largest entry (FP32 accumulation over the batch).
* The network input computed on the GPU matches the oracle's definition.
* The restricted E-step with every orientation proposed reproduces the
  exhaustive E-step (same poses, FP64 sums to 1e-4: the two FP32
  contractions sum in different orders).
* Training gain: after training on the exhaustive E-step's own posteriors,
  the network's top-k proposals contain the exhaustive posterior mode far
  more often than the untrained network's, and the proposal-restricted
  E-step agrees with the exhaustive one on held-out particles while
  evaluating a fraction of the hypotheses.
"""
import numpy as np
import pytest

from oracle import proposal_oracle as po
from rome_b200.map2d import GpuContext
from rome_b200.proposal import ProposalNet, dict_to_flat, expand_proposals, flat_to_dict, posterior_targets
from rome_b200.workload import Map2dWorkload, build_map2d, subset
from tests.util import relerr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = GpuContext(0, "fp32")
    yield c
    c.close()


def test_gradients_match_cpu_oracle(ctx):
    n_r, n_theta, ch, K, n = 12, 18, (8, 12), 5, 10
    rng = np.random.default_rng(3)
    params = {name: rng.normal(0, 0.1, shape) for name, shape in po.param_shapes(n_r, n_theta, ch, K)}
    x = rng.normal(size=(n, 2, n_r, n_theta)).astype(np.float32)
    t = rng.dirichlet(np.ones(K * n_theta) * 0.3, size=n).astype(np.float32)
    with ProposalNet(ctx, K, n_theta, n_r, ch) as net:
        net.set_params(dict_to_flat(params, n_r, n_theta, ch, K))
        loss, grad, logits = net.loss_grad(x, t)
    p32 = {k: v.astype(np.float32).astype(np.float64) for k, v in params.items()}
    rloss, rg, rz = po.loss_and_grads(p32, x.astype(np.float64), t.astype(np.float64))
    assert abs(loss - rloss) <= 1e-4 * abs(rloss)
    assert relerr(logits, rz) <= 1e-4
    g = flat_to_dict(grad, n_r, n_theta, ch, K)
    for k in rg:
        assert relerr(g[k], rg[k]) <= 2e-3, (k, relerr(g[k], rg[k]))


def test_features_match_oracle(ctx):
    w = Map2dWorkload(n_particles=8, ori_size=64, n_classes=3, n_blobs=12, psi_step=20, offset_range=2,
                      offset_step=1, max_shift=2, pixel=2.0, snr=0.1, seed=5)
    p, _, _, _ = build_map2d(w)
    with ProposalNet(ctx, 3, 9, 16, r_lo=2.0, r_hi=24.0) as net:
        x = net.features(p)
    r = po.features(p.Fimg_real, p.Fimg_imag, p.Fctf, p.current_size, 16, 9, 2.0, 24.0)
    assert np.max(np.abs(x - r)) <= 1e-4


def test_restricted_with_every_orientation_equals_exhaustive(ctx):
    w = Map2dWorkload(n_particles=16, ori_size=32, n_classes=3, n_blobs=8, blob_sigma=(1.5, 3.0), psi_step=15,
                      offset_range=3, offset_step=1, max_shift=2, pixel=4.0, snr=0.1, seed=11)
    p, proj, r_max, _ = build_map2d(w)
    J = p.nr_classes * p.nr_psi
    ctx.set_projectors(proj, p.ori_size, r_max)
    a = ctx.map2d_estep_pool(p, marginals=True)
    bp_a = np.stack([ctx.get_backprojector(k)[1] for k in range(p.nr_classes)])
    ctx.set_projectors(proj, p.ori_size, r_max)
    allj = np.tile(np.arange(J, dtype=np.int32), (p.nr_images, 1))
    b = ctx.map2d_estep_pool(p, marginals=True, proposals=allj)
    bp_b = np.stack([ctx.get_backprojector(k)[1] for k in range(p.nr_classes)])
    for k in ("cls", "psi", "xoff", "yoff"):
        assert np.array_equal(a[k], b[k]), k
    # both FP32 contractions, summed in a different order: diff2 agree to ~1e-7
    # relative, the FP64 sums (through exp(-diff2)) to ~1e-5
    for k in ("min_diff2", "sum_weight", "significant_weight", "wsum_sigma2_noise", "wsum_pdf_class",
              "post_class_psi"):
        assert relerr(b[k], a[k]) <= 1e-4, k
    assert relerr(bp_b, bp_a) <= 1e-4


def test_training_gain_and_restricted_search(ctx):
    w = Map2dWorkload(n_particles=3400, ori_size=64, n_classes=6, n_blobs=20, psi_step=10, offset_range=3,
                      offset_step=1, max_shift=2, pixel=2.0, snr=0.1, seed=17)
    p, proj, r_max, _ = build_map2d(w)
    K, npsi = p.nr_classes, p.nr_psi
    ctx.set_projectors(proj, p.ori_size, r_max)
    train, test = subset(p, 0, 3000), subset(p, 3000, 3400)
    tr = ctx.map2d_estep_pool(train, marginals=True)
    ex = ctx.map2d_estep_pool(test, marginals=True)
    best = posterior_targets(ex["post_class_psi"], K, npsi).argmax(axis=1)  # posterior mode of (class, psi mod 180)
    k = 8
    with ProposalNet(ctx, K, npsi // 2, 16, r_lo=2.0, r_hi=24.0, seed=7) as net:
        xtr, xte = net.features(train), net.features(test)
        idx0, _ = net.predict(xte, k)
        recall0 = np.mean([best[i] in idx0[i] for i in range(len(best))])
        losses = net.train(xtr, posterior_targets(tr["post_class_psi"], K, npsi), epochs=15, batch=128, lr=3e-3)
        idx1, prob1 = net.predict(xte, k)
        recall1 = np.mean([best[i] in idx1[i] for i in range(len(best))])
        props = expand_proposals(idx1, npsi)
        dprops, mass = net.propose(test, k)
    assert np.array_equal(dprops, props)  # the device-side expansion matches
    print(f"loss {losses[0]:.3f} -> {losses[-1]:.3f}; top-{k} recall untrained {recall0:.3f}, trained {recall1:.3f}")
    assert losses[-1] < losses[0]
    assert recall1 >= recall0 + 0.3
    assert recall1 >= 0.85
    r = ctx.map2d_estep_pool(test, proposals=props)
    agree = np.mean((r["cls"] == ex["cls"]) & (r["psi"] == ex["psi"]) & (r["xoff"] == ex["xoff"])
                    & (r["yoff"] == ex["yoff"]))
    frac = props.shape[1] / (K * npsi)
    print(f"restricted search over {frac:.3f} of the orientations: pose agreement {agree:.4f}")
    assert agree >= 0.85
