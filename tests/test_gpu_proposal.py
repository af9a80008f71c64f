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
        assert np.array_equal(net.features(ctx.stage_pool(p)), x)  # device inputs: the same kernel
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


@pytest.mark.parametrize("offset_range", [2, 4])  # 13 and 49 translations: 32- and 64-wide tiles
def test_restricted_tensor_core_modes_match_fp32(offset_range):
    """The tensor-core restricted contraction (w = xw * conj(P) formed in
    shared memory, contracted with the translation-phase operand) against
    the FP32 CUDA-core restricted path on the same proposal lists: split
    BF16 to 2e-5 in min_diff2 and identical poses; plain BF16 to 1e-3 and
    >= 97% identical poses (BF16 rounding of w and of the phases)."""
    w = Map2dWorkload(n_particles=300, ori_size=64, n_classes=4, n_blobs=16, psi_step=10, offset_range=offset_range,
                      offset_step=1, max_shift=3, pixel=2.0, snr=0.05, seed=23)
    p, proj, r_max, _ = build_map2d(w)
    J = p.nr_classes * p.nr_psi
    rng = np.random.default_rng(5)
    nprop = 40  # not a divisor of the 128-row tile: rows of one particle straddle tiles
    props = np.sort(np.stack([rng.choice(J, nprop, replace=False) for _ in range(p.nr_images)]), axis=1)
    props = props.astype(np.int32)
    out = {}
    for prec in ("fp32", "bf16x3", "bf16"):
        with GpuContext(0, prec) as c:
            c.set_projectors(proj, p.ori_size, r_max)
            out[prec] = c.map2d_estep_pool(p, proposals=props, marginals=True)
    ref = out["fp32"]
    for prec, tol, agree_min in (("bf16x3", 2e-5, 1.0), ("bf16", 1e-3, 0.97)):
        o = out[prec]
        assert relerr(o["min_diff2"], ref["min_diff2"]) <= tol, (prec, relerr(o["min_diff2"], ref["min_diff2"]))
        same = (o["cls"] == ref["cls"]) & (o["psi"] == ref["psi"]) & (o["xoff"] == ref["xoff"]) & (
            o["yoff"] == ref["yoff"])
        assert same.mean() >= agree_min, (prec, same.mean())
        # every reported orientation is one of the particle's proposals
        # reported psi: the table angle folded into (-180, 180]
        tab = np.asarray(p.over_psi[-1])[:, 0]
        ipsi = {(float(v) - 360.0 if v > 180 else float(v)): k for k, v in enumerate(tab)}
        jbest = (o["cls"] - 1) * p.nr_psi + np.array([ipsi[float(v)] for v in o["psi"]])
        assert all(jbest[i] in props[i] for i in range(p.nr_images))


def test_learned_pools_with_fallback_match_per_pool_calls(ctx):
    """learned_estep_pools (fallback particles of all pools in one exhaustive
    call) gives every particle the outputs of learned_estep on its own pool,
    and the same pool sums in total; with min_mass = 1 every particle is
    searched exhaustively and the outputs are the exhaustive E-step's."""
    from rome_b200.map2d import GpuContext as G
    from rome_b200.proposal import learned_estep, learned_estep_pools
    w = Map2dWorkload(n_particles=600, ori_size=64, n_classes=4, n_blobs=16, psi_step=10, offset_range=2,
                      offset_step=1, max_shift=2, pixel=2.0, snr=0.1, seed=31)
    p, proj, r_max, _ = build_map2d(w)
    pools = [subset(p, lo, lo + 200) for lo in (0, 200, 400)]
    with G(0, "bf16") as c:
        c.set_projectors(proj, p.ori_size, r_max)
        with ProposalNet(c, p.nr_classes, p.nr_psi // 2, 12, (8, 8), 2.0, 12.0, seed=1) as net:
            staged = [c.stage_pool(q) for q in pools]
            masses = np.concatenate([net.propose(q, 6)[1] for q in staged])
            mixed = float(np.median(masses))  # about half of the particles fall back
            for mm in (mixed, 1.0):
                got = learned_estep_pools(c, net, staged, 6, mm)
                want = [learned_estep(c, net, q, 6, mm) for q in staged]
                nlow = sum(len(g[3]) for g in got)
                assert nlow == sum(len(x[3]) for x in want)
                assert 0 < nlow and (mm == 1.0 or nlow < p.nr_images)
                for g, x in zip(got, want):
                    for key in ("cls", "psi", "xoff", "yoff"):
                        assert np.array_equal(g[0][key], x[0][key]), key
                    assert relerr(g[0]["sum_weight"], x[0]["sum_weight"]) <= 1e-9
                tot_g = sum(g[0]["wsum_pdf_class"] for g in got)
                tot_w = sum(x[0]["wsum_pdf_class"] for x in want)
                assert relerr(tot_g, tot_w) <= 1e-9
                if mm == 1.0:
                    assert nlow == p.nr_images
                    for g, q in zip(got, staged):
                        e = c.map2d_estep_pool(q)
                        assert np.array_equal(g[0]["cls"], e["cls"]) and np.array_equal(g[0]["psi"], e["psi"])
            # the prefetching iterator yields the same pools
            hs = [q for q in c.staged(pools)]
            assert all(np.array_equal(a.dev["Fctf"].cpu().numpy(), b.dev["Fctf"].cpu().numpy())
                       for a, b in zip(hs, staged))


def test_learned_pools_with_two_worker_threads_match_one():
    """Pools dealt to two host threads (two contexts, two copies of the
    network) give every particle the same outputs as one thread, and the
    back-projectors merged into the first context equal one context's."""
    from rome_b200.map2d import GpuContext as G
    from rome_b200.proposal import learned_estep_pools
    w = Map2dWorkload(n_particles=600, ori_size=64, n_classes=4, n_blobs=16, psi_step=10, offset_range=2,
                      offset_step=1, max_shift=2, pixel=2.0, snr=0.1, seed=37)
    p, proj, r_max, _ = build_map2d(w)
    pools = [subset(p, lo, lo + 100) for lo in range(0, 600, 100)]
    with G(0, "bf16") as c0, G(0, "bf16") as c1, G(0, "bf16") as ref:
        nets = []
        for c in (c0, c1, ref):
            c.set_projectors(proj, p.ori_size, r_max)
            nets.append(ProposalNet(c, p.nr_classes, p.nr_psi // 2, 12, (8, 8), 2.0, 12.0, seed=2))
        for n in nets[1:]:
            n.set_params(nets[0].get_params())
        mm = float(np.median(nets[2].propose(pools[0], 6)[1]))  # some particles fall back
        two = learned_estep_pools(c0, nets[0], [c0.stage_pool(q) for q in pools], 6, mm, workers=[(c1, nets[1])])
        one = learned_estep_pools(ref, nets[2], [ref.stage_pool(q) for q in pools], 6, mm)
        for a, b in zip(two, one):
            assert np.array_equal(a[1], b[1]) and np.array_equal(a[3], b[3])
            for k in ("cls", "psi", "xoff", "yoff"):
                assert np.array_equal(a[0][k], b[0][k]), k
            assert relerr(a[0]["sum_weight"], b[0]["sum_weight"]) == 0.0
        assert relerr(sum(a[0]["wsum_pdf_class"] for a in two), sum(b[0]["wsum_pdf_class"] for b in one)) <= 1e-12
        for k in range(p.nr_classes):
            d2, w2 = c0.get_backprojector(k)
            d1, w1 = ref.get_backprojector(k)
            assert relerr(d2, d1) <= 1e-12 and relerr(w2, w1) <= 1e-12
            assert not c1.get_backprojector(k)[1].any()  # cleared after the merge
        for n in nets:
            n.close()


def test_learned_bf16_with_fallback_agrees_with_plain_fp32():
    """The metric's comparison at test size: learned proposals (top 16 of the
    network's 108 (class, psi mod 180) outputs, i.e. 32 of 216 orientations)
    + the restricted E-step on the tensor cores, with the exhaustive E-step as
    the fallback for particles whose proposals carry less than 0.999 of the
    network's probability, on held-out particles.  Gates on identical best
    (class, psi, offset):
    - learned + split BF16 (as accurate as FP32) against the plain FP32
      exhaustive E-step: >= 99% (what the proposals lose);
    - learned + BF16 against plain FP32 no worse than the exhaustive BF16
      E-step itself (at 64^2 and SNR 0.1 BF16 rounding alone moves ~2% of
      the poses, where the FP32 posterior's top hypotheses are nearly tied;
      the restricted and the dense BF16 contractions round differently, so
      they also differ from each other at those ties);
    and the network, not the fallback, decides most particles.  Then the
    reconstructions (gridding-corrected, no MAP term) of every class from the
    learned split-BF16 pass's back-projectors and from the plain FP32 pass's
    are compared shell by shell: measured min FSC 0.9949 over the 6 classes
    and 31 shells of these 400 held-out particles (about 67 per class, so
    one particle whose pose or posterior tail differs moves a class by ~1.5 %);
    gated at 0.99."""
    from rome_b200.proposal import learned_estep_pools
    from tests.test_gpu_reconstruct import fsc
    w = Map2dWorkload(n_particles=4400, ori_size=64, n_classes=6, n_blobs=20, psi_step=10, offset_range=3,
                      offset_step=1, max_shift=2, pixel=2.0, snr=0.1, seed=29)
    p, proj, r_max, _ = build_map2d(w)
    K, npsi = p.nr_classes, p.nr_psi
    train, test = subset(p, 0, 4000), subset(p, 4000, 4400)

    def volumes(c, o):
        vols = []
        for k in range(K):
            if o["wsum_pdf_class"][k] > 0:
                vols.append(c.reconstruct(k, p.ori_size, 2, np.ones(p.ori_size // 2 + 1), 1.0,
                                          float(o["wsum_pdf_class"][k]), 10, False, 0)["vol"])
            else:
                vols.append(None)
        return vols

    with GpuContext(0, "fp32") as c32:
        c32.set_projectors(proj, p.ori_size, r_max)
        ref = c32.map2d_estep_pool(test)
        ref_vols = volumes(c32, ref)
    with GpuContext(0, "bf16") as cb, GpuContext(0, "bf16x3") as cx:
        cb.set_projectors(proj, p.ori_size, r_max)
        cx.set_projectors(proj, p.ori_size, r_max)
        tr = cb.map2d_estep_pool(train, marginals=True)
        with ProposalNet(cb, K, npsi // 2, 16, r_lo=2.0, r_hi=24.0, seed=7) as net:
            net.train(net.features(train), posterior_targets(tr["post_class_psi"], K, npsi), epochs=15, batch=128,
                      lr=3e-3)
            lb, props, mass, low = learned_estep_pools(cb, net, [test], 16, min_mass=0.999)[0]
            lx = learned_estep_pools(cx, net, [test], 16, min_mass=0.999)[0][0]
        lx_vols = volumes(cx, lx)
        ex = cb.map2d_estep_pool(test)
    fmin = min(float(fsc(a, b).min()) for a, b in zip(lx_vols, ref_vols) if a is not None and b is not None)
    print(f"learned split BF16 vs plain FP32 reconstructions: min FSC over classes and shells {fmin:.6f}")
    assert fmin >= 0.99

    def agree(o, r):
        return float(np.mean((o["cls"] == r["cls"]) & (o["psi"] == r["psi"]) & (o["xoff"] == r["xoff"])
                             & (o["yoff"] == r["yoff"])))

    print(f"{props.shape[1]} of {K * npsi} orientations searched, fallback {len(low) / test.nr_images:.3f}; pose "
          f"agreement: learned BF16 vs exhaustive BF16 {agree(lb, ex):.4f}, learned split BF16 vs plain FP32 "
          f"{agree(lx, ref):.4f}, learned BF16 vs plain FP32 {agree(lb, ref):.4f}, exhaustive BF16 vs plain FP32 "
          f"{agree(ex, ref):.4f}")
    assert agree(lx, ref) >= 0.99
    assert agree(lb, ref) >= agree(ex, ref) - 0.005
    assert len(low) <= 0.5 * test.nr_images
