"""Host logic of the 3D proposal-restricted E-steps (rome_b200.proposal:
learned_estep3d, lowres_proposals3d, lowres_estep3d), with the network's
proposals and the library's E-step replaced by fakes: the particles whose
proposals hold at least min_mass are searched over them, the others
exhaustively, and the two calls' outputs come back in pool order with the
pool sums added; the low-resolution proposals are the top k of one
exhaustive call at the small coarse size on the auxiliary context.  CPU
only."""
import numpy as np

from rome_b200 import map3d, proposal
from rome_b200.map3d import merge_results3d, pool3d_from_dump, take_pool3d


class FakeNet:
    def __init__(self, props, mass):
        self.props, self.mass = props, mass

    def propose(self, pool, k):
        assert pool.nr_images == len(self.mass)
        return self.props, self.mass


def fake_estep(calls, tag):
    """An E-step that names each particle by its highres_Xi2 and records the call."""
    def run(ctx, p, marginals=False, proposals=None, **kw):
        calls.append((tag, p.highres_Xi2.copy(), None if proposals is None else proposals.copy()))
        n = p.nr_images
        return {"min_diff2": p.highres_Xi2 * 2.0, "cls": np.arange(n, dtype=np.int32) + (100 if tag == "r" else 200),
                "wsum_pdf_class": np.full(2, float(n)), "wsum_sigma2_offset": np.ones(1)}
    return run


def test_split_and_merge(golden, monkeypatch):
    g = golden["map3d_a"]
    p = pool3d_from_dump(g, 0)
    p.highres_Xi2 = np.arange(p.nr_images, dtype=np.float64) + 1.0  # particle i is named i + 1
    calls = []
    monkeypatch.setattr(map3d, "map3d_estep_pool", fake_estep(calls, "r"))
    monkeypatch.setattr(map3d, "map3d_estep_pools_adaptive", fake_estep(calls, "x"))
    props = np.arange(4 * 6, dtype=np.int32).reshape(4, 6)
    mass = np.array([0.99, 0.5, 0.999, 0.1], np.float32)
    out, pr, ms, low = proposal.learned_estep3d(None, FakeNet(props, mass), p, 3, min_mass=0.95)
    assert low.tolist() == [1, 3]
    (t0, ids0, pr0), (t1, ids1, pr1) = calls
    assert t0 == "r" and ids0.tolist() == [1.0, 3.0] and np.array_equal(pr0, props[[0, 2]])
    assert t1 == "x" and ids1.tolist() == [2.0, 4.0] and pr1 is None
    assert out["min_diff2"].tolist() == [2.0, 4.0, 6.0, 8.0]
    assert out["cls"].tolist() == [100, 200, 101, 201]
    assert out["wsum_pdf_class"].tolist() == [4.0, 4.0] and out["wsum_sigma2_offset"].tolist() == [2.0]


def test_all_confident_is_one_restricted_call(golden, monkeypatch):
    g = golden["map3d_a"]
    p = pool3d_from_dump(g, 0)
    calls = []
    monkeypatch.setattr(map3d, "map3d_estep_pool", fake_estep(calls, "r"))
    monkeypatch.setattr(map3d, "map3d_estep_pools_adaptive", fake_estep(calls, "x"))
    props = np.zeros((4, 2), np.int32)
    out, _, _, low = proposal.learned_estep3d(None, FakeNet(props, np.ones(4, np.float32)), p, 1, min_mass=0.5)
    assert low.size == 0 and [c[0] for c in calls] == ["r"]
    assert np.array_equal(calls[0][1], p.highres_Xi2)


def test_take_and_merge_round_trip(golden):
    g = golden["map3d_a"]
    p = pool3d_from_dump(g, 0)
    q = take_pool3d(p, [2, 0])
    assert q.nr_images == 2 and np.array_equal(q.Fimg_real, p.Fimg_real[[2, 0]])
    assert np.array_equal(q.group, np.asarray(p.group)[[2, 0]]) and q.angles is p.angles
    m = merge_results3d([(np.array([2, 0]), {"pmax": np.array([0.5, 0.25]), "wsum_sumw_group": np.ones(3)}),
                         (np.array([1]), {"pmax": np.array([0.75]), "wsum_sumw_group": np.ones(3)})], 3)
    assert m["pmax"].tolist() == [0.25, 0.75, 0.5] and m["wsum_sumw_group"].tolist() == [2.0, 2.0, 2.0]


def test_lowres_proposals_from_the_small_coarse_pass(golden, monkeypatch):
    """lowres_proposals3d: one exhaustive E-step call on the auxiliary
    context at the small coarse size (its resolution table, a significance
    fraction that keeps one coarse point), and the k most probable coarse
    orientations of its posterior, ascending, with the mass they hold."""
    g = golden["map3d_a"]
    p = pool3d_from_dump(g, 0)
    Jc = p.nr_classes * p.nr_dir * p.nr_psi
    rng = np.random.default_rng(1)
    post = rng.random((p.nr_images, Jc))
    post /= post.sum(1, keepdims=True)
    seen = []

    def fake(ctx, q, marginals=False, proposals=None, **kw):
        seen.append((ctx, q.coarse_size, q.adaptive_fraction, marginals, proposals, q.Mresol_coarse))
        return {"post_coarse": post}
    monkeypatch.setattr(map3d, "map3d_estep_pool", fake)
    props, mass = proposal.lowres_proposals3d("aux", p, 5, coarse_size=8)
    (ctx, cs, frac, marg, pr, mres), = seen
    assert ctx == "aux" and cs == 8 and frac < 1e-9 and marg and pr is None
    from rome_b200.workload import mresol
    assert np.array_equal(mres, mresol(8))
    want = np.sort(np.argsort(-post, axis=1)[:, :5], axis=1)
    assert np.array_equal(props, want) and props.dtype == np.int32
    np.testing.assert_allclose(mass, np.take_along_axis(post, want, 1).sum(1), rtol=1e-12)
    # more proposals than coarse orientations: all of them
    props, mass = proposal.lowres_proposals3d("aux", p, Jc + 7, coarse_size=8)
    assert np.array_equal(props, np.tile(np.arange(Jc, dtype=np.int32), (p.nr_images, 1)))
    np.testing.assert_allclose(mass, 1.0, rtol=1e-12)


def test_lowres_estep_splits_on_the_low_resolution_mass(golden, monkeypatch):
    g = golden["map3d_a"]
    p = pool3d_from_dump(g, 0)
    p.highres_Xi2 = np.arange(p.nr_images, dtype=np.float64) + 1.0
    props = np.tile(np.arange(3, dtype=np.int32), (4, 1))
    monkeypatch.setattr(proposal, "lowres_proposals3d",
                        lambda aux, pool, k, cs=12, **kw: (props, np.array([0.2, 0.999, 0.9995, 0.5])))
    calls = []
    monkeypatch.setattr(map3d, "map3d_estep_pool", fake_estep(calls, "r"))
    monkeypatch.setattr(map3d, "map3d_estep_pools_adaptive", fake_estep(calls, "x"))
    out, pr, ms, low = proposal.lowres_estep3d("ctx", "aux", p, 3, min_mass=0.99)
    assert low.tolist() == [0, 3]
    assert [c[0] for c in calls] == ["r", "x"]
    assert calls[0][1].tolist() == [2.0, 3.0] and calls[1][1].tolist() == [1.0, 4.0]
    assert out["cls"].tolist() == [200, 100, 101, 201]


def test_device_images_follow_the_split(golden, monkeypatch):
    """With the images on the device (here CPU tensors standing in), each
    call gets its own particles' rows of every image tensor."""
    import torch
    g = golden["map3d_a"]
    p = pool3d_from_dump(g, 0)
    p.highres_Xi2 = np.arange(p.nr_images, dtype=np.float64) + 1.0
    dev = {"Fimg_real": torch.arange(4, dtype=torch.float64)[:, None].repeat(1, 3),
           "Fctf": 10.0 + torch.arange(4, dtype=torch.float64)[:, None]}
    seen = []

    def fake(tag):
        def run(ctx, q, marginals=False, proposals=None, dev=None, **kw):
            seen.append((tag, q.highres_Xi2.tolist(), None if dev is None else dev["Fimg_real"][:, 0].tolist(),
                         None if dev is None else dev["Fctf"][:, 0].tolist()))
            return {"pmax": q.highres_Xi2.copy()}
        return run
    monkeypatch.setattr(map3d, "map3d_estep_pool", fake("r"))
    monkeypatch.setattr(map3d, "map3d_estep_pools_adaptive", fake("x"))
    props = np.zeros((4, 2), np.int32)
    out, low = proposal._restricted_or_exhaustive3d("ctx", p, props, np.array([1.0, 0.0, 0.0, 1.0]), 0.5, False,
                                                    dev=dev)
    assert low.tolist() == [1, 2]
    assert seen == [("r", [1.0, 4.0], [0.0, 3.0], [10.0, 13.0]), ("x", [2.0, 3.0], [1.0, 2.0], [11.0, 12.0])]
    assert out["pmax"].tolist() == [1.0, 2.0, 3.0, 4.0]
