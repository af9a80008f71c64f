"""Host logic of the 2D learned E-step over several pools
(rome_b200.proposal.learned_estep / learned_estep_pools), with the network
and the library's E-step replaced by fakes: each pool's confident particles
are searched over their own proposals; the particles below min_mass from
every pool go to ONE exhaustive call, in pool order, whose per-particle
outputs return to their pools and whose pool sums are added to the first
pool's result; with worker lanes the pools are dealt round-robin and the
workers' back-projectors are added into the first context.  CPU only."""
import numpy as np

from rome_b200 import proposal
from rome_b200.map2d import pool_from_dump, take_pool


class FakeCtx:
    """Records every E-step call; a particle is named by its highres_Xi2."""

    def __init__(self, name, log):
        self.name, self.log, self.added = name, log, []

    def map2d_estep_pool(self, p, marginals=False, proposals=None):
        self.log.append((self.name, p.highres_Xi2.tolist(), None if proposals is None else proposals.tolist()))
        n = p.nr_images
        restricted = proposals is not None
        return {"min_diff2": p.highres_Xi2 * 10.0, "cls": np.full(n, 1 if restricted else 2, np.int32),
                "wsum_pdf_class": np.full(3, float(n)), "wsum_sigma2_offset": np.full(1, 100.0 if not restricted
                                                                                       else 1.0)}

    def add_backprojectors(self, src, clear=True):
        self.added.append((src.name, clear))


class FakeNet:
    """Proposals [P][2]: (name, name); mass from a table keyed by name."""

    def __init__(self, mass_of):
        self.mass_of = mass_of

    def propose(self, pool, k):
        names = pool.highres_Xi2
        props = np.stack([names, names], 1).astype(np.int32)
        return props, np.array([self.mass_of[int(v)] for v in names], np.float32)


def _pools(golden, sizes):
    g = golden["map2d_a"]
    base = pool_from_dump(g, 0)
    pools, name = [], 1
    for n in sizes:
        q = take_pool(base, np.arange(n) % base.nr_images)
        q.highres_Xi2 = np.arange(name, name + n, dtype=np.float64)
        name += n
        pools.append(q)
    return pools


def test_fallback_of_all_pools_in_one_call(golden):
    pools = _pools(golden, [3, 4, 2, 2])       # particles named 1..11
    low = {2, 5, 6, 9, 10, 11}                 # the last pool falls back entirely
    net = FakeNet({i: (0.1 if i in low else 0.999) for i in range(1, 12)})
    log = []
    ctx = FakeCtx("main", log)
    res = proposal.learned_estep_pools(ctx, net, pools, k=1, min_mass=0.9)
    restricted = [c for c in log if c[2] is not None]
    exhaustive = [c for c in log if c[2] is None]
    assert [c[1] for c in restricted] == [[1.0, 3.0], [4.0, 7.0], [8.0]]
    assert [c[2] for c in restricted] == [[[1, 1], [3, 3]], [[4, 4], [7, 7]], [[8, 8]]]
    assert len(exhaustive) == 1 and exhaustive[0][1] == [2.0, 5.0, 6.0, 9.0, 10.0, 11.0]
    for (out, props, mass, lowi), q in zip(res, pools):
        names = q.highres_Xi2
        assert out["min_diff2"].tolist() == (names * 10.0).tolist()
        assert out["cls"].tolist() == [2 if int(v) in low else 1 for v in names]
        assert lowi.tolist() == [i for i, v in enumerate(names) if int(v) in low]
    # the fallback call's sums are added to the first pool's result only; a pool without a call of
    # its own gets zero sums
    r0, r1, r2, r3 = (r[0] for r in res)
    assert r0["wsum_sigma2_offset"].tolist() == [101.0] and r0["wsum_pdf_class"].tolist() == [8.0] * 3
    assert r1["wsum_sigma2_offset"].tolist() == [1.0] and r1["wsum_pdf_class"].tolist() == [2.0] * 3
    assert r2["wsum_sigma2_offset"].tolist() == [1.0] and r2["wsum_pdf_class"].tolist() == [1.0] * 3
    assert r3["wsum_sigma2_offset"].tolist() == [0.0] and r3["wsum_pdf_class"].tolist() == [0.0] * 3


def test_worker_lanes_round_robin_and_backprojectors(golden):
    pools = _pools(golden, [2, 2, 2, 2])
    net = FakeNet({i: 0.999 for i in range(1, 9)})
    log = []
    ctx, w1 = FakeCtx("main", log), FakeCtx("w1", log)
    res = proposal.learned_estep_pools(ctx, net, pools, k=1, min_mass=0.9, workers=[(w1, net)])
    by_pool = {tuple(c[1]): c[0] for c in log}
    assert [by_pool[tuple(q.highres_Xi2.tolist())] for q in pools] == ["main", "w1", "main", "w1"]
    assert ctx.added == [("w1", True)] and w1.added == []
    assert all(r[3].size == 0 for r in res)
    assert [r[0]["min_diff2"].tolist() for r in res] == [(q.highres_Xi2 * 10).tolist() for q in pools]


def test_single_pool_learned_estep(golden):
    (q,) = _pools(golden, [5])
    net = FakeNet({1: 0.5, 2: 0.99, 3: 0.2, 4: 0.99, 5: 0.99})
    log = []
    out, props, mass, low = proposal.learned_estep(FakeCtx("main", log), net, q, k=1, min_mass=0.9)
    assert low.tolist() == [0, 2]
    assert [(c[1], c[2] is None) for c in log] == [([2.0, 4.0, 5.0], False), ([1.0, 3.0], True)]
    assert out["cls"].tolist() == [2, 1, 2, 1, 1]
    assert out["wsum_sigma2_offset"].tolist() == [101.0]
