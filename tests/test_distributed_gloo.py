"""Particle sharding and the per-iteration reduction on world size 2 (gloo,
CPU): the ranges reproduce the reference's divide_equally /
divide_equally_pool (src/mpi.cpp:34-61) -- disjoint, covering, sizes within
one -- and the all-reduce of the model sums gives every rank the total."""
import multiprocessing as mp
import os

import numpy as np
import pytest

from rome_b200.distributed import (MODEL_SUM_KEYS, allreduce_model_sums, divide_equally, divide_equally_pool,
                                   max_over_ranks)


def _ref_divide_equally(n, size, rank):
    # the reference's integer arithmetic, written out independently
    jobs = n // size
    rest = n % size
    if rank < rest:
        first = rank * (jobs + 1)
        last = first + jobs
    else:
        first = rank * jobs + rest
        last = first + jobs - 1
    return first, last


@pytest.mark.parametrize("n", [0, 1, 7, 50, 1000, 20001])
@pytest.mark.parametrize("size", [1, 2, 3, 8])
def test_divide_equally_covers_and_balances(n, size):
    ranges = [divide_equally(n, size, r) for r in range(size)]
    assert ranges == [_ref_divide_equally(n, size, r) for r in range(size)]
    got = [x for f, l in ranges for x in range(f, l + 1)]
    assert got == list(range(n))
    sizes = [l - f + 1 for f, l in ranges]
    assert max(sizes) - min(sizes) <= 1


@pytest.mark.parametrize("n,pool", [(20000, 2000), (1000, 50), (1001, 50), (7, 3)])
@pytest.mark.parametrize("size", [1, 2, 4])
def test_divide_equally_pool_whole_pools(n, pool, size):
    ranges = [divide_equally_pool(n, pool, size, r) for r in range(size)]
    got = [x for f, l in ranges for x in range(f, l + 1)]
    assert got == list(range(n))
    for f, l in ranges:
        if l >= f:
            assert f % pool == 0


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(rank)
        sums = {k: rng.normal(size=(3, 4) if k == "wsum_sigma2_noise" else (5,)) for k in MODEL_SUM_KEYS}
        sums["min_diff2"] = np.full(4, float(rank))  # per particle: not reduced
        sums["wsum_LL"] = float(rank) + 0.25             # a host-side scalar as a plain float
        out = allreduce_model_sums(sums)
        m = max_over_ranks(10.0 + rank)
        q.put((rank, {k: (v.tolist() if isinstance(v, np.ndarray) else v) for k, v in out.items()}, m))
    finally:
        dist.destroy_process_group()


def test_allreduce_model_sums_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 2000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict()
    for _ in range(2):
        rank, out, m = q.get(timeout=120)
        res[rank] = (out, m)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = {}
    for rank in range(2):
        rng = np.random.default_rng(rank)
        for k in MODEL_SUM_KEYS:
            v = rng.normal(size=(3, 4) if k == "wsum_sigma2_noise" else (5,))
            want[k] = want.get(k, 0) + v
    want["wsum_LL"] = 0.25 + 1.25
    for rank in range(2):
        out, m = res[rank]
        assert m == 11.0
        for k in MODEL_SUM_KEYS:
            np.testing.assert_allclose(np.array(out[k]), want[k], rtol=1e-15, atol=1e-15)
        assert isinstance(out["wsum_LL"], float)
        assert out["min_diff2"] == [float(rank)] * 4


class FakeBpContext:
    """A CPU stand-in for GpuContext's back-projector exchange interface
    (rome_gpu_backprojector_size / _device_copy): K classes of `vox` voxels,
    data [K][vox][2] then weight [K][vox] in the flat buffer."""

    torch_device = "cpu"

    def __init__(self, K, vox, seed):
        rng = np.random.default_rng(seed)
        self.data = rng.normal(size=(K, vox, 2))
        self.weight = rng.uniform(size=(K, vox))

    def backprojector_doubles(self):
        return self.data.size + self.weight.size

    def copy_backprojectors_to(self, buf):
        import torch
        buf.copy_(torch.from_numpy(np.concatenate([self.data.ravel(), self.weight.ravel()])))

    def copy_backprojectors_from(self, buf):
        a = buf.numpy()
        self.data = a[:self.data.size].reshape(self.data.shape).copy()
        self.weight = a[self.data.size:].reshape(self.weight.shape).copy()


def _bp_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    from rome_b200.distributed import (allreduce_backprojectors, broadcast_class_maps, owner_of_class,
                                       reduce_backprojectors_by_class)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        K, vox = 3, 50
        a = FakeBpContext(K, vox, 100 + rank)
        nbytes = allreduce_backprojectors(a)
        b = FakeBpContext(K, vox, 200 + rank)
        owned = reduce_backprojectors_by_class(b, K)
        maps = [torch.full((4,), float(10 * k + rank)) for k in range(K)]
        broadcast_class_maps(maps)
        q.put((rank, nbytes, a.data.tolist(), a.weight.tolist(), b.data.tolist(), b.weight.tolist(), owned,
               [m.tolist() for m in maps], [owner_of_class(k, world) for k in range(K)]))
    finally:
        dist.destroy_process_group()


def test_backprojector_exchange_world2():
    """All-reduce of every class's back-projector, and the class-partitioned
    reduce (class k onto rank k % world) with the broadcast of the owners'
    maps, on world size 2 through the device-copy interface."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 31500 + os.getpid() % 2000
    procs = [ctx.Process(target=_bp_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r = q.get(timeout=120)
        res[r[0]] = r[1:]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    K, vox = 3, 50
    src_a = [FakeBpContext(K, vox, 100 + r) for r in range(2)]
    src_b = [FakeBpContext(K, vox, 200 + r) for r in range(2)]
    for rank in range(2):
        nbytes, ad, aw, bd, bw, owned, maps, owners = res[rank]
        assert nbytes == 3 * K * vox * 8
        np.testing.assert_allclose(np.array(ad), src_a[0].data + src_a[1].data, rtol=1e-15)
        np.testing.assert_allclose(np.array(aw), src_a[0].weight + src_a[1].weight, rtol=1e-15)
        assert owners == [0, 1, 0] and owned == [k for k in range(K) if k % 2 == rank]
        for k in range(K):
            if k % 2 == rank:  # the owner holds the sum
                np.testing.assert_allclose(np.array(bd)[k], src_b[0].data[k] + src_b[1].data[k], rtol=1e-15)
                np.testing.assert_allclose(np.array(bw)[k], src_b[0].weight[k] + src_b[1].weight[k], rtol=1e-15)
            assert maps[k] == [float(10 * k + k % 2)] * 4  # every rank has the owner's map
