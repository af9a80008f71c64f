"""The device-resident back-projector exchange on one GPU: the device copy
round-trips the library's back-projectors exactly (checked against the host
download), and the NCCL all-reduce of allreduce_backprojectors runs on the
device buffer (a one-rank NCCL group, so the sum is the rank's own)."""
import os

import numpy as np
import pytest

from rome_b200.map2d import GpuContext
from rome_b200.workload import Map2dWorkload, build_map2d

pytestmark = pytest.mark.gpu


def test_device_copy_and_nccl_allreduce():
    import torch
    import torch.distributed as dist

    from rome_b200.distributed import allreduce_backprojectors
    w = Map2dWorkload(n_particles=32, ori_size=32, n_classes=3, n_blobs=8, blob_sigma=(1.5, 3.0), psi_step=15,
                      offset_range=3, offset_step=1, max_shift=2, pixel=4.0, snr=0.1, seed=21)
    p, proj, r_max, _ = build_map2d(w)
    with GpuContext(0, "fp32") as ctx:
        ctx.set_projectors(proj, p.ori_size, r_max)
        ctx.map2d_estep_pool(p)
        host = [ctx.get_backprojector(k) for k in range(p.nr_classes)]
        n = ctx.backprojector_doubles()
        vox = host[0][1].size
        assert n == 3 * vox * p.nr_classes
        buf = torch.empty(n, dtype=torch.float64, device="cuda:0")
        ctx.copy_backprojectors_to(buf)
        a = buf.cpu().numpy()
        for k in range(p.nr_classes):
            assert np.array_equal(a[2 * vox * k:2 * vox * (k + 1)], host[k][0].ravel())
            assert np.array_equal(a[2 * vox * p.nr_classes + vox * k:2 * vox * p.nr_classes + vox * (k + 1)],
                                  host[k][1].ravel())
        ctx.copy_backprojectors_from(buf * 2)
        for k in range(p.nr_classes):
            d, wt = ctx.get_backprojector(k)
            assert np.array_equal(d, 2 * host[k][0]) and np.array_equal(wt, 2 * host[k][1])
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", str(33500 + os.getpid() % 2000))
        dist.init_process_group("nccl", rank=0, world_size=1)
        try:
            nbytes = allreduce_backprojectors(ctx)
            torch.cuda.synchronize()
        finally:
            dist.destroy_process_group()
        assert nbytes == 8 * n
        for k in range(p.nr_classes):
            d, wt = ctx.get_backprojector(k)
            assert np.array_equal(d, 2 * host[k][0]) and np.array_equal(wt, 2 * host[k][1])
