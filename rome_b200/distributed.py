"""Multi-GPU plumbing for the MAP E-step: one process per GPU, particles
sharded across ranks with no collective on the data path, and the one real
exchange step of an EM iteration -- the sum of every rank's weighted sums and
back-projected class volumes -- as NCCL (or gloo) all-reduces.

Reference counterparts:
* particle ranges: ``divide_equally`` / ``divide_equally_pool``
  (src/mpi.cpp:34-61), used by ``setImagesDistribution``
  (src/map_optimizer_base.h:373-409);
* per-iteration reduction of the model sums: ``MLModel::reduceData``
  (src/ml_model.cpp:587-637) and of the back-projectors
  ``MAPModel::reduceData`` (src/map_model.cpp:604-620, all-reduce; :621-666,
  each class reduced onto the node that reconstructs it, then the new
  references broadcast).

The back-projectors never leave the device: the context copies them device
to device into one flat FP64 buffer (``rome_gpu_backprojector_device_copy``),
the collective runs on that buffer, and the result is copied back.
"""
from __future__ import annotations

import math
from typing import Dict, Tuple

import numpy as np

__all__ = ["divide_equally", "divide_equally_pool", "allreduce_model_sums", "allreduce_backprojectors",
           "reduce_backprojectors_by_class", "broadcast_class_maps", "owner_of_class", "max_over_ranks"]

# the model sums added over ranks (MLModel::reduceData, src/ml_model.cpp:587-637): the pool sums of the
# E-step calls (rome_b200.map2d.alloc_outputs, rome_b200.map3d.map3d_estep_pool), then those the host-side
# storeWeightedSums adds (the scale-correction group spectra, wsum_avg_norm_correction, wsum_LL,
# wsum_ave_Pmax; scalars may be plain floats)
MODEL_SUM_KEYS = ("wsum_sigma2_noise", "wsum_pdf_class", "wsum_pdf_direction", "wsum_prior_offsetx_class",
                  "wsum_prior_offsety_class", "wsum_sigma2_offset", "wsum_sumw_group",
                  "wsum_signal_product_spectra", "wsum_reference_power_spectra", "wsum_avg_norm_correction",
                  "wsum_LL", "wsum_ave_Pmax")


def divide_equally(n: int, size: int, rank: int) -> Tuple[int, int]:
    """Inclusive range [first, last] of rank `rank` when n jobs are split over
    `size` ranks: the first n % size ranks take one job more
    (src/mpi.cpp:34-49)."""
    per, rest = divmod(n, size)
    if rank < rest:
        first = rank * (per + 1)
        return first, first + per
    first = rank * per + rest
    return first, first + per - 1


def divide_equally_pool(n: int, nr_pool: int, size: int, rank: int) -> Tuple[int, int]:
    """The same over whole pools of nr_pool particles: inclusive particle
    range [first, last] of `rank` (src/mpi.cpp:52-61)."""
    blocks = math.ceil(n / nr_pool)
    b0, b1 = divide_equally(blocks, size, rank)
    return b0 * nr_pool, min((b1 + 1) * nr_pool - 1, n - 1)


def _allreduce_np(arrays: Dict[str, np.ndarray], device) -> Dict[str, np.ndarray]:
    """Sum FP64 host arrays over all ranks in one flattened all-reduce."""
    import torch
    import torch.distributed as dist
    keys = sorted(arrays)
    flat = np.concatenate([np.ascontiguousarray(arrays[k], np.float64).ravel() for k in keys]) if keys else np.zeros(0)
    t = torch.from_numpy(flat).to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    out, off = {}, 0
    flat = t.cpu().numpy()
    for k in keys:
        a = arrays[k]
        n = int(np.size(a))
        out[k] = float(flat[off]) if np.ndim(a) == 0 else flat[off:off + n].reshape(np.shape(a)).copy()
        off += n
    return out


def allreduce_model_sums(sums: Dict[str, np.ndarray], device="cpu") -> Dict[str, np.ndarray]:
    """The iteration's weighted sums (wsum_*) of this rank, summed over all
    ranks (every rank gets the total).  Keys other than MODEL_SUM_KEYS pass
    through unchanged: per-particle outputs stay with their rank."""
    picked = {k: v for k, v in sums.items() if k in MODEL_SUM_KEYS}
    out = dict(sums)
    out.update(_allreduce_np(picked, device))
    return out


def _bp_buffer(ctx):
    """One flat FP64 tensor holding every class's back-projector, filled
    device to device from the context (data [K][vox][2], then weight [K][vox])."""
    import torch
    buf = torch.empty(ctx.backprojector_doubles(), dtype=torch.float64, device=ctx.torch_device)
    ctx.copy_backprojectors_to(buf)
    return buf


def allreduce_backprojectors(ctx, group=None) -> int:
    """Every class's back-projector (data and weight, FP64) summed over all
    ranks, in place in each rank's context (MAPModel::reduceData with the
    all-reduce, src/map_model.cpp:604-620): one device-to-device copy into a
    flat buffer, one all-reduce on it (NCCL on the rank's GPU), one copy
    back; nothing crosses to the host.  Returns the bytes each rank
    contributes."""
    import torch.distributed as dist
    buf = _bp_buffer(ctx)
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    ctx.copy_backprojectors_from(buf)
    return int(buf.numel()) * 8


def owner_of_class(iclass: int, world: int) -> int:
    """The rank that reconstructs class iclass when the back-projectors are
    reduced by class: round-robin, as the reference deals classes to nodes
    (src/map_model.cpp:621-666)."""
    return iclass % world


def reduce_backprojectors_by_class(ctx, nr_classes: int, group=None) -> list:
    """Class-partitioned exchange (the reference's MAPModel::reduceData
    without the all-reduce, src/map_model.cpp:621-666): class k's
    back-projector is summed onto rank owner_of_class(k) only, on the
    device, so that each rank reconstructs its own classes; the other ranks'
    copies of class k are left as they were.  Returns the classes this rank
    owns."""
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    buf = _bp_buffer(ctx)
    vox = buf.numel() // (3 * nr_classes)
    data, weight = buf[:2 * vox * nr_classes], buf[2 * vox * nr_classes:]
    for k in range(nr_classes):
        dst = owner_of_class(k, world)
        dist.reduce(data[2 * vox * k:2 * vox * (k + 1)], dst=dst, op=dist.ReduceOp.SUM, group=group)
        dist.reduce(weight[vox * k:vox * (k + 1)], dst=dst, op=dist.ReduceOp.SUM, group=group)
    ctx.copy_backprojectors_from(buf)
    return [k for k in range(nr_classes) if owner_of_class(k, world) == rank]


def broadcast_class_maps(maps, group=None):
    """After a class-partitioned reconstruction: every rank receives every
    class's map from its owner (the reference's broadcast of the new
    references).  maps: one tensor per class, on the rank's device, the
    owner's holding its reconstruction; all of them are overwritten in place."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    for k, m in enumerate(maps):
        dist.broadcast(m, src=owner_of_class(k, world), group=group)
    return maps


def max_over_ranks(value: float, device="cpu") -> float:
    """The maximum of a per-rank scalar (e.g. device time of a step)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
