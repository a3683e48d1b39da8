"""Instance sharding of the per-frame path across GPUs (no counterpart in the
reference, which runs on one host).

One process per GPU (torch.distributed).  Given the camera pose, each
instance's allocation, integration and object tracking are independent of
the others (kfusion.cpp:397-413, 607-648); only the composite raycast
(rendering.cpp:81-133) couples them, per pixel.  So every rank registers every
instance (poses and labels), holds and integrates the volumes of its own
instances, records its instances' raycasts (mf_raycast_records), and the
records are gathered so that every rank folds the same composite maps
(mf_raycast_fold) -- the maps one GPU would make, bit for bit.

These helpers are the host side of that exchange: the partition of the
instances and the gathers (torch.distributed.all_gather: NCCL over
NVLink / NVSwitch for CUDA tensors, gloo for CPU tensors).  No collective
touches a peer's memory other than through the library.
"""
from __future__ import annotations

import torch
import torch.distributed as dist

RECORD_BYTES = 48   # mf_ray_record
ORIGIN_BYTES = 32   # mf_ray_origin


def partition(sizes, world):
    """Instance ids per rank: the background (instance 0) on rank 0, the
    objects largest first onto the rank with the least work so far (work ~
    the volume's voxel count, a bound on its blocks)."""
    load = [0] * world
    out = [[] for _ in range(world)]
    out[0].append(0)
    load[0] += int(sizes[0]) ** 3
    for i in sorted(range(1, len(sizes)), key=lambda i: -int(sizes[i]) ** 3):
        r = min(range(world), key=lambda r: (load[r], r))
        out[r].append(i)
        load[r] += int(sizes[i]) ** 3
    return [sorted(ids) for ids in out]


def _gather_rows(local, parts, n, group=None):
    """local: (len(parts[rank]), ...) tensor of this rank's rows; returns the
    (n, ...) tensor of every rank's rows in instance order."""
    world = len(parts)
    k = max(len(p) for p in parts)
    pad = torch.zeros((k,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[:local.shape[0]] = local
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad, group=group)
    out = torch.empty((n,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    for r, ids in enumerate(parts):
        for j, i in enumerate(ids):
            out[i] = bufs[r][j]
    return out


def gather_records(records, origins, parts, n, group=None):
    """Every instance's raycast records and origin records, in instance order,
    from each rank's records of its own instances: records (k, H, W, 48)
    uint8, origins (k, 32) uint8 -> (n, H, W, 48), (n, 32)."""
    return (_gather_rows(records, parts, n, group), _gather_rows(origins, parts, n, group))


def gather_poses(poses, parts, n, group=None):
    """Every instance's volume pose (n, 4, 4) float32 from each rank's poses of
    its own instances (k, 4, 4), after each rank has tracked its objects."""
    return _gather_rows(poses, parts, n, group)
