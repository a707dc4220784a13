"""One molecule over several GPUs: contiguous slices of the packed vector, one per rank.

Shell quartets are independent; rank r computes the quartets whose highest shell index lies
in its shell range, which are exactly the integrals of one contiguous slice of the packed
iindex vector (molints_shard_range / molints_plan_create_shard).  The compute needs no
collective.  ``gather_slices`` assembles the full vector on every rank when a caller wants
it (an all-gather of the slices, padded to the longest; NCCL between GPUs, gloo on CPU).
"""
from __future__ import annotations

import numpy as np


def shard_ranges(shells, nshards: int):
    """[(lo, hi)] of every shard: they tile [0, npacked) in order."""
    from . import engine as E
    return [E.shard_range(shells, r, nshards) for r in range(nshards)]


def compute_shard(engine, shells, rank: int, world: int, out_device_ptr: int, **opts):
    """Queue rank `rank`'s slice into out_device_ptr (hi - lo doubles) on the engine's
    stream; returns the plan (keep it alive until the work is done) and (lo, hi)."""
    plan = engine.plan_shard(shells, rank, world, **opts)
    plan.execute(out_device_ptr)
    return plan, plan.slice


def gather_slices(local, shells, group=None):
    """All ranks' slices (torch tensors of length hi - lo, in rank order) concatenated into
    the full packed vector on every rank."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    ranges = shard_ranges(shells, world)
    longest = max(hi - lo for lo, hi in ranges)
    pad = torch.zeros(longest, dtype=local.dtype, device=local.device)
    pad[:local.numel()] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([p[:hi - lo] for p, (lo, hi) in zip(parts, ranges)])


def owner_of(shells, nshards: int, i: int, j: int, k: int, l: int) -> int:
    """The shard whose slice holds integral (ij|kl) (0-based functions)."""
    from .basis import Shells  # noqa: F401
    def tri(n):
        return n * (n + 1) // 2
    ij = tri(max(i, j)) + min(i, j)
    kl = tri(max(k, l)) + min(k, l)
    idx = tri(max(ij, kl)) + min(ij, kl)
    for r, (lo, hi) in enumerate(shard_ranges(shells, nshards)):
        if lo <= idx < hi:
            return r
    raise IndexError(idx)


def shell_of_function(shells) -> np.ndarray:
    off = shells.fn_offsets()
    out = np.zeros(shells.nbf, dtype=np.int64)
    for s in range(shells.nshell):
        out[off[s]:off[s + 1]] = s
    return out
