"""Multi-GPU form: sources sharded across ranks, one reduction of bc[].

Brandes dependencies of different sources are independent, so N ranks (one
process per GPU, torch.distributed) each run their own block of sources on a
full replica of the graph and the FP64 bc vectors are summed once.  This is
the only exchange of the path; the reference's 2-D row/column frontier
exchange over MPI (bc2d.h:28-96, cuda_kernels.cu:338-394, 601-649) is not
needed on a 1x1 tile and is not rebuilt.
"""
from __future__ import annotations

import numpy as np


def shard_sources(sources, rank: int, world: int, mode: str = "block") -> np.ndarray:
    """This rank's share of the source list.

    block:  contiguous blocks, sizes differ by at most one (rank order kept);
    cyclic: sources[rank::world] (spreads neighbouring ids across ranks)."""
    s = np.ascontiguousarray(np.asarray(sources, dtype=np.uint32))
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    if mode == "cyclic":
        return np.ascontiguousarray(s[rank::world])
    if mode != "block":
        raise ValueError(f"unknown shard mode {mode}")
    q, r = divmod(len(s), world)
    lo = rank * q + min(rank, r)
    hi = lo + q + (1 if rank < r else 0)
    return s[lo:hi]


def reduce_bc(bc, group=None, deterministic: bool = False):
    """Sums the per-rank bc tensors in place over the process group.

    deterministic=False: one all_reduce (NCCL on GPU tensors, gloo on CPU).
    deterministic=True: all_gather the partials and add them in rank order,
    so the FP64 result does not depend on the collective's summation order."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    if world == 1:
        return bc
    if not deterministic:
        dist.all_reduce(bc, group=group)
        return bc
    parts = [torch.empty_like(bc) for _ in range(world)]
    dist.all_gather(parts, bc, group=group)
    acc = parts[0].clone()
    for p in parts[1:]:
        acc += p
    bc.copy_(acc)
    return bc
