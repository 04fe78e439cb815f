"""Multi-GPU evaluation: one process per GPU, each evaluating its shard of the
blocks (bv_opts.shard_count / shard_index), then one exchange of the FP64
partial log-likelihoods.

Blocks are independent given theta, so the only data-path exchange per
evaluation is 8 bytes per rank.  The partials are all-gathered and summed in
rank order, so every rank returns the same, reproducible value.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def combine_partials(partial: float, group=None, device=None) -> float:
    """Sum of every rank's partial log-likelihood, in rank order."""
    if not dist.is_available() or not dist.is_initialized():
        return float(partial)
    world = dist.get_world_size(group)
    backend = dist.get_backend(group)
    dev = device if device is not None else (torch.device("cuda", torch.cuda.current_device())
                                             if backend == "nccl" else torch.device("cpu"))
    t = torch.tensor([partial], dtype=torch.float64, device=dev)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    total = 0.0
    for p in parts:  # fixed rank order
        total += float(p.item())
    return total


class ShardedLlh:
    """This rank's share of one log-likelihood evaluation.

    `data` is a LlhData built with shard_count = world size and
    shard_index = rank; calling the object returns the full log-likelihood on
    every rank."""

    def __init__(self, data, group=None):
        self.data = data
        self.group = group

    def __call__(self, theta) -> float:
        return combine_partials(self.data(theta), self.group)
