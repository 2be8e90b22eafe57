"""Host logic for running independent simulations on several GPUs.

The reference has no domain decomposition, and the monodomain step has no data
exchange between simulations, so the multi-GPU form is one process per GPU
running its own simulations ("replicas only"): no collective on the step path.
The only cross-rank operations are host-side: timing as the maximum over ranks,
totals as sums, and a deterministic split of a list of simulations over ranks.
They work with the gloo backend (CPU tensors) and with NCCL (CUDA tensors).
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def active() -> bool:
    return dist.is_available() and dist.is_initialized()


def _reduce(x: float, op) -> float:
    if not active() or dist.get_world_size() == 1:
        return float(x)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def reduce_max(x: float) -> float:
    """Maximum of ``x`` over the ranks (every rank gets it)."""
    return _reduce(x, dist.ReduceOp.MAX)


def reduce_sum(x: float) -> float:
    """Sum of ``x`` over the ranks (every rank gets it)."""
    return _reduce(x, dist.ReduceOp.SUM)


def shard(items, rank: int, world: int, weight=None):
    """The items rank ``rank`` of ``world`` runs: largest weight first, each to the
    rank with the least total so far (ties to the lowest rank); every rank computes
    the same split, so no communication is needed.  Items keep their order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank outside [0, world)")
    w = [1.0 if weight is None else float(weight(x)) for x in items]
    load = [0.0] * world
    owner = [0] * len(items)
    for i in sorted(range(len(items)), key=lambda j: (-w[j], j)):
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += w[i]
    return [x for x, o in zip(items, owner) if o == rank]
