"""One evaluation sharded over several GPUs (one process per GPU).

The reference splits the BFS sources of one evaluation over MPI ranks --
rank r takes source chunks r, r+procs, ... (general/evaluation.c:166) -- and
joins the partial results with two scalar all-reduces: MAX of the diameter
and SUM of the distance sum (general/evaluation.c:247-248).  Here each rank
runs its strided share of the source windows on its own GPU
(ggb_eval_general_partial) and the ranks join the same two scalars with
torch.distributed (NCCL between GPUs, gloo on CPU).  That 16-byte exchange is
the only communication: sources are independent, and the adjacency (at most a
few MiB) is replicated, not exchanged.
"""
from __future__ import annotations

from typing import Callable

import numpy as np

from ._native import ggb_partial
from .evaluator import Result, evaluate_partial, finish_general


def allreduce_partial(p: ggb_partial, device=None, group=None) -> tuple[int, int, int]:
    """MAX of (diam, disconnected) and SUM of sum over the ranks of `group`."""
    import torch
    import torch.distributed as dist
    mx = torch.tensor([int(p.diam), int(p.disconnected)], dtype=torch.int64, device=device)
    sm = torch.tensor([int(p.sum)], dtype=torch.int64, device=device)
    dist.all_reduce(mx, op=dist.ReduceOp.MAX, group=group)
    dist.all_reduce(sm, op=dist.ReduceOp.SUM, group=group)
    return int(mx[0].item()), int(mx[1].item()), int(sm[0].item())


def evaluate_sharded(adj, based_nodes: int | None = None, groups: int = 1, added_centers: int = 0,
                     group=None, device=None,
                     partial_fn: Callable[..., ggb_partial] | None = None) -> Result:
    """Exact APSP of one general graph with its source windows spread over the
    ranks of `group`; every rank returns the full result.  `partial_fn`
    replaces the GPU partial (tests pass a CPU stand-in)."""
    import torch.distributed as dist
    a = np.ascontiguousarray(adj, dtype=np.int32)
    nodes = a.shape[0]
    if based_nodes is None:
        based_nodes = (nodes - added_centers) // groups
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    fn = partial_fn or evaluate_partial
    p = fn(a, rank, world, based_nodes=based_nodes, groups=groups, added_centers=added_centers)
    diam, disc, total = allreduce_partial(p, device=device, group=group)
    return finish_general(nodes, diam, disc, total)
