"""Sharding a cloth batch over GPUs: one process per GPU, each stepping its own cloths.

Cloths never interact (no cloth-cloth coupling; rigid coupling is one-way, physxcoopa/cloth/cloth.h:28-29),
so the step needs no collective: the batch is split once, greedily by cost (largest first onto the
least-loaded rank, cost = vertices x iterations x substeps, the work of one step), and every rank
steps its share. The one exchange is optional and at frame end: the per-cloth bounds and speed
that the caller's broadphase reads (PhysicsWorld::step_cloths_, world.h:1777-1779, 1837) are
gathered to every rank with an all-gather.
"""
from typing import List, Sequence

import numpy as np


def cloth_cost(vertices: int, iterations: int = 10, substeps: int = 4) -> int:
    """Work of one step of one cloth, in vertex-iteration-substeps."""
    return int(vertices) * int(iterations) * int(substeps)


def partition(costs: Sequence[int], n_ranks: int) -> List[List[int]]:
    """Greedy longest-processing-time bin packing: cloths by decreasing cost (index order on
    ties) onto the least-loaded rank (lowest rank on ties). Deterministic, so every rank computes
    the same split without communicating. Returns each rank's cloth indices, ascending."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be positive")
    order = sorted(range(len(costs)), key=lambda i: (-int(costs[i]), i))
    load = [0] * n_ranks
    shares: List[List[int]] = [[] for _ in range(n_ranks)]
    for i in order:
        r = min(range(n_ranks), key=lambda k: (load[k], k))
        shares[r].append(i)
        load[r] += int(costs[i])
    return [sorted(s) for s in shares]


def gather_results(local: np.ndarray, shares: List[List[int]], n_total: int, group=None) -> np.ndarray:
    """Frame-end exchange: every rank contributes the per-cloth results (a structured array in
    its share's order) and receives all of them in global cloth order. One tensor all-gather of
    the records' bytes, each rank's block padded to the largest share (on the GPU under NCCL, in
    host memory under gloo); the only collective of a sharded step."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rec = local.dtype.itemsize
    width = max(len(s) for s in shares) * rec
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")
    mine = torch.zeros(width, dtype=torch.uint8)
    raw = np.ascontiguousarray(local).view(np.uint8).reshape(-1)
    mine[:len(raw)] = torch.from_numpy(raw.copy())
    mine = mine.to(dev)
    parts = [torch.empty(width, dtype=torch.uint8, device=dev) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    out = np.zeros(n_total, local.dtype)
    for r in range(world):
        block = parts[r].cpu().numpy()[:len(shares[r]) * rec].view(local.dtype)
        out[np.asarray(shares[r], np.int64)] = block
    return out
