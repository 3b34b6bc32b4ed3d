"""One process per GPU for the two hot paths, which shard without exchange.

The reference distributes trajectories over MPI groups (`MQCT_SOURCE_CODES/head.f`)
and reduces the per-trajectory results for the cross sections
(`MQCT_SOURCE_CODES/propagator.f:4752-4983`).  Here each rank propagates (or
builds) its own share on its own GPU; the only collectives are the ones that
assemble results and the max-over-ranks timing, both on the host side of the
path, through `torch.distributed` (NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

import numpy as np


def shard(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous share [begin, end) of n items for `rank` of `world` (the first
    n % world ranks take one more)."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError(f"bad shard request n={n} rank={rank} world={world}")
    q, r = divmod(n, world)
    begin = rank * q + min(rank, r)
    return begin, begin + q + (1 if rank < r else 0)


def max_over_ranks(x: float, dist=None, device=None) -> float:
    """Largest value of x over the ranks (identity without a process group)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_rows(local: np.ndarray, n_total: int, dist=None, device=None) -> np.ndarray | None:
    """Concatenate the ranks' row blocks (rank order, as `shard` splits them) on
    every rank.  Blocks may differ in length by one row."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return np.asarray(local)
    import torch
    world = dist.get_world_size()
    local = np.ascontiguousarray(local, dtype=np.float64)
    rows = local.shape[0]
    width = int(np.prod(local.shape[1:])) if local.ndim > 1 else 1
    cap = -(-n_total // world)  # ceil: the largest share
    buf = torch.zeros((cap, width), dtype=torch.float64, device=device)
    if rows:
        buf[:rows] = torch.from_numpy(local.reshape(rows, width)).to(buf.device)
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    out = []
    for r in range(world):
        b, e = shard(n_total, r, world)
        out.append(parts[r][: e - b].cpu().numpy())
    full = np.concatenate(out, axis=0)
    return full.reshape((n_total,) + tuple(local.shape[1:]))
