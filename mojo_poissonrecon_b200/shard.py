"""Reconstructions of many clouds across the GPUs of one node (replicas).

A single reconstruction does not shard without a halo exchange per smoothing
sweep, but clouds are independent: each rank (one process per GPU, launched by
torchrun) reconstructs a share of the batch on its own GPU and the meshes are
gathered on rank 0.  No collective runs on the data path; the only collectives
are the gather of finished results and the max-over-ranks reduction of timings.

The partition is greedy longest-processing-time by estimated HBM footprint
(serve.footprint_bytes, a proxy for work): clouds in decreasing footprint order,
each to the rank with the least assigned so far (ties to the lower rank), so it
is deterministic and the same on every rank without communication.
"""

from __future__ import annotations

import torch

from . import serve


def partition(footprints, world: int) -> list[list[int]]:
    """Indices of the items each of `world` ranks takes (ascending per rank)."""
    if world < 1:
        raise ValueError("world must be positive")
    order = sorted(range(len(footprints)), key=lambda i: (-int(footprints[i]), i))
    load = [0] * world
    shares: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += int(footprints[i])
        shares[r].append(i)
    return [sorted(s) for s in shares]


def _dist():
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        raise RuntimeError("torch.distributed is not initialised (launch one process per GPU with torchrun)")
    return dist


def reconstruct_sharded(clouds, *, runner=None, lanes: int = 4, **kwargs) -> list | None:
    """Reconstruct `clouds` ((points, normals) or (points, normals, depth)
    tuples, identical on every rank) across the ranks of the default process
    group.  Returns the results in input order on rank 0, None on the others.

    runner: optional callable(list of clouds) -> list of results that replaces
    the GPU batch (serve.reconstruct_batch on this rank's GPU)."""
    dist = _dist()
    rank, world = dist.get_rank(), dist.get_world_size()
    footprints = [serve.footprint_bytes(int(c[2]) if len(c) == 3 else int(kwargs.get("depth", 6)), len(c[0]))
                  for c in clouds]
    mine = partition(footprints, world)[rank]
    local = [clouds[i] for i in mine]
    if runner is None:
        results = serve.reconstruct_batch(local, lanes=lanes, **kwargs) if local else []
    else:
        results = list(runner(local))
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(list(zip(mine, results)), gathered, dst=0)
    if rank != 0:
        return None
    out = [None] * len(clouds)
    for share in gathered:
        for i, result in share:
            out[i] = result
    return out


def max_over_ranks(value: float, device: torch.device | None = None) -> float:
    """The largest `value` over the ranks (the job's time is its slowest rank's)."""
    dist = _dist()
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
