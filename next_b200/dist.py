"""Host-side helpers for sharding one system over several GPUs.

One process per GPU, launched by torchrun (or any launcher that sets RANK /
WORLD_SIZE / LOCAL_RANK); torch.distributed is only the plumbing that carries
the 128-byte NCCL id from rank 0 to the others and the max-over-ranks timing.
The library (next_dist_attach) then does the per-step force exchange with its
own NCCL communicator on its own stream.

Share of rank r: working positions [r*c, min(n, (r+1)*c)), c = ceil(n/world)
-- the same formula the library uses, so every body has exactly one owner.
Compare the reference's slice [r*N/size, (r+1)*N/size) (src/gravity/step.h:54-55).

Independent systems (an ensemble) are not sliced by position but split
whole over the ranks, balanced by their N log N work (split_systems).
"""
from __future__ import annotations

import os


def env_rank():
    """(rank, world, local_rank) from the launcher's environment."""
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def partition(n: int, world: int, rank: int):
    """(lo, hi, chunk): the bodies whose forces `rank` computes."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    chunk = (n + world - 1) // world
    lo = min(n, rank * chunk)
    hi = min(n, lo + chunk)
    return lo, hi, chunk


def padded_length(n: int, world: int) -> int:
    """Length of each rank's force lanes: `world` equal chunks of ceil(n/world),
    so the in-place all-gather sends chunk r from offset r*chunk of the same
    buffer it receives into (the layout next_dist_attach allocates)."""
    return -(-n // world) * world


def system_cost(sizes):
    """Work estimate of a Barnes-Hut step per system: N log2 N (walk
    interactions grow as log N per body; the build is ~N per system)."""
    import numpy as np
    sizes = np.asarray(sizes, dtype=np.float64)
    return sizes * np.log2(np.maximum(sizes, 2.0))


def split_systems(sizes, world: int):
    """Independent systems over `world` ranks, balanced by N log2 N.

    Longest-processing-time greedy: systems in decreasing cost, each to the
    rank with the least work so far (ties to the lower rank), which keeps the
    largest rank load within a few per cent of the mean for ensembles of
    uneven sizes.  Returns, per rank, the sorted system numbers it owns.
    Every rank computes the same split from the same sizes.
    """
    import numpy as np
    if world < 1:
        raise ValueError("world must be >= 1")
    cost = system_cost(sizes)
    order = np.lexsort((np.arange(cost.shape[0]), -cost))   # cost descending, stable by index
    load = np.zeros(world)
    owned = [[] for _ in range(world)]
    for s in order:
        r = int(np.argmin(load))
        owned[r].append(int(s))
        load[r] += cost[s]
    return [np.array(sorted(o), dtype=np.int64) for o in owned]


def select_systems(bodies, offsets, systems):
    """The bodies of `systems` (sorted system numbers) and their new offsets."""
    import numpy as np
    offsets = np.asarray(offsets, dtype=np.int64)
    idx = np.concatenate([np.arange(offsets[s], offsets[s + 1]) for s in systems]) if len(systems) else \
        np.zeros(0, dtype=np.int64)
    sizes = np.diff(offsets)[np.asarray(systems, dtype=np.int64)]
    new_offsets = np.zeros(len(systems) + 1, dtype=np.int64)
    new_offsets[1:] = np.cumsum(sizes)
    return {k: v[idx] for k, v in bodies.items()}, new_offsets


def broadcast_bytes(payload: bytes | None, size: int, src: int = 0, group=None) -> bytes:
    """Send `size` bytes from rank `src` to all ranks of the torch process group."""
    import torch
    import torch.distributed as dist
    backend = dist.get_backend(group)
    device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    if dist.get_rank(group) == src:
        t = torch.tensor(list(payload), dtype=torch.uint8, device=device)
    else:
        t = torch.zeros(size, dtype=torch.uint8, device=device)
    dist.broadcast(t, src=src, group=group)
    return bytes(t.cpu().tolist())


def shared_unique_id(group=None) -> bytes:
    """The NCCL id made on rank 0, delivered to every rank."""
    import torch.distributed as dist
    from .native import dist_unique_id
    uid = dist_unique_id() if dist.get_rank(group) == 0 else None
    return broadcast_bytes(uid, 128, src=0, group=group)


def attach(sim, group=None):
    """Join `sim` to a sharded run over the ranks of the torch process group."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    sim.dist_attach(rank, world, shared_unique_id(group) if world > 1 else None)
    return rank, world
