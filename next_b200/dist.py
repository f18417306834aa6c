"""Host-side helpers for sharding one system over several GPUs.

One process per GPU, launched by torchrun (or any launcher that sets RANK /
WORLD_SIZE / LOCAL_RANK); torch.distributed is only the plumbing that carries
the 128-byte NCCL id from rank 0 to the others and the max-over-ranks timing.
The library (next_dist_attach) then does the per-step force exchange with its
own NCCL communicator on its own stream.

Share of rank r: working positions [r*c, min(n, (r+1)*c)), c = ceil(n/world)
-- the same formula the library uses, so every body has exactly one owner.
Compare the reference's slice [r*N/size, (r+1)*N/size) (src/gravity/step.h:54-55).
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
