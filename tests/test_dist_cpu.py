"""Host logic of the sharded (multi-GPU) path, on CPU with gloo, world size 2.

The device side (restricted walk + NCCL all-gather) needs GPUs; here two
processes check what the ranks agree on over their process group: the body
shares tile [0, n) exactly with equal padded chunks (the layout the in-place
all-gather needs), and the NCCL id made on rank 0 reaches rank 1 intact.
"""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from next_b200.dist import partition  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        from next_b200.dist import shared_unique_id
        lo, hi, chunk = partition(n, world, rank)
        got = [None] * world
        dist.all_gather_object(got, (lo, hi, chunk))
        uid = shared_unique_id()
        ids = [None] * world
        dist.all_gather_object(ids, uid)
        out[rank] = (got, ids)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n", [1, 7, 1_048_576, 1_000_003])
def test_shares_tile_and_ids_agree(n):
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), n, out), nprocs=world, start_method="spawn")
    shares, ids = out[0]
    assert out[1][0] == shares
    chunk = shares[0][2]
    assert all(c == chunk for _, _, c in shares) and chunk * world >= n
    covered = []
    for r, (lo, hi, _) in enumerate(shares):
        assert lo == min(n, r * chunk) and hi - lo <= chunk
        covered += list(range(lo, hi)) if n < 100 else [lo, hi]
    if n < 100:
        assert covered == list(range(n))
    else:
        assert shares[0][0] == 0 and shares[-1][1] == n and shares[0][1] == shares[1][0]
    assert len(ids[0]) == 128 and ids[0] == ids[1] == out[1][1][0]


def test_partition_formula_matches_reference_slicing_sizes():
    # the reference slices [r*N/size, (r+1)*N/size) (step.h:54-55); here equal
    # padded chunks, so no rank's share exceeds ceil(N/size)
    for n in (10, 11, 12):
        for world in (1, 2, 3, 4):
            sizes = [partition(n, world, r)[1] - partition(n, world, r)[0] for r in range(world)]
            assert sum(sizes) == n and max(sizes) == -(-n // world)
