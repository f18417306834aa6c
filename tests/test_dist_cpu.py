"""Host logic of the sharded (multi-GPU) path, on CPU with gloo, world size 2.

The device side (restricted walk + NCCL all-gather) needs GPUs; here two
processes check what the ranks agree on over their process group: the body
shares tile [0, n) exactly with equal padded chunks (the layout the in-place
all-gather needs), an in-place all-gather over that padded layout leaves every
rank with every body's value, the NCCL id made on rank 0 reaches rank 1
intact, and the ensemble split (whole systems per rank, balanced by N log N)
is the same on every rank, covers each system once and balances the load.
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
        from next_b200.dist import padded_length, shared_unique_id
        lo, hi, chunk = partition(n, world, rank)
        got = [None] * world
        dist.all_gather_object(got, (lo, hi, chunk))
        uid = shared_unique_id()
        ids = [None] * world
        dist.all_gather_object(ids, uid)
        # The force exchange's layout: lanes of padded_length(n, world), each
        # rank fills its share and all-gathers chunk r from offset r*chunk of
        # the same buffer it receives into (ncclAllGather in place).
        buf = torch.full((padded_length(n, world),), float("nan"), dtype=torch.float64)
        buf[lo:hi] = torch.arange(lo, hi, dtype=torch.float64) * 0.5 + 1.0
        views = list(buf.split(chunk))
        dist.all_gather(views, views[rank].clone())
        ok = bool(torch.equal(buf[:n], torch.arange(n, dtype=torch.float64) * 0.5 + 1.0))
        out[rank] = (got, ids, ok)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n", [1, 7, 1_048_576, 1_000_003])
def test_shares_tile_and_ids_agree(n):
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), n, out), nprocs=world, start_method="spawn")
    shares, ids, ok0 = out[0]
    assert out[1][0] == shares
    assert ok0 and out[1][2]          # every rank holds every body's force after the exchange
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


def _split_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        import numpy as np
        from next_b200 import ic
        from next_b200.dist import select_systems, split_systems, system_cost
        b, offsets = ic.ensemble(64, seed=3, nmin=64, nmax=4096)
        mine = split_systems(np.diff(offsets), world)[rank]
        sub, sub_off = select_systems(b, offsets, mine)
        # the rank's bodies are exactly its systems' bodies, in system order
        want = np.concatenate([b["x"][offsets[s]:offsets[s + 1]] for s in mine])
        got = [None] * world
        dist.all_gather_object(got, (mine.tolist(), float(system_cost(np.diff(sub_off)).sum()),
                                     bool(np.array_equal(sub["x"], want)), int(sub_off[-1])))
        out[rank] = got
    finally:
        dist.destroy_process_group()


def test_ensemble_split_agrees_and_balances():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_split_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
    assert out[0] == out[1]
    owned = [set(o[0]) for o in out[0]]
    assert owned[0].isdisjoint(owned[1]) and owned[0] | owned[1] == set(range(64))
    loads = [o[1] for o in out[0]]
    assert max(loads) / (sum(loads) / world) - 1 < 0.05
    assert all(o[2] for o in out[0])


@pytest.mark.parametrize("world", [2, 4, 8])
def test_split_of_the_256_system_ensemble_within_5_percent(world):
    import numpy as np
    from next_b200 import ic
    from next_b200.dist import split_systems, system_cost
    _, offsets = ic.ensemble(256, seed=3)
    sizes = np.diff(offsets)
    parts = split_systems(sizes, world)
    assert sorted(np.concatenate(parts).tolist()) == list(range(256))
    loads = [float(system_cost(sizes[p]).sum()) for p in parts]
    assert max(loads) / (sum(loads) / world) - 1 < 0.05
