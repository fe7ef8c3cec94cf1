"""Multi-process host logic with world_size 2 on the gloo backend (CPU):
frame sharding covers every frame once, the bench's max-over-ranks timing
reduction and barrier work, and row bands tile the frame."""
import os
import socket

import pytest

from tile_processor_gpu_b200.sharding import frame_shard, row_bands


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, num_frames, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = frame_shard(num_frames, rank, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        # the bench's timing reduction: every rank sees the max
        t = bench.max_over_ranks(dist, float(10 + rank))
        bench.barrier(dist)
        out[rank] = (sorted(f for g in gathered for f in g), t)
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    import torch.multiprocessing as mp
    port = _free_port()
    world, frames = 2, 9
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, frames, out), nprocs=world, join=True)
    for rank in range(world):
        allf, t = out[rank]
        assert allf == list(range(frames))
        assert t == 11.0


@pytest.mark.parametrize("ty,world", [(242, 1), (242, 2), (242, 8), (32, 3), (3, 8)])
def test_row_bands(ty, world):
    bands = row_bands(ty, world)
    assert len(bands) == world
    assert bands[0][0] == 0 and bands[-1][1] == ty
    for (a, b, h), (c, d, _) in zip(bands, bands[1:]):
        assert b == c
    assert all(h in (0, 1) for _, _, h in bands)
    assert bands[-1][2] == 0


def test_frame_shard_rejects_bad_rank():
    with pytest.raises(ValueError):
        frame_shard(4, 2, 2)
