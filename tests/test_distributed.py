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


def _strip_worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from tile_processor_gpu_b200.sharding import exchange_strip
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # each band's image: 4 slices of 24 rows x 10 columns; its last 8 rows are the strip it sends down
        img = torch.full((4, 24, 10), float(rank + 1))
        img[:, 16:] = 100.0 * (rank + 1)
        strip_in = torch.zeros(4, 8, 10)
        exchange_strip(img[:, 16:].contiguous(), strip_in, rank, world)
        img[:, :8] += strip_in
        out[rank] = img[:, :8].clone().numpy()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_strip_exchange_gloo(world):
    """Every band adds the strip of the band above into its first 8 rows; the
    first band receives nothing."""
    import numpy as np
    import torch.multiprocessing as mp
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_strip_worker, args=(world, port, out), nprocs=world, join=True)
    for rank in range(world):
        want = float(rank + 1) + (100.0 * rank if rank > 0 else 0.0)
        assert np.all(out[rank] == want), (rank, out[rank][0, 0, 0])


def test_band_tasks_and_rows():
    """Band task selection (band rows plus one halo row each side, clipped)
    and the pixel rows each band keeps or sends, which together cover every
    image row of a dense frame exactly once (the strips twice: own + sent)."""
    import numpy as np
    from tile_processor_gpu_b200 import synth
    from tile_processor_gpu_b200.sharding import band_core_tasks, band_image_rows, band_tasks
    geom = synth.geometry(128, 96)
    TX, TY, _ = synth.tiles(geom)
    tasks = synth.tasks_grid(geom)
    cover = np.zeros((TY + 1) * 8, int)
    for first, last, _ in row_bands(TY, 3):
        t = band_tasks(tasks, first, last, TY)
        ty = t["txy"] >> 16
        assert ty.min() == max(0, first - 1) and ty.max() == min(TY - 1, last)
        core = band_core_tasks(tasks, first, last)["txy"] >> 16
        assert core.min() == first and core.max() == last - 1
        # window of interest as generate_RBGA returns it: x0, y0, width and height in tiles
        woi = [0, max(0, first - 1), TX, min(TY - 1, last) - max(0, first - 1) + 1]
        r = band_image_rows(woi, first, last, TY)
        l0, g0, n = r["own"]
        assert l0 == g0 - 8 * woi[1] and n > 0
        cover[g0:g0 + n] += 1
        l0, g0, n = r["send"]
        if last < TY:
            assert (g0, n) == (8 * last, 8)
    assert np.all(cover == 1)
