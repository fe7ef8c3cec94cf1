"""Work partitioning across GPUs (one process per GPU).

Frames are independent, so the default multi-GPU layout is
frame replicas: rank r processes frames r, r + N, r + 2N, ... with its own
copy of the kernel tables; no data crosses between GPUs.  Splitting one frame
by tile rows is also independent for the forward CLT and the correlation;
only the overlapped RGBA texture would need an 8-pixel halo exchanged between
neighbouring bands (`row_bands` reports it).
"""


def frame_shard(num_frames, rank, world):
    """Frame indices processed by `rank` (round robin)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d outside world %d" % (rank, world))
    return list(range(rank, num_frames, world))


def row_bands(tiles_y, world):
    """Split tiles_y tile rows into `world` contiguous bands.

    Returns [(first_row, last_row_exclusive, halo_rows_below)] per rank; the
    halo is the 8-pixel strip of the overlapped texture that a band's last
    tile row adds into the next band's first rows (1 tile row), 0 for the
    last band and for empty bands."""
    if world < 1:
        raise ValueError("world must be >= 1")
    base, extra = divmod(tiles_y, world)
    out, start = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        end = start + n
        out.append((start, end, 1 if (n and end < tiles_y) else 0))
        start = end
    return out
