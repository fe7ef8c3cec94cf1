"""Work partitioning across GPUs (one process per GPU).

Frames are independent, so the default multi-GPU layout is frame replicas:
rank r processes frames r, r + N, r + 2N, ... with its own copy of the
kernel tables; no data crosses between GPUs.

One frame can also be split by tile rows (`row_bands`).  The forward CLT and
the correlations of a band's tiles need nothing from the other bands.  The
overlapped RGBA texture needs two things: the band's list builder must see
the tile row above and below the band (neighbour bits, border classes and
the alpha fade of the band's edge tiles depend on them; `band_tasks` and
tp_generate_RBGA_rows), and the 8 pixel rows that the band's last tile row
adds below it belong to the next band, which adds them to its own first
rows: one strip exchange per frame (`band_image_rows`, `exchange_strip`).
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


def band_tasks(tasks, first, last, tiles_y, halo=1):
    """Tasks (TASK_DTYPE records) of tile rows [first - halo, last + halo)
    clipped to the frame: the input of a band's texture list."""
    ty = tasks["txy"] >> 16
    lo, hi = max(0, first - halo), min(tiles_y, last + halo)
    return tasks[(ty >= lo) & (ty < hi)]


def band_core_tasks(tasks, first, last):
    """Tasks of tile rows [first, last): the band's forward CLT and correlations."""
    ty = tasks["txy"] >> 16
    return tasks[(ty >= first) & (ty < last)]


def band_image_rows(woi, first, last, tiles_y):
    """Pixel rows of a band's RGBA image (relative to its window of interest
    woi = [x0, y0, w, h] in tiles, as generate_RBGA returns it).

    Returns dict(own=(local0, global0, rows), send=(local0, global0, rows)):
    `own` are the rows [8 first, 8 last) the band keeps (through the image's
    last row for the last band), `send` the 8 rows [8 last, 8 last + 8) it
    adds to the next band's image (none for the last band); both clipped to
    the image, which covers the global rows [8 y0, 8 (y0 + h + 1))."""
    y0, h = int(woi[1]), int(woi[3])
    img0, img1 = 8 * y0, 8 * (y0 + h + 1)

    def clip(g0, g1):
        a, b = max(g0, img0), min(g1, img1)
        return (a - img0, a, b - a) if b > a else (0, g0, 0)

    own = clip(8 * first, 8 * last + (8 if last >= tiles_y else 0))
    send = clip(8 * last, 8 * last + 8) if last < tiles_y else (0, 8 * last, 0)
    return {"own": own, "send": send}


def exchange_strip(strip_out, strip_in, rank, world, group=None):
    """Send this band's strip (the rows it adds below itself, all slices) to
    rank + 1 and receive the strip of rank - 1 into strip_in (torch tensors
    on the process group's device); every rank takes part, the first only
    sends and the last only receives.  Even ranks send first, odd ranks
    receive first, so blocking send / recv pairs never wait on each other."""
    import torch.distributed as dist
    up, down = rank - 1, rank + 1
    if rank % 2 == 0:
        if down < world:
            dist.send(strip_out, down, group=group)
        if up >= 0:
            dist.recv(strip_in, up, group=group)
    else:
        if up >= 0:
            dist.recv(strip_in, up, group=group)
        if down < world:
            dist.send(strip_out, down, group=group)
