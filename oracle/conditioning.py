"""Which texture outputs are well conditioned (checker infrastructure: used by
the tests, smoke() and bench.py's CPU-baseline leg beside the FP64 oracle).

The camera fusion of the texture stage (tile_combine_rgba) takes discrete
choices -- best and second-best camera, worst camera for dust removal -- from
weights that can be equal to within float32 rounding.  Near such a tie, any
two correct implementations that round differently (the reference's
butterflies with 6-digit constants, this library's butterflies with exact
constants, the FP64 oracle's matrix products) may legitimately produce
different outputs.

A texture output is called *stable* when the FP64 oracle reproduces it to
1e-5 (relative to the slice maximum) both after its input CLT is perturbed by
random relative noise of 1e-6 -- about the size of the differences between
float32 evaluations -- in each of eight trials, and when its window tables
are rounded to 6 decimals
as the reference's printed tables are (the 1/sin^4 edge weighting of the
fusion amplifies that rounding, 3.8e-5 at the first tap).  The oracle keeps
the camera weights in float32, as the reference does, so exact float ties
resolve the same way.  Parity of texture outputs is checked, slice by slice,
on stable outputs; the fraction of unstable ones is bounded.  On smooth
scenes the colour and alpha slices are stable almost everywhere; the port
weights of high-dynamic-range scenes, whose weights sit near the 1e-4 floor,
are the ill-conditioned ones.

Random trials sample the near-tie pixels rather than enumerate them: on the
HDR test scene the flagged fraction grows from 0.008% of the colour outputs
with two trials to 0.015% with eight and 0.018% with sixteen.  The smallest
relative gap between the weights behind each discrete choice (the oracle's
`margin`) does not separate them either: exact ties at the 1e-4 floor are
common and mostly harmless (10% of a smooth scene's pixels have a gap below
1e-5, of which a few hundredths of a percent move under perturbation).
"""
import numpy as np

EPS = 1e-6
TOL = 1e-5


def texture_outputs(oracle, case, clt64, idx, keep_weights=0, colors=3):
    ns = (12 if keep_weights else 4) if colors == 3 else (8 if keep_weights else 2)
    out = np.zeros((len(idx), ns * 256))
    oracle.textures_accumulate(case.geom, None, clt64, idx, case.port_offsets, colors=colors,
                               keep_weights=keep_weights, texture_stride=ns * 256, texture_tiles=out)
    return out.reshape(len(idx), ns, 16, 16)


def unstable_mask(oracle, case, clt64, idx, keep_weights=0, colors=3, trials=8, seed=100, eps=EPS):
    """(unstable [n][ns][16][16] bool per slice, oracle outputs [n][ns][16][16]);
    eps: the relative size of the input perturbations (the probed path's own
    error level; 1e-6 for float32 evaluations)"""
    base = texture_outputs(oracle, case, clt64, idx, keep_weights, colors)
    scale = np.maximum(np.abs(base).max(axis=(0, 2, 3)), 1e-300)[None, :, None, None]
    bad = np.zeros(base.shape, dtype=bool)
    for t in range(trials):
        rng = np.random.default_rng(seed + t)
        pert = [c * (1.0 + eps * rng.standard_normal(c.shape)) for c in clt64]
        o = texture_outputs(oracle, case, pert, idx, keep_weights, colors)
        bad |= np.abs(o - base) / scale > TOL
    oracle.set_table_mode(1)
    try:
        o = texture_outputs(oracle, case, clt64, idx, keep_weights, colors)
    finally:
        oracle.set_table_mode(0)
    bad |= np.abs(o - base) / scale > TOL
    return bad, base


def unstable_image_mask(bad_tiles, idx, woi, TX, shape, slices):
    """Map unstable tile pixels ([n][16][16], any slice) of the listed tiles
    into the overlapped RGBA image ([slices * h][w]); shape = (h, w) of one
    slice."""
    h, w = shape
    m = np.zeros((h, w), dtype=bool)
    for k, code in enumerate(idx):
        tile = int(code) >> 8
        ty, tx = divmod(tile, TX)
        y0, x0 = (ty - woi[1]) * 8, (tx - woi[0]) * 8
        if y0 < 0 or x0 < 0:
            continue
        m[y0:y0 + 16, x0:x0 + 16] |= bad_tiles[k]
    return np.concatenate([m] * slices, axis=0)


class _Frame:
    """geometry and port offsets of a frame, as texture_outputs reads them"""

    def __init__(self, geom, port_offsets):
        self.geom = geom
        self.port_offsets = port_offsets


def unstable_tiles(oracle, geom, port_offsets, clt, tiles, keep_weights=0, colors=3, chunk=8192, trials=8, eps=EPS):
    """unstable_mask for the tiles `tiles` (tile numbers) of a large frame,
    in chunks, so host memory stays bounded: each chunk's CLT is gathered into
    compact FP64 arrays and its tiles renumbered 0..n-1 (the per-tile outputs
    depend only on a tile's own CLT).  Returns (unstable, oracle outputs),
    [n][ns][16][16] each, in the order of `tiles`."""
    tiles = np.asarray(tiles, dtype=np.int64)
    fr = _Frame(geom, port_offsets)
    chunk = max(1, min(chunk, (geom["img_width"] // 8) * (geom["img_height"] // 8)))
    bads, bases = [], []
    for a in range(0, tiles.size, chunk):
        t = tiles[a:a + chunk]
        sub = [np.asarray(c, dtype=np.float32).reshape(-1, 768)[t].astype(np.float64).reshape(-1) for c in clt]
        idx = ((np.arange(t.size, dtype=np.int64) << 8) | 0x80 | 0xF).astype(np.int32)
        b, o = unstable_mask(oracle, fr, sub, idx, keep_weights, colors, trials=trials, eps=eps)
        bads.append(b)
        bases.append(o)
    return np.concatenate(bads), np.concatenate(bases)


def stable_errors(got, want, keep):
    """Per-slice comparison on the stable outputs: the unstable fraction, the
    largest error relative to the slice maximum of `want`, and the fraction of
    stable outputs above 1e-5.  got, want, keep: [n][ns][...] arrays."""
    out = []
    for s in range(want.shape[1]):
        g = np.asarray(got[:, s], np.float64)
        w = np.asarray(want[:, s], np.float64)
        k = keep[:, s]
        den = np.abs(w).max() or 1.0
        e = np.abs(g - w)[k] / den
        out.append({"unstable": float(1.0 - k.mean()), "max": float(e.max()) if e.size else 0.0,
                    "frac_gt_1e-5": float((e > TOL).mean()) if e.size else 0.0})
    return out
