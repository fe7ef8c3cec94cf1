"""Seeded parity cases shared by the tests (host side only, no GPU needed).

A Case bundles one frame's inputs in the reference's layouts.  The source
images are allocated with `pad_rows` extra rows and a pitch wider than the
image, both filled with seeded random values, so any difference in how the
fetch addresses pixels outside the image shows up in the outputs instead of
being hidden by zeros.
"""
import numpy as np

from tile_processor_gpu_b200 import synth


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).max() if b.size else 0.0
    if den == 0.0:
        return float(np.abs(a - b).max()) if a.size else 0.0
    return float(np.abs(a - b).max() / den)


def rms_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.sqrt((b * b).mean()) if b.size else 0.0
    return float(np.sqrt(((a - b) ** 2).mean()) / den) if den else 0.0


class Case:
    def __init__(self, width=256, height=256, seed=0, border_mode=0, pad_rows=16, pitch_extra=64,
                 kernels="gauss", zero_extra=False, jitter=0.5, scene=None, mask=None,
                 task_bits=synth.ALL_TASK_BITS, debug_marks=0, peak=1.0):
        self.seed = seed
        rng = np.random.default_rng(seed)
        self.geom = synth.geometry(width, height, border_mode=border_mode, image_rows=height + pad_rows,
                                   debug_marks=debug_marks)
        self.W, self.H = width, height
        self.TX, self.TY, self.TYA = synth.tiles(self.geom)
        self.dstride = width + pitch_extra
        self.rows = height + pad_rows
        disp = None
        if scene == "plane":
            imgs, disp = synth.plane_scene(rng, width, height, disparity=(0.0, 16.0), peak=peak)
        else:
            imgs = synth.smooth_bayer(rng, width, height)
        self.images = imgs
        pitched = rng.uniform(0.0, 1.0, size=(4, self.rows, self.dstride)).astype(np.float32)
        pitched[:, :height, :width] = imgs
        self.pitched = pitched
        self.kernels, self.extra = synth.kernel_tables(rng, self.geom, kind=kernels, pool=64,
                                                       zero_extra=zero_extra)
        self.tasks = synth.tasks_grid(self.geom, rng, jitter=jitter, task_bits=task_bits, disparity=disp,
                                      mask=mask)
        self.corr_idx = synth.corr_indices_fast(self.tasks, self.geom)
        self.tex_idx = synth.texture_indices(self.tasks, self.geom)
        self.port_offsets = synth.PORT_OFFSETS.copy()

    @property
    def num_tiles(self):
        return int(self.tasks.size)


def blob_mask(rng, tx, ty, fraction):
    """Seeded blob-shaped activity mask covering about `fraction` of the tiles."""
    m = np.zeros((ty, tx), dtype=bool)
    target = int(round(fraction * tx * ty))
    yy, xx = np.mgrid[0:ty, 0:tx]
    while m.sum() < target:
        cy, cx = rng.integers(0, ty), rng.integers(0, tx)
        r = rng.uniform(1.5, max(2.0, min(tx, ty) / 4))
        m |= (yy - cy) ** 2 + (xx - cx) ** 2 <= r * r
    return m
