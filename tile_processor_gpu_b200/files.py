"""The reference harness's data files and host lists (src/dtt8x8.cu:144-165,
:228-264, :383-446), through the library's host helpers.

Every file is a raw native-endian float32 array without a header; the shapes
come from the frame geometry:

* ``*.kernel``          [kernels_vert][kernels_hor][3][4][8][8]  per camera
* ``*.kernel_offsets``  [kernels_vert][kernels_hor][3][8]        per camera (CltExtra)
* ``*.bayer``           [img_height][img_width]                  per camera
* ``*.portsxy``         [tilesy * tilesx][2]                     per camera (tile centres)
* ``*.clt``             [tilesy][tilesx][3][4][8][8]             per camera
* ``*.rbg``             [3][img_height + 8][img_width + 8]       per camera
* ``*.corr``            [num_corr][(2r+1)^2]
* ``*.rgba``            texture tiles [n][slices * 256], or the window [slices][h][w]
"""
import ctypes

import numpy as np

from . import _native
from .synth import TASK_DTYPE, ALL_TASK_BITS


def read_floats(path, count=None):
    """float32 array of `count` values (None: the whole file)."""
    if count is None:
        import os
        count = os.path.getsize(path) // 4
    out = np.empty(int(count), dtype=np.float32)
    got = _native.load().tp_read_floats(str(path).encode(), out.ctypes.data_as(ctypes.c_void_p), out.size)
    if got < 0:
        raise OSError("cannot read %s" % path)
    if got != out.size:
        raise OSError("%s: %d of %d floats" % (path, got, out.size))
    return out


def write_floats(path, array):
    a = np.ascontiguousarray(array, dtype=np.float32)
    put = _native.load().tp_write_floats(str(path).encode(), a.ctypes.data_as(ctypes.c_void_p), a.size)
    if put != a.size:
        raise OSError("cannot write %s" % path)


def kernel_floats(geom):
    return geom["kernels_vert"] * geom["kernels_hor"] * 3 * 256


def read_kernels(path, geom):
    return read_floats(path, kernel_floats(geom))


def read_kernel_offsets(path, geom):
    return read_floats(path, geom["kernels_vert"] * geom["kernels_hor"] * 3 * 8)


def read_bayer(path, geom):
    return read_floats(path, geom["img_width"] * geom["img_height"]).reshape(geom["img_height"], geom["img_width"])


def read_portsxy(path, geom):
    n = (geom["img_width"] // 8) * (geom["img_height"] // 8)
    return read_floats(path, 2 * n).reshape(n, 2)


def tasks_from_portsxy(portsxy, geom, task_bits=ALL_TASK_BITS):
    """The harness's linescan task list from the four cameras' tile centres."""
    tx, ty = geom["img_width"] // 8, geom["img_height"] // 8
    ports = [np.ascontiguousarray(p, dtype=np.float32).reshape(-1) for p in portsxy]
    ptrs = (ctypes.c_void_p * 4)(*[p.ctypes.data for p in ports])
    tasks = np.zeros(tx * ty, dtype=TASK_DTYPE)
    _native.call("tp_tasks_from_portsxy", ptrs, tx, ty, int(task_bits), tasks.ctypes.data_as(ctypes.c_void_p))
    return tasks


def corr_indices(tasks, geom):
    """(tile << 8) | pair for every pair bit of every task, in task order."""
    t = np.ascontiguousarray(tasks, dtype=TASK_DTYPE)
    tx = geom["img_width"] // 8
    n = _native.call("tp_corr_indices_from_tasks", t.ctypes.data_as(ctypes.c_void_p), t.size, tx, None)
    out = np.zeros(max(n, 1), dtype=np.int32)
    _native.call("tp_corr_indices_from_tasks", t.ctypes.data_as(ctypes.c_void_p), t.size, tx,
                 out.ctypes.data_as(ctypes.c_void_p))
    return out[:n]


def load_harness_set(paths, geom):
    """The harness's inputs for four cameras: `paths` maps 'kernel',
    'kernel_offsets', 'bayer', 'portsxy' to lists of four file names.
    Returns dict(kernels, kernel_offsets, images [4][H][W], tasks)."""
    return dict(kernels=[read_kernels(p, geom) for p in paths["kernel"]],
                kernel_offsets=[read_kernel_offsets(p, geom) for p in paths["kernel_offsets"]],
                images=np.stack([read_bayer(p, geom) for p in paths["bayer"]]),
                tasks=tasks_from_portsxy([read_portsxy(p, geom) for p in paths["portsxy"]], geom))
