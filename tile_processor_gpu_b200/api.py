"""Host-side mirror of the reference's kernel interface, over the C ABI.

Each function has the name and the argument order of one `extern "C"`
kernel of mfkiwl/tile_processor_gpu (src/TileProcessor.cuh) and launches the
B200 implementation through libtp_b200.so.  Buffers are torch CUDA tensors
(device memory and streams are torch's; the compute is the library's).  Where
the reference takes `float **` (one device array per camera) these functions
take a list of tensors, or a prebuilt `PointerArray`.

Errors: a negative status from the library raises `TpError` with the
library's message.  There is no CPU fallback.
"""
import ctypes

import numpy as np
import torch

from . import _native
from ._native import TpGeometry, TpError  # noqa: F401
from .synth import TASK_DTYPE


class Geometry:
    """Runtime geometry (replaces IMG_WIDTH / IMG_HEIGHT / KERNELS_* defines)."""

    def __init__(self, img_width, img_height, kernels_hor=None, kernels_vert=None, kernels_lstep=4,
                 image_rows=None, border_mode=0, debug_marks=0):
        step = 1 << kernels_lstep
        self.c = TpGeometry(int(img_width), int(img_height),
                            int(kernels_hor if kernels_hor is not None else img_width // step + 2),
                            int(kernels_vert if kernels_vert is not None else img_height // step + 2),
                            int(kernels_lstep), int(image_rows if image_rows is not None else img_height),
                            int(border_mode), int(debug_marks))

    @classmethod
    def from_dict(cls, d):
        return cls(d["img_width"], d["img_height"], d["kernels_hor"], d["kernels_vert"], d["kernels_lstep"],
                   d.get("image_rows"), d.get("border_mode", 0), d.get("debug_marks", 0))

    @property
    def ptr(self):
        return ctypes.byref(self.c)

    width = property(lambda self: self.c.img_width)
    height = property(lambda self: self.c.img_height)
    tiles_x = property(lambda self: self.c.img_width // 8)
    tiles_y = property(lambda self: self.c.img_height // 8)
    tiles_ya = property(lambda self: (self.c.img_height // 8 + 3) & ~3)
    num_tiles = property(lambda self: self.tiles_x * self.tiles_y)
    kernels_hor = property(lambda self: self.c.kernels_hor)
    kernels_vert = property(lambda self: self.c.kernels_vert)


class PointerArray:
    """Device array of device pointers (the reference's `float **`)."""

    def __init__(self, tensors, device=None):
        self.tensors = list(tensors)
        dev = device or self.tensors[0].device
        ptrs = torch.tensor([t.data_ptr() for t in self.tensors], dtype=torch.int64)
        self.dev = ptrs.to(dev)

    @property
    def ptr(self):
        return ctypes.c_void_p(self.dev.data_ptr())


def _parr(x):
    if isinstance(x, PointerArray):
        return x.ptr
    if isinstance(x, (list, tuple)):
        return PointerArray(x).ptr
    raise TypeError("expected a list of tensors or a PointerArray")


def _dptr(t):
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def _stream(stream):
    """torch stream (None = torch's current stream), or a raw cudaStream_t int"""
    if isinstance(stream, int):
        return ctypes.c_void_p(stream)
    if stream is None:
        if not torch.cuda.is_available():
            return ctypes.c_void_p(0)
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


def tasks_to_device(tasks, device="cuda"):
    """numpy TASK_DTYPE array -> int32 [n, 10] device tensor (struct tp_task)."""
    a = np.ascontiguousarray(tasks, dtype=TASK_DTYPE)
    return torch.from_numpy(a.view(np.int32).reshape(-1, 10).copy()).to(device)


def tasks_from_device(t):
    return t.cpu().numpy().reshape(-1).view(TASK_DTYPE).copy()


def convert_correct_tiles(geom, gpu_kernel_offsets, gpu_kernels, gpu_images, gpu_tasks, gpu_clt, dstride,
                          num_tiles, lpf_mask=0, stream=None):
    """Forward CLT with aberration correction (convert_correct_tiles)."""
    _native.call("tp_convert_correct_tiles", geom.ptr, _parr(gpu_kernel_offsets), _parr(gpu_kernels),
                 _parr(gpu_images), _dptr(gpu_tasks), _parr(gpu_clt), int(dstride), int(num_tiles),
                 int(lpf_mask), _stream(stream))


def convert_correct_tiles_tma(geom, gpu_kernel_offsets, gpu_kernels, gpu_images, gpu_tasks, gpu_clt, dstride,
                              num_tiles, lpf_mask=0, stream=None):
    """convert_correct_tiles with the Bayer windows staged in shared memory by
    the TMA unit (tp_convert_correct_tiles_tma; the same CLT)."""
    _native.call("tp_convert_correct_tiles_tma", geom.ptr, _parr(gpu_kernel_offsets), _parr(gpu_kernels),
                 _parr(gpu_images), _dptr(gpu_tasks), _parr(gpu_clt), int(dstride), int(num_tiles),
                 int(lpf_mask), _stream(stream))


def correlate2D(geom, gpu_clt, colors, scale0, scale1, scale2, fat_zero, num_corr_tiles, gpu_corr_indices,
                corr_stride, corr_radius, gpu_corrs, stream=None):
    """Pairwise 2-D phase correlation (correlate2D)."""
    _native.call("tp_correlate2D", geom.ptr, _parr(gpu_clt), int(colors), float(scale0), float(scale1),
                 float(scale2), float(fat_zero), int(num_corr_tiles), _dptr(gpu_corr_indices), int(corr_stride),
                 int(corr_radius), _dptr(gpu_corrs), _stream(stream))


TC_FP16X2, TC_BF16X2 = 0, 1


def correlate2D_tc(geom, gpu_clt, colors, scale0, scale1, scale2, fat_zero, num_corr_tiles, gpu_corr_indices,
                   corr_stride, corr_radius, gpu_corrs, fmt=TC_FP16X2, stream=None):
    """correlate2D with the pixel-domain transforms on the tensor cores
    (split 16-bit operands: fmt TC_FP16X2 or TC_BF16X2)."""
    _native.call("tp_correlate2D_tc", geom.ptr, _parr(gpu_clt), int(colors), float(scale0), float(scale1),
                 float(scale2), float(fat_zero), int(num_corr_tiles), _dptr(gpu_corr_indices), int(corr_stride),
                 int(corr_radius), _dptr(gpu_corrs), int(fmt), _stream(stream))


def convert_correct_tiles_tc(geom, gpu_kernel_offsets, gpu_kernels, gpu_images, gpu_tasks, gpu_clt, dstride,
                             num_tiles, lpf_mask=0, fmt=TC_FP16X2, stream=None):
    """convert_correct_tiles with the 2-D DCT-IV / DST-IV on the tensor cores."""
    _native.call("tp_convert_correct_tiles_tc", geom.ptr, _parr(gpu_kernel_offsets), _parr(gpu_kernels),
                 _parr(gpu_images), _dptr(gpu_tasks), _parr(gpu_clt), int(dstride), int(num_tiles),
                 int(lpf_mask), int(fmt), _stream(stream))


def textures_accumulate_tc(geom, woi, gpu_clt, num_texture_tiles, gpu_texture_indices, gpu_port_offsets, colors,
                           is_lwir, min_shot, scale_shot, diff_sigma, diff_threshold, min_agree, weight0, weight1,
                           weight2, dust_remove, keep_weights, texture_rbg_stride, gpu_texture_rbg, texture_stride,
                           gpu_texture_tiles, gpu_tile_scratch, fmt=TC_FP16X2, stream=None):
    """textures_accumulate with the inverse CLT on the tensor cores (into gpu_tile_scratch)."""
    _native.call("tp_textures_accumulate_tc", geom.ptr, _dptr(woi), _parr(gpu_clt), int(num_texture_tiles),
                 _dptr(gpu_texture_indices), _dptr(gpu_port_offsets), int(colors), int(is_lwir), float(min_shot),
                 float(scale_shot), float(diff_sigma), float(diff_threshold), float(min_agree), float(weight0),
                 float(weight1), float(weight2), int(dust_remove), int(keep_weights), int(texture_rbg_stride),
                 _dptr(gpu_texture_rbg), int(texture_stride), _dptr(gpu_texture_tiles), _parr(gpu_tile_scratch),
                 int(fmt), _stream(stream))


def generate_RBGA_tc(geom, gpu_tasks, num_tiles, gpu_texture_indices, num_texture_tiles, woi, width, height,
                     gpu_clt, gpu_port_offsets, colors, is_lwir, min_shot, scale_shot, diff_sigma, diff_threshold,
                     min_agree, weight0, weight1, weight2, dust_remove, keep_weights, texture_rbga_stride,
                     gpu_texture_tiles, gpu_tile_scratch, fmt=TC_FP16X2, stream=None):
    """generate_RBGA with the inverse CLT on the tensor cores (into gpu_tile_scratch)."""
    _native.call("tp_generate_RBGA_tc", geom.ptr, _dptr(gpu_tasks), int(num_tiles), _dptr(gpu_texture_indices),
                 _dptr(num_texture_tiles), _dptr(woi), int(width), int(height), _parr(gpu_clt),
                 _dptr(gpu_port_offsets), int(colors), int(is_lwir), float(min_shot), float(scale_shot),
                 float(diff_sigma), float(diff_threshold), float(min_agree), float(weight0), float(weight1),
                 float(weight2), int(dust_remove), int(keep_weights), int(texture_rbga_stride),
                 _dptr(gpu_texture_tiles), _parr(gpu_tile_scratch), int(fmt), _stream(stream))


def tc_status(clear=True):
    """1 when a tensor-core stage kernel's bounded wait ran out since the last clear"""
    v = ctypes.c_int(0)
    _native.call("tp_tc_status", ctypes.byref(v), int(bool(clear)))
    return v.value


def tc_table_image(fmt, stage):
    """The 64 KB shared-memory image of the split transform matrices of a
    stage (0 correlation, 1 inverse CLT, 2 forward CLT) as uint16 [32768]
    (host-side, no device needed)."""
    out = np.zeros(32768, dtype=np.uint16)
    _native.call("tp_tc_table_image", int(fmt), int(stage), out.ctypes.data_as(ctypes.c_void_p))
    return out


def textures_accumulate(geom, woi, gpu_clt, num_texture_tiles, gpu_texture_indices, gpu_port_offsets, colors,
                        is_lwir, min_shot, scale_shot, diff_sigma, diff_threshold, min_agree, weight0, weight1,
                        weight2, dust_remove, keep_weights, texture_rbg_stride, gpu_texture_rbg, texture_stride,
                        gpu_texture_tiles, stream=None):
    """Texture tiles and/or overlapped RGBA accumulation (textures_accumulate)."""
    _native.call("tp_textures_accumulate", geom.ptr, _dptr(woi), _parr(gpu_clt), int(num_texture_tiles),
                 _dptr(gpu_texture_indices), _dptr(gpu_port_offsets), int(colors), int(is_lwir),
                 float(min_shot), float(scale_shot), float(diff_sigma), float(diff_threshold), float(min_agree),
                 float(weight0), float(weight1), float(weight2), int(dust_remove), int(keep_weights),
                 int(texture_rbg_stride), _dptr(gpu_texture_rbg), int(texture_stride), _dptr(gpu_texture_tiles),
                 _stream(stream))


def imclt_rbg(geom, gpu_clt, gpu_rbg, color, v_offset, h_offset, dstride, stream=None):
    """One parity pass of the overlap-add inverse CLT of one color (imclt_rbg)."""
    _native.call("tp_imclt_rbg", geom.ptr, _dptr(gpu_clt), _dptr(gpu_rbg), int(color), int(v_offset),
                 int(h_offset), int(dstride), _stream(stream))


def imclt_rbg_all(geom, gpu_clt, gpu_rbg, dstride, stream=None):
    """All 3 colors x 4 passes of one camera, in the reference driver's order."""
    _native.call("tp_imclt_rbg_all", geom.ptr, _dptr(gpu_clt), _dptr(gpu_rbg), int(dstride), _stream(stream))


def prepare_texture_list(geom, gpu_tasks, num_tiles, gpu_texture_indices, num_texture_tiles, woi, width, height,
                         stream=None):
    """Texture list, neighbour bits and window of interest (prepare_texture_list)."""
    _native.call("tp_prepare_texture_list", geom.ptr, _dptr(gpu_tasks), int(num_tiles),
                 _dptr(gpu_texture_indices), _dptr(num_texture_tiles), _dptr(woi), int(width), int(height),
                 _stream(stream))


def clear_texture_rbga(geom, texture_width, texture_slice_height, texture_rbga_stride, gpu_texture_tiles,
                       stream=None):
    _native.call("tp_clear_texture_rbga", geom.ptr, int(texture_width), int(texture_slice_height),
                 int(texture_rbga_stride), _dptr(gpu_texture_tiles), _stream(stream))


def generate_RBGA(geom, gpu_tasks, num_tiles, gpu_texture_indices, num_texture_tiles, woi, width, height,
                  gpu_clt, gpu_port_offsets, colors, is_lwir, min_shot, scale_shot, diff_sigma, diff_threshold,
                  min_agree, weight0, weight1, weight2, dust_remove, keep_weights, texture_rbga_stride,
                  gpu_texture_tiles, stream=None):
    """List + clear + one overlap-add pass per tile parity into the RGBA image (generate_RBGA)."""
    _native.call("tp_generate_RBGA", geom.ptr, _dptr(gpu_tasks), int(num_tiles), _dptr(gpu_texture_indices),
                 _dptr(num_texture_tiles), _dptr(woi), int(width), int(height), _parr(gpu_clt),
                 _dptr(gpu_port_offsets), int(colors), int(is_lwir), float(min_shot), float(scale_shot),
                 float(diff_sigma), float(diff_threshold), float(min_agree), float(weight0), float(weight1),
                 float(weight2), int(dust_remove), int(keep_weights), int(texture_rbga_stride),
                 _dptr(gpu_texture_tiles), _stream(stream))


def generate_RBGA_rows(geom, gpu_tasks, num_tiles, gpu_texture_indices, num_texture_tiles, woi, width, height,
                       gpu_clt, gpu_port_offsets, colors, min_shot, scale_shot, diff_sigma, weight0, weight1, weight2,
                       dust_remove, texture_rbga_stride, gpu_texture_tiles, row_first, row_last, stream=None):
    """generate_RBGA for the band of tile rows [row_first, row_last) of a frame
    split across GPUs: every task marks its tile, only the band's tiles are
    listed and accumulated (pass the band's tasks plus one tile row above and
    below; sharding.band_tasks)."""
    _native.call("tp_generate_RBGA_rows", geom.ptr, _dptr(gpu_tasks), int(num_tiles), _dptr(gpu_texture_indices),
                 _dptr(num_texture_tiles), _dptr(woi), int(width), int(height), _parr(gpu_clt),
                 _dptr(gpu_port_offsets), int(colors), float(min_shot), float(scale_shot), float(diff_sigma),
                 float(weight0), float(weight1), float(weight2), int(dust_remove), int(texture_rbga_stride),
                 _dptr(gpu_texture_tiles), int(row_first), int(row_last), _stream(stream))


def generate_RBGA_noalloc(geom, gpu_tasks, num_tiles, width, height, gpu_clt, gpu_port_offsets, colors, is_lwir,
                          min_shot, scale_shot, diff_sigma, diff_threshold, min_agree, weight0, weight1, weight2,
                          dust_remove, keep_weights, texture_rbga_stride, gpu_texture_tiles, stream=None):
    """generate_RBGA with the texture list in library-owned device scratch,
    for callers that cannot allocate device memory (no list buffers from the
    caller).  The first call on a device does the set-up; calls that overlap
    on the GPU race."""
    _native.call("tp_generate_RBGA_noalloc", geom.ptr, _dptr(gpu_tasks), int(num_tiles), int(width), int(height),
                 _parr(gpu_clt), _dptr(gpu_port_offsets), int(colors), int(is_lwir), float(min_shot),
                 float(scale_shot), float(diff_sigma), float(diff_threshold), float(min_agree), float(weight0),
                 float(weight1), float(weight2), int(dust_remove), int(keep_weights), int(texture_rbga_stride),
                 _dptr(gpu_texture_tiles), _stream(stream))


def process_frame(geom, gpu_kernel_offsets, gpu_kernels, gpu_images, dstride, gpu_tasks, num_tiles, gpu_corrs,
                  corr_stride, gpu_port_offsets, gpu_texture_indices, num_texture_tiles, woi, texture_rbga_stride,
                  gpu_texture_rbga, lpf_mask=0, corr_colors=3, scale0=0.25, scale1=0.25, scale2=0.5, fat_zero=30.0,
                  corr_radius=7, min_shot=10.0, scale_shot=3.0, diff_sigma=1.5, weight0=0.294118, weight1=0.117647,
                  weight2=0.588235, dust_remove=1, gpu_clt=None, stream=None):
    """One frame through the whole hot path (forward CLT, all pair
    correlations, overlapped RGBA texture) with the CLT kept on chip.
    gpu_corrs: [num_tiles][6][corr_stride]."""
    clt = _parr(gpu_clt) if gpu_clt is not None else ctypes.c_void_p(0)
    _native.call("tp_process_frame", geom.ptr, _parr(gpu_kernel_offsets), _parr(gpu_kernels), _parr(gpu_images),
                 int(dstride), _dptr(gpu_tasks), int(num_tiles), int(lpf_mask), int(corr_colors), float(scale0),
                 float(scale1), float(scale2), float(fat_zero), int(corr_radius), int(corr_stride), _dptr(gpu_corrs),
                 _dptr(gpu_port_offsets), float(min_shot), float(scale_shot), float(diff_sigma), float(weight0),
                 float(weight1), float(weight2), int(dust_remove), _dptr(gpu_texture_indices),
                 _dptr(num_texture_tiles), _dptr(woi), int(texture_rbga_stride), _dptr(gpu_texture_rbga), clt,
                 _stream(stream))


def disparity_fit(geom, gpu_corrs, corr_stride, corr_radius, num_corr_tiles, gpu_corr_indices, gpu_port_offsets,
                  gpu_disparity, gpu_strength, pair_mask=0x3F, mode=0, stream=None):
    """Residual disparity and strength per tile from the pair correlations
    (written into gpu_disparity / gpu_strength, float[tilesx * tilesy])."""
    _native.call("tp_disparity_fit", geom.ptr, _dptr(gpu_corrs), int(corr_stride), int(corr_radius),
                 int(num_corr_tiles), _dptr(gpu_corr_indices), _dptr(gpu_port_offsets), int(pair_mask), int(mode),
                 _dptr(gpu_disparity), _dptr(gpu_strength), _stream(stream))


def psf_to_clt(gpu_psf, gpu_clt_kernels, stream=None):
    """CLT kernel tables [n][4][8][8] from spatial kernels [n][15][15] (device)."""
    n = gpu_psf.numel() // 225
    _native.call("tp_psf_to_clt", _dptr(gpu_psf), int(n), _dptr(gpu_clt_kernels), _stream(stream))


def set_lpf(which, values):
    """Replace a low-pass table on the current device (0..3 lpf_data, 4 lpf_rb_corr, 5 lpf_corr)."""
    a = np.ascontiguousarray(values, dtype=np.float32).reshape(64)
    _native.call("tp_set_lpf", int(which), a.ctypes.data_as(ctypes.c_void_p))


def get_lpf(which):
    a = np.zeros(64, dtype=np.float32)
    _native.call("tp_get_lpf", int(which), a.ctypes.data_as(ctypes.c_void_p))
    return a


def reset_lpf():
    _native.call("tp_reset_lpf")


# texture defaults of the reference's harness (src/dtt8x8.cu:791-814)
TEXTURE_DEFAULTS = dict(colors=3, is_lwir=0, min_shot=10.0, scale_shot=3.0, diff_sigma=1.5, diff_threshold=10.0,
                        min_agree=3.0, weight0=0.294118, weight1=0.117647, weight2=0.588235, dust_remove=1)
# correlation defaults of the harness (src/dtt8x8.cu:719-730) with a 15x15 output
CORR_DEFAULTS = dict(colors=3, scale0=0.25, scale1=0.25, scale2=0.5, fat_zero=30.0, corr_radius=7)
