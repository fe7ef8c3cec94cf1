"""Run a Case through the B200 library (C ABI) or the rebuilt reference
kernels, on cuda:0.  GPU tests only."""
import numpy as np
import torch

import refgpu
from tile_processor_gpu_b200 import api

DEV = "cuda:0"


class Frame:
    """Device copies of a Case's inputs plus zeroed outputs."""

    def __init__(self, case, device=DEV):
        self.case = case
        self.g = api.Geometry.from_dict(case.geom)
        self.images = [torch.from_numpy(case.pitched[c]).to(device) for c in range(4)]
        self.kernels = [torch.from_numpy(case.kernels[c]).to(device) for c in range(4)]
        self.extra = [torch.from_numpy(case.extra[c]).to(device) for c in range(4)]
        self.tasks = api.tasks_to_device(case.tasks, device)
        n = case.TX * case.TY * 3 * 256
        self.clt = [torch.zeros(n, dtype=torch.float32, device=device) for _ in range(4)]
        self.p_images = api.PointerArray(self.images)
        self.p_kernels = api.PointerArray(self.kernels)
        self.p_extra = api.PointerArray(self.extra)
        self.p_clt = api.PointerArray(self.clt)
        self.port_offsets = torch.from_numpy(case.port_offsets.reshape(-1)).to(device)

    def tile_scratch(self):
        """per-camera tile buffers of the CLT's size (the tensor-core texture path)"""
        if not hasattr(self, "_tiles"):
            self._tiles = [torch.zeros_like(c) for c in self.clt]
            self.p_tiles = api.PointerArray(self._tiles)
        return self.p_tiles

    def clt_numpy(self):
        return [c.cpu().numpy() for c in self.clt]

    def set_clt(self, clt):
        for c in range(4):
            self.clt[c].copy_(torch.from_numpy(np.asarray(clt[c], dtype=np.float32)))


def _tc_fmt(impl):
    return api.TC_FP16X2 if impl == "tc_fp16" else api.TC_BF16X2


def convert(fr, lpf_mask=0, impl="b200", num_tiles=None):
    c = fr.case
    n = c.num_tiles if num_tiles is None else num_tiles
    for t in fr.clt:
        t.zero_()
    if impl == "b200":
        api.convert_correct_tiles(fr.g, fr.p_extra, fr.p_kernels, fr.p_images, fr.tasks, fr.p_clt, c.dstride, n,
                                  lpf_mask)
    elif impl == "tma":
        api.convert_correct_tiles_tma(fr.g, fr.p_extra, fr.p_kernels, fr.p_images, fr.tasks, fr.p_clt, c.dstride,
                                      n, lpf_mask)
    elif impl.startswith("tc_"):
        api.convert_correct_tiles_tc(fr.g, fr.p_extra, fr.p_kernels, fr.p_images, fr.tasks, fr.p_clt, c.dstride, n,
                                     lpf_mask, fmt=_tc_fmt(impl))
    else:
        refgpu.call(c.geom, "ref_convert_correct_tiles", fr.p_extra.dev.data_ptr(), fr.p_kernels.dev.data_ptr(),
                    fr.p_images.dev.data_ptr(), fr.tasks.data_ptr(), fr.p_clt.dev.data_ptr(), c.dstride, n, lpf_mask)
    torch.cuda.synchronize()
    return fr.clt_numpy()


def correlate(fr, idx, colors=3, scales=(0.25, 0.25, 0.5), fat_zero=0.05, radius=7, stride=None, impl="b200"):
    c = fr.case
    stride = stride or (2 * radius + 1) ** 2 + 3
    idx_d = torch.from_numpy(np.ascontiguousarray(idx, dtype=np.int32)).to(DEV)
    out = torch.full((max(len(idx), 1), stride), -7.0, dtype=torch.float32, device=DEV)
    if impl == "b200":
        api.correlate2D(fr.g, fr.p_clt, colors, *scales, fat_zero, len(idx), idx_d, stride, radius, out)
    elif impl in ("tc_fp16", "tc_bf16"):
        api.correlate2D_tc(fr.g, fr.p_clt, colors, *scales, fat_zero, len(idx), idx_d, stride, radius, out,
                           fmt=api.TC_FP16X2 if impl == "tc_fp16" else api.TC_BF16X2)
    else:
        refgpu.call(c.geom, "ref_correlate2D", fr.p_clt.dev.data_ptr(), colors, *scales, fat_zero, len(idx),
                    idx_d.data_ptr(), stride, radius, out.data_ptr())
    torch.cuda.synchronize()
    return out.cpu().numpy()[: len(idx)]


TEX = dict(colors=3, is_lwir=0, min_shot=10.0, scale_shot=3.0, diff_sigma=1.5, diff_threshold=10.0, min_agree=3.0,
           weight0=0.294118, weight1=0.117647, weight2=0.588235, dust_remove=1)


def textures_tiles(fr, idx, keep_weights=0, impl="b200", **kw):
    p = dict(TEX, **kw)
    ns = (12 if keep_weights else 4) if p["colors"] == 3 else (8 if keep_weights else 2)
    stride = ns * 256 + 32
    idx_d = torch.from_numpy(np.ascontiguousarray(idx, dtype=np.int32)).to(DEV)
    out = torch.full((max(len(idx), 1), stride), -7.0, dtype=torch.float32, device=DEV)
    args = (p["colors"], p["is_lwir"], p["min_shot"], p["scale_shot"], p["diff_sigma"], p["diff_threshold"],
            p["min_agree"], p["weight0"], p["weight1"], p["weight2"], p["dust_remove"], keep_weights)
    if impl == "b200":
        api.textures_accumulate(fr.g, None, fr.p_clt, len(idx), idx_d, fr.port_offsets, *args, 0, None, stride, out)
    elif impl.startswith("tc_"):
        api.textures_accumulate_tc(fr.g, None, fr.p_clt, len(idx), idx_d, fr.port_offsets, *args, 0, None, stride,
                                   out, fr.tile_scratch(), fmt=_tc_fmt(impl))
    else:
        refgpu.call(fr.case.geom, "ref_textures_accumulate", None, fr.p_clt.dev.data_ptr(), len(idx),
                    idx_d.data_ptr(), fr.port_offsets.data_ptr(), *args, 0, None, stride, out.data_ptr())
    torch.cuda.synchronize()
    return out.cpu().numpy()[: len(idx), : ns * 256].reshape(len(idx), ns, 16, 16)


def imclt_all(fr, cam=0, impl="b200"):
    c = fr.case
    dst = c.W + 8 + 24
    rbg = torch.zeros(3 * (c.H + 8) * dst, dtype=torch.float32, device=DEV)
    if impl == "b200":
        api.imclt_rbg_all(fr.g, fr.clt[cam], rbg, dst)
    else:
        for color in range(3):
            for v in range(2):
                for h in range(2):
                    refgpu.call(c.geom, "ref_imclt_rbg", fr.clt[cam].data_ptr(), rbg.data_ptr(), color, v, h, dst)
    torch.cuda.synchronize()
    return rbg.cpu().numpy().reshape(3 * (c.H + 8), dst), dst


def texture_list(fr, impl="b200", width=None, height=None):
    c = fr.case
    tasks = api.tasks_to_device(c.tasks, DEV)
    idx = torch.zeros(c.TX * c.TYA + 256, dtype=torch.int32, device=DEV)  # the reference clears one past the end
    counts = torch.zeros(8, dtype=torch.int32, device=DEV)
    woi = torch.zeros(4, dtype=torch.int32, device=DEV)
    w = c.TX if width is None else width
    h = c.TY if height is None else height
    if impl == "b200":
        api.prepare_texture_list(fr.g, tasks, c.num_tiles, idx, counts, woi, w, h)
    else:
        refgpu.call(c.geom, "ref_prepare_texture_list", tasks.data_ptr(), c.num_tiles, idx.data_ptr(),
                    counts.data_ptr(), woi.data_ptr(), w, h)
    torch.cuda.synchronize()
    return api.tasks_from_device(tasks), idx.cpu().numpy(), counts.cpu().numpy(), woi.cpu().numpy()


def rgba(fr, impl="b200", **kw):
    c = fr.case
    p = dict(TEX, **kw)
    stride = (c.TX + 1) * 8 + 40
    rows = (c.TY + 1) * 8 * (p["colors"] + 1)
    out = torch.full((rows + 8, stride), 3.0, dtype=torch.float32, device=DEV)
    tasks = api.tasks_to_device(c.tasks, DEV)
    idx = torch.zeros(c.TX * c.TYA + 256, dtype=torch.int32, device=DEV)  # the reference clears one past the end
    counts = torch.zeros(8, dtype=torch.int32, device=DEV)
    woi = torch.zeros(4, dtype=torch.int32, device=DEV)
    args = (p["colors"], p["is_lwir"], p["min_shot"], p["scale_shot"], p["diff_sigma"], p["diff_threshold"],
            p["min_agree"], p["weight0"], p["weight1"], p["weight2"], p["dust_remove"], 0)
    if impl == "b200":
        api.generate_RBGA(fr.g, tasks, c.num_tiles, idx, counts, woi, c.TX, c.TY, fr.p_clt, fr.port_offsets,
                          *args, stride, out)
    elif impl.startswith("tc_"):
        api.generate_RBGA_tc(fr.g, tasks, c.num_tiles, idx, counts, woi, c.TX, c.TY, fr.p_clt, fr.port_offsets,
                             *args, stride, out, fr.tile_scratch(), fmt=_tc_fmt(impl))
    else:
        refgpu.call(c.geom, "ref_generate_RBGA", tasks.data_ptr(), c.num_tiles, idx.data_ptr(), counts.data_ptr(),
                    woi.data_ptr(), c.TX, c.TY, fr.p_clt.dev.data_ptr(), fr.port_offsets.data_ptr(), *args, stride,
                    out.data_ptr())
    torch.cuda.synchronize()
    return out.cpu().numpy(), woi.cpu().numpy(), stride, rows
