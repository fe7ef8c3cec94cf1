"""ctypes wrapper of the FP64 CPU oracle (oracle/libtp_oracle.so).

TEST INFRASTRUCTURE ONLY: the checker the CUDA path is compared against.  Only
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use it.
Arrays are numpy; outputs are float64.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "libtp_oracle.so")
TASK_DTYPE = np.dtype([("task", "<i4"), ("txy", "<i4"), ("xy", "<f4", (4, 2))])


class Geom(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("img_width", "img_height", "kernels_hor", "kernels_vert",
                                            "kernels_lstep", "image_rows", "border_mode", "debug_marks")]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE, "all"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = ctypes.CDLL(LIB)
    return _lib


def _g(geom):
    return Geom(*(int(geom.get(k, 0) if k != "image_rows" else geom.get(k) or geom["img_height"])
                  for k, _ in Geom._fields_))


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _parr(arrs):
    ptrs = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    return ptrs


def set_table_mode(mode):
    lib().tpo_set_table_mode(int(mode))


def set_threads(n):
    lib().tpo_set_threads(int(n))


def get_threads():
    return lib().tpo_get_threads()


def default_lpf(which):
    out = np.zeros(64, dtype=np.float32)
    lib().tpo_default_lpf(int(which), _p(out))
    return out


def alpha_fade():
    out = np.zeros((16, 256), dtype=np.float64)
    lib().tpo_alpha_fade(_p(out))
    return out


def dtt_matrix(kind):
    out = np.zeros(64, dtype=np.float64)
    lib().tpo_dtt_matrix(int(kind), _p(out))
    return out.reshape(8, 8)


def convert_correct_tiles(geom, kernel_offsets, kernels, images, dstride, tasks, lpf_mask=0, lpf=None,
                          want_corners=False):
    """images: [cams][rows][dstride] float32.  Returns clt [4][TY*TX*3*256]
    float64 (and int corners [n][4][3][4] = ktile_x, ktile_y, itlx, itly)."""
    TX, TY = geom["img_width"] // 8, geom["img_height"] // 8
    ko = [np.ascontiguousarray(k, dtype=np.float32) for k in kernel_offsets]
    kr = [np.ascontiguousarray(k, dtype=np.float32) for k in kernels]
    im = [np.ascontiguousarray(i, dtype=np.float32) for i in images]
    t = np.ascontiguousarray(tasks, dtype=TASK_DTYPE)
    clt = [np.zeros(TY * TX * 3 * 256, dtype=np.float64) for _ in range(4)]
    corners = np.zeros((max(t.size, 1), 4, 3, 4), dtype=np.int32) if want_corners else None
    lp = None if lpf is None else np.ascontiguousarray(lpf, dtype=np.float32).reshape(4 * 64)
    g = _g(geom)
    lib().tpo_convert_correct_tiles(ctypes.byref(g), _parr(ko), _parr(kr), _parr(im), ctypes.c_size_t(dstride),
                                    _p(t), ctypes.c_int(t.size), ctypes.c_int(lpf_mask), _p(lp), _parr(clt),
                                    _p(corners))
    if want_corners:
        return clt, corners[: t.size]
    return clt


def correlate2D(geom, clt, colors, scale0, scale1, scale2, fat_zero, corr_indices, corr_stride, corr_radius,
                lpf_rb_corr=None, lpf_corr=None):
    c = [np.ascontiguousarray(x, dtype=np.float64) for x in clt]
    idx = np.ascontiguousarray(corr_indices, dtype=np.int32)
    out = np.zeros((max(idx.size, 1), corr_stride), dtype=np.float64)
    f = ctypes.c_double
    lib().tpo_correlate2D(ctypes.byref(_g(geom)), _parr(c), ctypes.c_int(colors), f(scale0), f(scale1), f(scale2),
                          f(fat_zero), ctypes.c_int(idx.size), _p(idx), ctypes.c_size_t(corr_stride),
                          ctypes.c_int(corr_radius), _p(lpf_rb_corr), _p(lpf_corr), _p(out))
    return out[: idx.size]


def textures_accumulate(geom, woi, clt, texture_indices, port_offsets, colors=3, is_lwir=0, min_shot=10.0,
                        scale_shot=3.0, diff_sigma=1.5, diff_threshold=10.0, min_agree=3.0, weight0=0.294118,
                        weight1=0.117647, weight2=0.588235, dust_remove=1, keep_weights=0,
                        texture_rbg_stride=0, texture_rbg=None, texture_stride=0, texture_tiles=None, lpf=None,
                        want_margin=False):
    c = [np.ascontiguousarray(x, dtype=np.float64) for x in clt]
    idx = np.ascontiguousarray(texture_indices, dtype=np.int32)
    po = np.ascontiguousarray(port_offsets, dtype=np.float32).reshape(8)
    w = None if woi is None else np.ascontiguousarray(woi, dtype=np.int32)
    margin = np.ones((max(idx.size, 1), 256), dtype=np.float64) if want_margin else None
    lp = None if lpf is None else np.ascontiguousarray(lpf, dtype=np.float32).reshape(4 * 64)
    f = ctypes.c_double
    lib().tpo_textures_accumulate(ctypes.byref(_g(geom)), _p(w), _parr(c), ctypes.c_int(idx.size), _p(idx), _p(po),
                                  ctypes.c_int(colors), ctypes.c_int(is_lwir), f(min_shot), f(scale_shot),
                                  f(diff_sigma), f(diff_threshold), f(min_agree), f(weight0), f(weight1), f(weight2),
                                  ctypes.c_int(dust_remove), ctypes.c_int(keep_weights),
                                  ctypes.c_size_t(texture_rbg_stride), _p(texture_rbg),
                                  ctypes.c_size_t(texture_stride), _p(texture_tiles), _p(lp), _p(margin))
    return margin[: idx.size] if want_margin else None


def imclt_rbg(geom, clt_one_cam, rbg, color, v_offset, h_offset, dstride):
    c = np.ascontiguousarray(clt_one_cam, dtype=np.float64)
    assert rbg.dtype == np.float64 and rbg.flags.c_contiguous
    lib().tpo_imclt_rbg(ctypes.byref(_g(geom)), _p(c), _p(rbg), ctypes.c_int(color), ctypes.c_int(v_offset),
                        ctypes.c_int(h_offset), ctypes.c_size_t(dstride))


def imclt_rbg_all(geom, clt_one_cam, rbg, dstride):
    for color in range(3):
        for v in range(2):
            for h in range(2):
                imclt_rbg(geom, clt_one_cam, rbg, color, v, h, dstride)


def prepare_texture_list(geom, tasks, width, height, texture_indices=None):
    TX, TY = geom["img_width"] // 8, geom["img_height"] // 8
    TYA = (TY + 3) & ~3
    t = np.array(tasks, dtype=TASK_DTYPE, copy=True)
    idx = np.zeros(TX * TYA, dtype=np.int32) if texture_indices is None else np.array(texture_indices, dtype=np.int32)
    counts = np.zeros(8, dtype=np.int32)
    woi = np.zeros(4, dtype=np.int32)
    lib().tpo_prepare_texture_list(ctypes.byref(_g(geom)), _p(t), ctypes.c_int(t.size), _p(idx), _p(counts), _p(woi),
                                   ctypes.c_int(width), ctypes.c_int(height))
    return t, idx, counts, woi


def generate_RBGA(geom, tasks, width, height, clt, port_offsets, texture_rbga_stride, rows, colors=3, is_lwir=0,
                  min_shot=10.0, scale_shot=3.0, diff_sigma=1.5, diff_threshold=10.0, min_agree=3.0,
                  weight0=0.294118, weight1=0.117647, weight2=0.588235, dust_remove=1, lpf=None, out=None):
    TX, TY = geom["img_width"] // 8, geom["img_height"] // 8
    TYA = (TY + 3) & ~3
    t = np.array(tasks, dtype=TASK_DTYPE, copy=True)
    idx = np.zeros(TX * TYA, dtype=np.int32)
    counts = np.zeros(8, dtype=np.int32)
    woi = np.zeros(4, dtype=np.int32)
    c = [np.ascontiguousarray(x, dtype=np.float64) for x in clt]
    po = np.ascontiguousarray(port_offsets, dtype=np.float32).reshape(8)
    if out is None:
        out = np.zeros((rows, texture_rbga_stride), dtype=np.float64)
    lp = None if lpf is None else np.ascontiguousarray(lpf, dtype=np.float32).reshape(4 * 64)
    f = ctypes.c_double
    lib().tpo_generate_RBGA(ctypes.byref(_g(geom)), _p(t), ctypes.c_int(t.size), _p(idx), _p(counts), _p(woi),
                            ctypes.c_int(width), ctypes.c_int(height), _parr(c), _p(po), ctypes.c_int(colors),
                            ctypes.c_int(is_lwir), f(min_shot), f(scale_shot), f(diff_sigma), f(diff_threshold),
                            f(min_agree), f(weight0), f(weight1), f(weight2), ctypes.c_int(dust_remove),
                            ctypes.c_int(0), ctypes.c_size_t(texture_rbga_stride), _p(out), ctypes.c_size_t(rows),
                            _p(lp))
    return out, t, idx, counts, woi


def disparity_fit(geom, corrs, corr_indices, corr_radius=7, port_offsets=None, pair_mask=0x3F, mode=0):
    """Residual disparity and strength per tile (NaN where not fitted)."""
    TX, TY = geom["img_width"] // 8, geom["img_height"] // 8
    c = np.ascontiguousarray(corrs, dtype=np.float32)
    idx = np.ascontiguousarray(corr_indices, dtype=np.int32)
    if port_offsets is None:
        port_offsets = np.array([[-0.5, -0.5], [0.5, -0.5], [-0.5, 0.5], [0.5, 0.5]], dtype=np.float32)
    po = np.ascontiguousarray(port_offsets, dtype=np.float32).reshape(8)
    disp = np.full(TX * TY, np.nan)
    strength = np.full(TX * TY, np.nan)
    lib().tpo_disparity_fit(ctypes.byref(_g(geom)), _p(c), ctypes.c_size_t(c.shape[1]), ctypes.c_int(corr_radius),
                            ctypes.c_int(idx.size), _p(idx), _p(po), ctypes.c_int(pair_mask), ctypes.c_int(mode),
                            _p(disp), _p(strength))
    return disp, strength


def fit_profile(S, valid=None, mode=0):
    S = np.ascontiguousarray(S, dtype=np.float64)
    v = np.ones(S.size, dtype=np.int32) if valid is None else np.ascontiguousarray(valid, dtype=np.int32)
    rho = ctypes.c_double()
    pk = ctypes.c_double()
    lib().tpo_fit_profile(_p(S), _p(v), ctypes.c_int((S.size - 1) // 2), ctypes.c_int(mode), ctypes.byref(rho),
                          ctypes.byref(pk))
    return rho.value, pk.value


def psf_to_clt(h):
    """CLT kernel quadrants [..., 4, 8, 8] of spatial kernels h[..., 15, 15]
    (taps -7..7, rows vertical), FP64, as a direct sum over the taps:
    K_q[u][v] = sum_mn h[m][n] A(u, m) B(v, n), A = cos (CC, SC) or sin (CS,
    SS) of pi m (2u+1)/16, B = cos (CC, CS) or sin (SC, SS) of pi n (2v+1)/16."""
    h = np.asarray(h, dtype=np.float64)
    taps = np.arange(-7, 8)
    k = np.arange(8)
    ang = np.pi * (2 * k[:, None] + 1) * taps[None, :] / 16.0   # [8][15]
    c, s = np.cos(ang), np.sin(ang)
    out = np.zeros(h.shape[:-2] + (4, 8, 8))
    for q, (A, B) in enumerate(((c, c), (c, s), (s, c), (s, s))):
        for u in range(8):
            for v in range(8):
                out[..., q, u, v] = np.sum(h * A[u][:, None] * B[v][None, :], axis=(-2, -1))
    return out


# ---- the learned disparity residual (FP64 restatement of the tp_mlp_* math) --
def mlp_gelu(x):
    from scipy.special import erf
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def mlp_gelu_grad(x):
    from scipy.special import erf
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def mlp_forward(p, x):
    """x [n][1350] -> (out [n][2], cache)"""
    P = {k: np.asarray(v, np.float64) for k, v in p.items()}
    z1 = x @ P["W1"] + P["b1"]
    h1 = mlp_gelu(z1)
    z2 = h1 @ P["W2"] + P["b2"]
    h2 = mlp_gelu(z2)
    out = h2 @ P["W3"] + P["b3"]
    return out, (x, z1, h1, z2, h2)


def mlp_loss_and_grads(p, x, target, w=None):
    """mean over rows with weight 1 of 0.5 exp(-s) (d - target)^2 + 0.5 s
    (s clamped to [-12, 12]) and its gradients w.r.t. every parameter"""
    P = {k: np.asarray(v, np.float64) for k, v in p.items()}
    x = np.asarray(x, np.float64)
    out, (_, z1, h1, z2, h2) = mlp_forward(P, x)
    w = np.ones(len(x)) if w is None else np.asarray(w, np.float64)
    cnt = max(w.sum(), 1.0)
    d, s_raw = out[:, 0], out[:, 1]
    s = np.clip(s_raw, -12.0, 12.0)
    e = d - target
    iv = np.exp(-s)
    loss = (w * (0.5 * iv * e * e + 0.5 * s)).sum() / cnt
    dout = np.zeros_like(out)
    dout[:, 0] = w * iv * e / cnt
    dout[:, 1] = np.where((s_raw > -12.0) & (s_raw < 12.0), w * (0.5 - 0.5 * iv * e * e) / cnt, 0.0)
    g = {"W3": h2.T @ dout, "b3": dout.sum(0)}
    dz2 = (dout @ P["W3"].T) * mlp_gelu_grad(z2)
    g["W2"], g["b2"] = h1.T @ dz2, dz2.sum(0)
    dz1 = (dz2 @ P["W2"].T) * mlp_gelu_grad(z1)
    g["W1"], g["b1"] = x.T @ dz1, dz1.sum(0)
    return loss, g
