"""Seeded synthetic inputs for the tile processor (host side, numpy).

There is no camera data here, so every input is generated: GR/BG Bayer
mosaics, CLT-domain aberration-kernel tables made from anisotropic Gaussian
PSFs, kernel-centre offset tables, per-tile task lists and the correlation /
texture index lists that the reference's harness builds
(src/dtt8x8.cu:418-470).  Layouts are the reference's:

* image      float32 [H][dstride]              (pitched, GR/BG, red at row 0 col 1)
* kernels    float32 [kv][kh][3][4][8][8]      per camera
* offsets    float32 [kv][kh][3][8]            per camera (struct CltExtra)
* tasks      TASK_DTYPE [n]                    (struct tp_task, 40 bytes)

Coordinates that feed the float32 integer-corner logic are kept on dyadic
grids (task centres in 1/256 px, offsets in 1/64 px, Jacobians in 1/4096) so
that every product in that logic is exact in float32 and the chosen integer
corners do not depend on how a compiler contracts multiply-adds.
"""
import math

import numpy as np

TASK_DTYPE = np.dtype([("task", "<i4"), ("txy", "<i4"), ("xy", "<f4", (4, 2))])
assert TASK_DTYPE.itemsize == 40

PORT_OFFSETS = np.array([[-0.5, -0.5], [0.5, -0.5], [-0.5, 0.5], [0.5, 0.5]], dtype=np.float32)
PAIRS = ((0, 1), (2, 3), (0, 2), (1, 3), (0, 3), (2, 1))
ALL_TASK_BITS = 0xF | (0x3F << 4)


def geometry(width, height, kernels_lstep=4, border_mode=0, image_rows=None, debug_marks=0):
    """Frame geometry (the reference's compile-time defines, as a dict)."""
    step = 1 << kernels_lstep
    return dict(img_width=int(width), img_height=int(height),
                kernels_hor=int(width // step + 2), kernels_vert=int(height // step + 2),
                kernels_lstep=int(kernels_lstep),
                image_rows=int(image_rows if image_rows is not None else height),
                border_mode=int(border_mode), debug_marks=int(debug_marks))


def tiles(geom):
    tx, ty = geom["img_width"] // 8, geom["img_height"] // 8
    return tx, ty, (ty + 3) & ~3


def _upsample(a, H, W):
    """bilinear resample of a coarse grid to H x W"""
    h, w = a.shape
    y = np.linspace(0, h - 1, H, dtype=np.float64)
    x = np.linspace(0, w - 1, W, dtype=np.float64)
    y0 = np.floor(y).astype(np.int64); y1 = np.minimum(y0 + 1, h - 1); fy = (y - y0)[:, None]
    x0 = np.floor(x).astype(np.int64); x1 = np.minimum(x0 + 1, w - 1); fx = (x - x0)[None, :]
    top = a[y0][:, x0] * (1 - fx) + a[y0][:, x1] * fx
    bot = a[y1][:, x0] * (1 - fx) + a[y1][:, x1] * fx
    return top * (1 - fy) + bot * fy


def smooth_noise(rng, H, W, scales=(64, 16, 4), weights=(1.0, 0.5, 0.25)):
    out = np.zeros((H, W), dtype=np.float64)
    for s, wgt in zip(scales, weights):
        coarse = rng.standard_normal((H // s + 2, W // s + 2))
        out += wgt * _upsample(coarse, H, W)
    out -= out.min()
    out /= max(out.max(), 1e-12)
    return out


def bayer_color_map(H, W):
    """0 = red (even row, odd col), 1 = blue (odd row, even col), 2 = green"""
    r = np.arange(H)[:, None] & 1
    c = np.arange(W)[None, :] & 1
    m = np.full((H, W), 2, dtype=np.int8)
    m[(r == 0) & (c == 1)] = 0
    m[(r == 1) & (c == 0)] = 1
    return m


def smooth_bayer(rng, width, height, cams=4):
    """cams x [H][W] float32 mosaics of seeded smooth noise in [0, 1]."""
    return np.stack([smooth_noise(rng, height, width).astype(np.float32) for _ in range(cams)])


# texture octaves of plane_scene: (scale px, weight); 'smooth' is dominated by
# 48-px structure, 'detail' adds strong 4-px and 2-px octaves (fine texture
# that correlation can lock onto under the shot noise)
TEXTURES = {"smooth": ((48, 12, 3), (1.0, 0.6, 0.35)), "detail": ((24, 8, 4, 2), (0.6, 0.8, 1.0, 1.0))}


def plane_scene(rng, width, height, disparity=(0.0, 64.0), port_offsets=PORT_OFFSETS, gain=0.01,
                read_sigma=0.002, peak=1.0, texture="smooth"):
    """Quad-camera Bayer frame of a random-texture slanted plane.

    The plane has disparity d(s) = d0 + gx sx + gy sy (s in scene
    coordinates) spanning `disparity`; camera k sees scene point s at pixel
    p = s + d(s) o_k, o_k = port_offsets[k] (so a tile centred at c in the
    scene is centred at c + d(c) o_k in camera k, exactly as tasks_grid
    places it).  Each camera pixel p is rendered from the scene point
    s = q - o_k (g . q) / (1 + g . o_k), q = p - d0 o_k, g = (gx, gy), the
    inverse of that map.  Poisson-Gaussian noise: v + sqrt(gain v) N +
    read_sigma N.  Returns (images [4][H][W], disparity function coefficients
    (d0, gx, gy)).
    """
    H, W = height, width
    scales, weights = TEXTURES[texture]
    tex = np.stack([smooth_noise(rng, H + 96, W + 96, scales=scales, weights=weights) for _ in range(3)])
    dlo, dhi = disparity
    gx = (dhi - dlo) * rng.uniform(0.3, 0.7) / W
    gy = (dhi - dlo - gx * W) / H
    d0 = dlo
    cmap = bayer_color_map(H, W)
    yy, xx = np.mgrid[0:H, 0:W].astype(np.float64)
    imgs = []
    for k in range(len(port_offsets)):
        ox, oy = float(port_offsets[k][0]), float(port_offsets[k][1])
        qx, qy = xx - d0 * ox, yy - d0 * oy
        gq = (gx * qx + gy * qy) / (1.0 + gx * ox + gy * oy)
        sx = qx - ox * gq + 48.0
        sy = qy - oy * gq + 48.0
        x0 = np.clip(np.floor(sx).astype(np.int64), 0, W + 94); fx = sx - x0
        y0 = np.clip(np.floor(sy).astype(np.int64), 0, H + 94); fy = sy - y0
        t = tex[cmap, y0, x0] * (1 - fx) * (1 - fy) + tex[cmap, y0, x0 + 1] * fx * (1 - fy) + \
            tex[cmap, y0 + 1, x0] * (1 - fx) * fy + tex[cmap, y0 + 1, x0 + 1] * fx * fy
        v = peak * t
        v = v + np.sqrt(np.maximum(gain * v, 0.0)) * rng.standard_normal(v.shape) + read_sigma * rng.standard_normal(v.shape)
        imgs.append(v.astype(np.float32))
    return np.stack(imgs), (d0, gx, gy)


class TwoPlaneDisparity:
    """d(x, y) of occlusion_scene: the foreground plane where n . (x, y) > c,
    else the background plane (a picklable callable)."""

    def __init__(self, back, front, edge):
        self.back, self.front, self.edge = tuple(back), tuple(front), tuple(edge)

    def __call__(self, x, y):
        x = np.asarray(x, np.float64); y = np.asarray(y, np.float64)
        (b0, bx, by), (f0, fx, fy), (nx, ny, c) = self.back, self.front, self.edge
        return np.where(nx * x + ny * y > c, f0 + fx * x + fy * y, b0 + bx * x + by * y)


def occlusion_scene(rng, width, height, disparity=(0.0, 64.0), port_offsets=PORT_OFFSETS, gain=0.01,
                    read_sigma=0.002, peak=1.0, texture="detail"):
    """Quad-camera Bayer frame of two slanted textured planes with an
    occlusion edge.

    The background plane B spans the lower part of `disparity`; the
    foreground plane F = B + delta (delta 4..16 px, its own small slope) is
    nearer everywhere and covers the scene points s with n . s > c, a seeded
    straight edge through the frame.  Camera k shows at pixel p the
    foreground point s_F (the inverse of p = s + d_F(s) o_k, as in
    plane_scene) when s_F lies in the foreground region, else the background
    point s_B; the two planes carry independent textures.  Returns (images,
    d) with d(x, y) the disparity of the surface seen at scene point (x, y)
    in the reference view (F inside the region, B outside)."""
    H, W = height, width
    scales, weights = TEXTURES[texture]
    texb = np.stack([smooth_noise(rng, H + 96, W + 96, scales=scales, weights=weights) for _ in range(3)])
    texf = np.stack([smooth_noise(rng, H + 96, W + 96, scales=scales, weights=weights) for _ in range(3)])
    dlo, dhi = disparity
    delta = rng.uniform(4.0, 16.0)
    span = max(dhi - dlo - delta - 4.0, 1.0)
    gxb = span * rng.uniform(0.3, 0.7) / W
    gyb = (span - gxb * W) / H
    d0b = dlo
    gxf = gxb + rng.uniform(-2.0, 2.0) / W
    gyf = gyb + rng.uniform(-2.0, 2.0) / H
    d0f = d0b + delta + 2.0
    ang = rng.uniform(0, 2 * math.pi)
    nx, ny = math.cos(ang), math.sin(ang)
    px, py = rng.uniform(0.3, 0.7) * W, rng.uniform(0.3, 0.7) * H
    cc = nx * px + ny * py

    dfun = TwoPlaneDisparity((d0b, gxb, gyb), (d0f, gxf, gyf), (nx, ny, cc))

    cmap = bayer_color_map(H, W)
    yy, xx = np.mgrid[0:H, 0:W].astype(np.float64)

    def inverse(k, d0, gx, gy):
        ox, oy = float(port_offsets[k][0]), float(port_offsets[k][1])
        qx, qy = xx - d0 * ox, yy - d0 * oy
        gq = (gx * qx + gy * qy) / (1.0 + gx * ox + gy * oy)
        return qx - ox * gq, qy - oy * gq

    def sample(tex, sx, sy):
        sx = sx + 48.0; sy = sy + 48.0
        x0 = np.clip(np.floor(sx).astype(np.int64), 0, W + 94); fx = sx - x0
        y0 = np.clip(np.floor(sy).astype(np.int64), 0, H + 94); fy = sy - y0
        return tex[cmap, y0, x0] * (1 - fx) * (1 - fy) + tex[cmap, y0, x0 + 1] * fx * (1 - fy) + \
            tex[cmap, y0 + 1, x0] * (1 - fx) * fy + tex[cmap, y0 + 1, x0 + 1] * fx * fy

    imgs = []
    for k in range(len(port_offsets)):
        fxs, fys = inverse(k, d0f, gxf, gyf)
        bxs, bys = inverse(k, d0b, gxb, gyb)
        fg = nx * fxs + ny * fys > cc
        v = peak * np.where(fg, sample(texf, fxs, fys), sample(texb, bxs, bys))
        v = v + np.sqrt(np.maximum(gain * v, 0.0)) * rng.standard_normal(v.shape) + read_sigma * rng.standard_normal(v.shape)
        imgs.append(v.astype(np.float32))
    return np.stack(imgs), dfun


def pitched(images, dstride, rows=None, fill=0.0):
    """Copy [cams][H][W] into [cams][rows][dstride] (extra rows / columns = fill)."""
    cams, H, W = images.shape
    rows = H if rows is None else rows
    out = np.full((cams, rows, dstride), fill, dtype=np.float32)
    out[:, :H, :W] = images
    return out


def _psf_pool(rng, n, sigma=(0.5, 1.5), offset=0.25):
    """n normalised 15x15 anisotropic Gaussian PSFs (taps -7..7)."""
    m = np.arange(-7, 8, dtype=np.float64)
    Y, X = np.meshgrid(m, m, indexing="ij")
    sx = rng.uniform(*sigma, n); sy = rng.uniform(*sigma, n)
    th = rng.uniform(0, math.pi, n)
    ox = rng.uniform(-offset, offset, n); oy = rng.uniform(-offset, offset, n)
    c, s = np.cos(th)[:, None, None], np.sin(th)[:, None, None]
    xr = (X[None] - ox[:, None, None]) * c + (Y[None] - oy[:, None, None]) * s
    yr = -(X[None] - ox[:, None, None]) * s + (Y[None] - oy[:, None, None]) * c
    h = np.exp(-0.5 * ((xr / sx[:, None, None]) ** 2 + (yr / sy[:, None, None]) ** 2))
    h /= h.sum(axis=(1, 2), keepdims=True)
    return h


def psf_to_clt(h):
    """Spatial kernels h[..., 15, 15] (rows = vertical taps -7..7) to the CLT
    domain [..., 4, 8, 8]: quadrant (CC, SC, CS, SS) = sum_mn h[m][n] *
    {cos|sin}(pi m (2u+1)/16) * {cos|sin}(pi n (2v+1)/16), vertical factor
    first, quadrant index = 2 * (vertical is sine) + (horizontal is sine)."""
    m = np.arange(-7, 8, dtype=np.float64)
    u = np.arange(8, dtype=np.float64)
    ang = math.pi * np.outer(2 * u + 1, m) / 16.0  # [8][15]
    C, S = np.cos(ang), np.sin(ang)
    out = np.empty(h.shape[:-2] + (4, 8, 8), dtype=np.float64)
    for q, (A, B) in enumerate(((C, C), (C, S), (S, C), (S, S))):
        out[..., q, :, :] = np.einsum("um,...mn,vn->...uv", A, h, B, optimize=True)
    return out


def kernel_tables(rng, geom, kind="gauss", pool=256, zero_extra=False, cams=4, psf_offset=0.25):
    """CLT kernel tables and CltExtra tables for every camera.

    kind 'gauss': seeded anisotropic Gaussian PSFs (sigma 0.5..1.5 px, centre
    within +-psf_offset px) drawn from a pool of `pool` shapes; 'identity':
    CC = 1, other quadrants 0.  Random kernel-centre offsets and Jacobians
    unless zero_extra.  Centred PSFs with zero_extra shift no camera, so the
    scene's disparity is measured without bias.
    Returns (kernels [cams][kv*kh*3*256], extra [cams][kv*kh*3*8]) float32.
    """
    kh, kv = geom["kernels_hor"], geom["kernels_vert"]
    nk = kv * kh * 3
    if kind == "identity":
        k = np.zeros((cams, nk, 4, 8, 8), dtype=np.float32)
        k[:, :, 0] = 1.0
    else:
        clt_pool = psf_to_clt(_psf_pool(rng, pool, offset=psf_offset)).astype(np.float32)
        pick = rng.integers(0, pool, size=(cams, nk))
        k = clt_pool[pick]
    extra = np.zeros((cams, nk, 8), dtype=np.float32)
    step = 1 << geom["kernels_lstep"]
    ky, kx = np.meshgrid(np.arange(kv), np.arange(kh), indexing="ij")
    cxk = np.repeat((kx * step - step // 2).reshape(-1), 3).astype(np.float32)
    cyk = np.repeat((ky * step - step // 2).reshape(-1), 3).astype(np.float32)
    extra[:, :, 2] = cxk
    extra[:, :, 3] = cyk
    if not zero_extra:
        extra[:, :, 0] = rng.integers(-16, 17, size=(cams, nk)) / 64.0
        extra[:, :, 1] = rng.integers(-16, 17, size=(cams, nk)) / 64.0
        extra[:, :, 4:8] = rng.integers(-40, 41, size=(cams, nk, 4)) / 4096.0
    return k.reshape(cams, -1), extra.reshape(cams, -1)


def tasks_grid(geom, rng=None, jitter=0.5, task_bits=ALL_TASK_BITS, disparity=None,
               port_offsets=PORT_OFFSETS, mask=None, disparity_error=0.0, return_error=False):
    """One task per tile in raster order (tiles with mask False are left out).

    xy[cam] = tile centre (8 tx + 4, 8 ty + 4) + U[-jitter, jitter] per
    camera + (d(tx, ty) + e) * port_offsets[cam] when `disparity` = (d0, gx,
    gy) (d = d0 + gx x + gy y at the tile centre) or a function d(x, y),
    rounded to 1/256 px; e = U[-disparity_error, disparity_error] per
    tile, the same for all cameras (the task's disparity error, so the tile's
    residual disparity is -e).  With return_error, returns (tasks, e)."""
    TX, TY, _ = tiles(geom)
    ty, tx = np.meshgrid(np.arange(TY), np.arange(TX), indexing="ij")
    tx = tx.reshape(-1); ty = ty.reshape(-1)
    if mask is not None:
        keep = np.asarray(mask).reshape(-1)
        tx, ty = tx[keep], ty[keep]
    n = tx.size
    t = np.zeros(n, dtype=TASK_DTYPE)
    t["task"] = task_bits
    t["txy"] = tx + (ty << 16)
    cx = (tx * 8 + 4).astype(np.float64)
    cy = (ty * 8 + 4).astype(np.float64)
    err = np.zeros(n)
    if disparity_error and rng is not None:
        err = rng.uniform(-disparity_error, disparity_error, n)
    for cam in range(4):
        x, y = cx.copy(), cy.copy()
        if rng is not None and jitter:
            x += rng.uniform(-jitter, jitter, n)
            y += rng.uniform(-jitter, jitter, n)
        if disparity is not None:
            if callable(disparity):
                d = disparity(cx, cy) + err
            else:
                d0, gx, gy = disparity
                d = d0 + gx * cx + gy * cy + err
            x += d * port_offsets[cam][0]
            y += d * port_offsets[cam][1]
        t["xy"][:, cam, 0] = np.round(x * 256.0) / 256.0
        t["xy"][:, cam, 1] = np.round(y * 256.0) / 256.0
    return (t, err) if return_error else t


def corr_indices(tasks, geom):
    """(tile << 8) | pair for every pair bit of every task (src/dtt8x8.cu:432-446)."""
    TX = geom["img_width"] // 8
    txy = tasks["txy"]
    tile = (txy & 0xFFFF) + (txy >> 16) * TX
    out = []
    for n in range(tasks.size):
        cm = (int(tasks["task"][n]) >> 4) & 0x3F
        for b in range(6):
            if cm & (1 << b):
                out.append((int(tile[n]) << 8) | b)
    return np.array(out, dtype=np.int32)


def corr_indices_fast(tasks, geom):
    TX = geom["img_width"] // 8
    txy = tasks["txy"].astype(np.int64)
    tile = (txy & 0xFFFF) + (txy >> 16) * TX
    cm = (tasks["task"].astype(np.int64) >> 4) & 0x3F
    bits = ((cm[:, None] >> np.arange(6)[None, :]) & 1).astype(bool)
    codes = (tile[:, None] << 8) | np.arange(6)[None, :]
    return codes[bits].astype(np.int32)


def texture_indices(tasks, geom, with_neighbors=False):
    """(tile << 8) | (1 << 7) for texture tasks (src/dtt8x8.cu:452-463)."""
    TX = geom["img_width"] // 8
    txy = tasks["txy"].astype(np.int64)
    tile = (txy & 0xFFFF) + (txy >> 16) * TX
    tex = (tasks["task"] & 0xF) != 0
    codes = (tile << 8) | (1 << 7)
    if with_neighbors:
        codes = codes | (tasks["task"] & 0xF)
    return codes[tex].astype(np.int32)
