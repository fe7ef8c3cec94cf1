"""CPU tests of the FP64 oracle: known-answer tests derived from the
mathematics, and pins against the reference's own outputs (golden fixtures
made by tests/golden/make_golden.py from the reference kernels)."""
import os

import numpy as np
import pytest

from cases import Case, blob_mask, rel_err
from tile_processor_gpu_b200 import synth as S

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_256x256_seed11.npz")


def test_dtt_matrices(oracle):
    c4, s4 = oracle.dtt_matrix(0), oracle.dtt_matrix(1)
    eye = np.eye(8)
    # orthonormal and symmetric -> involutory (DCT-IV o DCT-IV = I)
    assert np.abs(c4 @ c4.T - eye).max() < 1e-14
    assert np.abs(s4 @ s4.T - eye).max() < 1e-14
    assert np.abs(c4 @ c4 - eye).max() < 1e-14
    c2, s2 = oracle.dtt_matrix(2), oracle.dtt_matrix(3)
    # "non-orthonormal" DCT-II / DST-II: every row scaled by 1/2
    assert np.abs(c2 @ c2.T - np.diag([2.0] + [1.0] * 7)).max() < 1e-14
    assert np.abs(s2 @ s2.T - np.diag([1.0] * 7 + [2.0])).max() < 1e-14


def test_default_tables_match_library(oracle, native):
    from tile_processor_gpu_b200 import api
    for w in range(6):
        assert np.array_equal(oracle.default_lpf(w), api.get_lpf(w)), w
    # LPF tables: separable, 1 at DC, decreasing
    for w in range(6):
        t = oracle.default_lpf(w).reshape(8, 8).astype(np.float64)
        assert t[0, 0] == 1.0
        assert np.abs(t - np.outer(t[0], t[0])).max() < 1e-7
        assert np.all(np.diff(t[0]) < 0)


def test_alpha_fade_partition_of_unity(oracle):
    af = oracle.alpha_fade().reshape(16, 16, 16)
    # opposite single-neighbour fades sum to one: the overlap-add of two
    # neighbouring tiles reconstructs a flat field
    assert np.abs(af[1] + af[4] - 1).max() < 1e-12
    assert np.abs(af[2] + af[8] - 1).max() < 1e-12
    assert np.all(af[0] == 0) and np.all(af[15] == 1)


@pytest.mark.parametrize("border_mode", [0, 1])
def test_forward_inverse_reconstructs_bayer_planes(oracle, border_mode):
    """Identity kernel, zero residual shift: the forward CLT followed by the
    4-pass overlap-add inverse returns each sparse Bayer color plane exactly
    (shifted by the 4-pixel margin of the output image), on interior tiles."""
    rng = np.random.default_rng(1)
    W = H = 64
    g = S.geometry(W, H, border_mode=border_mode)
    imgs = S.smooth_bayer(rng, W, H)
    ker, ext = S.kernel_tables(rng, g, kind="identity", zero_extra=True)
    tasks = S.tasks_grid(g, None, jitter=0)
    clt = oracle.convert_correct_tiles(g, ext, ker, imgs, W, tasks)
    dst = W + 8
    cmap = S.bayer_color_map(H, W)
    for cam in range(4):
        rbg = np.zeros((3 * (H + 8), dst))
        oracle.imclt_rbg_all(g, clt[cam], rbg, dst)
        for color in range(3):
            plane = rbg[color * (H + 8):(color + 1) * (H + 8)]
            ref = np.zeros((H + 8, W + 8))
            ref[4:4 + H, 4:4 + W] = np.where(cmap == color, imgs[cam], 0.0)
            inner = (slice(12, H - 4), slice(12, W - 4))
            assert np.abs(plane[inner] - ref[inner]).max() < 1e-12


def _translated(rng, W, H, shifts):
    tex = np.stack([S.smooth_noise(rng, H + 64, W + 64, scales=(16, 4, 2), weights=(1, .7, .5)) for _ in range(3)])
    cmap = S.bayer_color_map(H, W)
    yy, xx = np.mgrid[0:H, 0:W].astype(np.float64)
    out = []
    for sx, sy in shifts:
        X = xx - sx + 32
        Y = yy - sy + 32
        x0 = np.floor(X).astype(int); y0 = np.floor(Y).astype(int); fx = X - x0; fy = Y - y0
        t = (tex[cmap, y0, x0] * (1 - fx) * (1 - fy) + tex[cmap, y0, x0 + 1] * fx * (1 - fy) +
             tex[cmap, y0 + 1, x0] * (1 - fx) * fy + tex[cmap, y0 + 1, x0 + 1] * fx * fy)
        out.append(t.astype(np.float32))
    return np.stack(out)


@pytest.mark.parametrize("s", [0.3, 0.7, 2.6])
def test_fractional_shift_aligns_tiles(oracle, s):
    """Cameras see the texture moved by (s,0), (0,s), (s,s); tasks centred
    on the moved positions: after the residual-shift rotation every pair
    correlates with its peak at the centre (interior tiles)."""
    rng = np.random.default_rng(0)
    W = H = 128
    g = S.geometry(W, H, border_mode=1)
    shifts = [(0, 0), (s, 0), (0, s), (s, s)]
    imgs = _translated(rng, W, H, shifts)
    ker, ext = S.kernel_tables(rng, g, kind="identity", zero_extra=True)
    tasks = S.tasks_grid(g, None, jitter=0)
    for k, (a, b) in enumerate(shifts):
        tasks["xy"][:, k, 0] += a
        tasks["xy"][:, k, 1] += b
    clt = oracle.convert_correct_tiles(g, ext, ker, imgs, W, tasks)
    idx = S.corr_indices_fast(tasks, g)
    co = oracle.correlate2D(g, clt, 3, .25, .25, .5, 0.5, idx, 225, 7).reshape(-1, 6, 225)
    TX = W // 8
    inner = np.arange(TX * TX).reshape(TX, TX)[4:-4, 4:-4].reshape(-1)
    assert np.mean(co[inner].argmax(2) == 112) > 0.99


@pytest.mark.parametrize("dx,dy", [(2, 0), (0, -3), (1, 2)])
def test_integer_offset_peak_position(oracle, dx, dy):
    """Camera 1 content moved by (dx, dy) without moving its tiles: the pair
    (0, 1) correlation peaks on the side of (+dx, +dy) in the centred 15x15,
    within one pixel of it (the tile window pulls the peak towards the
    centre)."""
    rng = np.random.default_rng(3)
    W = H = 128
    g = S.geometry(W, H, border_mode=1)
    imgs = _translated(rng, W, H, [(0, 0), (dx, dy), (0, 0), (0, 0)])
    ker, ext = S.kernel_tables(rng, g, kind="identity", zero_extra=True)
    tasks = S.tasks_grid(g, None, jitter=0)
    clt = oracle.convert_correct_tiles(g, ext, ker, imgs, W, tasks)
    TX = W // 8
    inner = np.arange(TX * TX).reshape(TX, TX)[4:-4, 4:-4].reshape(-1)
    idx = (inner << 8).astype(np.int32)  # pair 0 = cameras 0, 1
    co = oracle.correlate2D(g, clt, 3, .25, .25, .5, 0.05, idx, 225, 7)
    am = co.argmax(1)
    py, px = am // 15 - 7, am % 15 - 7
    ok = (np.sign(px) == np.sign(dx)) & (np.sign(py) == np.sign(dy)) & (np.abs(px - dx) <= 1) & (np.abs(py - dy) <= 1)
    assert np.mean(ok) > 0.95


def _list_model(tasks, TX, TY):
    """Direct statement of the texture-list rules (neighbours, window,
    sub-list of every tile)."""
    tex = {}
    for n, t in enumerate(tasks):
        if t["task"] & 0xF:
            tex[(int(t["txy"]) & 0xFFFF, int(t["txy"]) >> 16)] = n
    xs = [k[0] for k in tex]
    ys = [k[1] for k in tex]
    woi = [min(xs), min(ys), max(xs), max(ys)]
    nbr, entries = {}, {s: [] for s in range(8)}
    for (x, y), n in tex.items():
        d = ((y > 0 and (x, y - 1) in tex) * 1 | (x < TX - 1 and (x + 1, y) in tex) * 2 |
             (y < TY - 1 and (x, y + 1) in tex) * 4 | (x > 0 and (x - 1, y) in tex) * 8)
        nbr[n] = d
        if d:
            border = x == woi[0] or y == woi[1] or x == TX - 1 or y == woi[3]
            slot = 2 * (x & 1) + 4 * (y & 1) + int(border)
            entries[slot].append(d | ((x + y * TX) << 8) | 0x80)
    return nbr, entries, [woi[0], woi[1], woi[2] + 1 - woi[0], woi[3] + 1 - woi[1]]


@pytest.mark.parametrize("fraction", [0.2, 0.6, 1.0])
def test_texture_list_rules(oracle, fraction):
    rng = np.random.default_rng(7)
    g = S.geometry(128, 96)
    TX, TY, TYA = S.tiles(g)
    m = blob_mask(rng, TX, TY, fraction) if fraction < 1 else np.ones((TY, TX), bool)
    tasks = S.tasks_grid(g, rng, mask=m)
    t_out, idx, counts, woi = oracle.prepare_texture_list(g, tasks, TX, TY)
    nbr, entries, woi_m = _list_model(tasks, TX, TY)
    assert list(woi) == woi_m
    for n, d in nbr.items():
        assert t_out["task"][n] & 0xF == d
    quarter = TX * (TYA >> 2)
    for q in range(4):
        inner = idx[q * quarter: q * quarter + counts[2 * q]]
        border = idx[(q + 1) * quarter - counts[2 * q + 1]: (q + 1) * quarter]
        assert sorted(inner.tolist()) == sorted(entries[2 * q])
        assert sorted(border.tolist()) == sorted(entries[2 * q + 1])


# ---- pins against the reference's own outputs --------------------------------

@pytest.fixture(scope="module")
def golden():
    if not os.path.exists(GOLDEN):
        pytest.skip("golden fixture not generated")
    import make_golden as MG
    d = dict(np.load(GOLDEN))
    case = MG.golden_case()
    assert MG.input_digest(case) == str(d["input_sha256"]), "input generator drifted"
    return MG, case, d


def _golden_clt_arrays(MG, case, d):
    """the reference's CLT of the selected tiles, placed into zero arrays"""
    n = case.TX * case.TY * 768
    clt = [np.zeros(n) for _ in range(4)]
    for k, t in enumerate(MG.sel_tile_ids(case)):
        for c in range(4):
            clt[c][t * 768:(t + 1) * 768] = d["clt"][k, c]
    return clt


def test_golden_convert(oracle, golden):
    MG, case, d = golden
    clt = oracle.convert_correct_tiles(case.geom, case.extra, case.kernels, case.pitched, case.dstride, case.tasks)
    sel = MG.sel_tile_ids(case)
    mine = np.stack([np.stack([clt[c].reshape(-1, 768)[t] for c in range(4)]) for t in sel])
    assert rel_err(mine, d["clt"]) < 1e-5


def test_golden_correlate(oracle, golden):
    MG, case, d = golden
    clt = _golden_clt_arrays(MG, case, d)
    sel = MG.sel_tile_ids(case)
    idx = np.array([(int(t) << 8) | p for t in sel for p in range(6)], dtype=np.int32)
    co = oracle.correlate2D(case.geom, clt, 3, .25, .25, .5, 0.05, idx, 225, 7)
    assert rel_err(co, d["corr"]) < 1e-5
    co4 = oracle.correlate2D(case.geom, clt, 1, .25, .25, .5, 0.05, idx[:24], 81, 4)
    assert rel_err(co4, d["corr_r4m"]) < 1e-5


def test_golden_textures(oracle, golden):
    import conditioning
    MG, case, d = golden
    clt = _golden_clt_arrays(MG, case, d)
    sel = MG.sel_tile_ids(case)
    tex_idx = np.array([(int(t) << 8) | (1 << 7) for t in sel], dtype=np.int32)
    bad, out = conditioning.unstable_mask(oracle, case, clt, tex_idx, keep_weights=1)
    keep = ~bad
    ref = d["tex"].reshape(out.shape)
    for s in range(4):
        assert keep[:, s].mean() > 0.99
        assert rel_err(out[:, s][keep[:, s]], ref[:, s][keep[:, s]]) < 1e-5, s
    for s in range(4, 8):
        assert rel_err(out[:, s][keep[:, s]], ref[:, s][keep[:, s]]) < 1e-4, s
    # the reference's one-pass variance cancels where the cameras agree
    for s in range(8, 12):
        assert rel_err(out[:, s][keep[:, s]], ref[:, s][keep[:, s]]) < 1e-3, s


def test_golden_imclt(oracle, golden):
    MG, case, d = golden
    clt = oracle.convert_correct_tiles(case.geom, case.extra, case.kernels, case.pitched, case.dstride, case.tasks)
    g = dict(case.geom, debug_marks=1)
    dst = case.W + 8 + 24
    img = np.zeros((3 * (case.H + 8), dst))
    oracle.imclt_rbg_all(g, clt[0], img, dst)
    H = case.H + 8
    mine = np.stack([np.stack([img[c * H + r: c * H + r + 40, x: x + 40] for r, x in MG.CROPS]) for c in range(3)])
    assert rel_err(mine, d["imclt"]) < 1e-5


def test_golden_texture_list(oracle, golden):
    MG, case, d = golden
    st = MG.sparse_tasks(case)
    t_out, idx, counts, woi = oracle.prepare_texture_list(case.geom, st, case.TX, case.TY)
    assert np.array_equal(t_out["task"], d["list_task"])
    assert np.array_equal(counts, d["list_counts"])
    assert np.array_equal(woi, d["list_woi"])
    quarter = case.TX * (case.TYA >> 2)
    subl = []
    for q in range(4):
        subl.append(np.sort(idx[q * quarter: q * quarter + counts[2 * q]]))
        subl.append(np.sort(idx[(q + 1) * quarter - counts[2 * q + 1]: (q + 1) * quarter]))
    assert np.array_equal(np.concatenate(subl), d["list_entries"])


def test_golden_rgba(oracle, golden):
    MG, case, d = golden
    clt = oracle.convert_correct_tiles(case.geom, case.extra, case.kernels, case.pitched, case.dstride, case.tasks)
    stride = (case.TX + 1) * 8 + 40
    rows = (case.TY + 1) * 8 * 4 + 8
    out, _, _, _, woi = oracle.generate_RBGA(case.geom, case.tasks, case.TX, case.TY, clt, case.port_offsets, stride,
                                             rows)
    assert np.array_equal(woi, d["rgba_woi"])
    h = (woi[3] + 1) * 8
    mine = np.stack([np.stack([out[s * h + r: s * h + r + 40, c: c + 40] for r, c in MG.CROPS]) for s in range(4)])
    # smooth [0, 1] scene: no unstable pixels fall in the crops
    assert rel_err(mine, d["rgba"]) < 1e-5
