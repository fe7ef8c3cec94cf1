"""GPU tests of tp_disparity_fit against the oracle's fit on the same
correlation tiles, and of the whole plain method's accuracy on a plane scene
of known disparity."""
import numpy as np
import pytest
import torch

from cases import Case
from tile_processor_gpu_b200 import synth as S

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def _fit_gpu(geom, corrs, idx, radius=7, mode=0, pair_mask=0x3F, port_offsets=S.PORT_OFFSETS):
    from tile_processor_gpu_b200 import api
    g = api.Geometry.from_dict(geom)
    TX, TY = geom["img_width"] // 8, geom["img_height"] // 8
    c = torch.from_numpy(np.ascontiguousarray(corrs, np.float32)).to(DEV)
    i = torch.from_numpy(np.ascontiguousarray(idx, np.int32)).to(DEV)
    po = torch.from_numpy(np.ascontiguousarray(port_offsets, np.float32).reshape(-1)).to(DEV)
    d = torch.full((TX * TY,), float("nan"), device=DEV)
    s = torch.full((TX * TY,), float("nan"), device=DEV)
    api.disparity_fit(g, c, c.shape[1], radius, len(idx), i, po, d, s, pair_mask=pair_mask, mode=mode)
    torch.cuda.synchronize()
    return d.cpu().numpy().astype(np.float64), s.cpu().numpy().astype(np.float64)


def _profile_gap(corrs, idx, TX, TY, radius=7):
    """per tile: relative gap between the two largest S(k) (FP64), NaN where
    not fitted -- a tiny gap may pick another integer maximum in float32"""
    n = 2 * radius + 1
    c = corrs.reshape(len(idx), n, n).astype(np.float64)
    k = np.arange(-radius, radius + 1)
    prof = {}
    for e, code in enumerate(idx):
        t, p = int(code) >> 8, int(code) & 0xFF
        bx, by = S.PORT_OFFSETS[S.PAIRS[p][1]] - S.PORT_OFFSETS[S.PAIRS[p][0]]
        v = c[e, (k * by).astype(int) + radius, (k * bx).astype(int) + radius]
        prof[t] = prof.get(t, 0.0) + v
    gap = np.full(TX * TY, np.nan)
    for t, v in prof.items():
        a = np.sort(v)
        gap[t] = (a[-1] - a[-2]) / max(abs(a[-1]), 1e-30)
    return gap


@pytest.mark.parametrize("name,kw", [("A256", dict(width=256, height=256, seed=1)),
                                     ("B512plane", dict(width=512, height=384, seed=2, scene="plane"))])
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_fit_matches_oracle(oracle, name, kw, mode):
    import gpu_runner as R
    c = Case(border_mode=0, **kw)
    fr = R.Frame(c)
    R.convert(fr)
    co = R.correlate(fr, c.corr_idx, stride=225)
    dg, sg = _fit_gpu(c.geom, co, c.corr_idx, mode=mode)
    do, so = oracle.disparity_fit(c.geom, co, c.corr_idx, 7, mode=mode)
    fitted = ~np.isnan(do)
    assert np.array_equal(fitted, ~np.isnan(dg))
    gap = _profile_gap(co, c.corr_idx, c.TX, c.TY)
    clear = fitted & (gap > 1e-5)
    assert clear.mean() > 0.99 * fitted.mean()
    assert np.max(np.abs(dg[clear] - do[clear])) < 1e-4
    assert np.max(np.abs(sg[clear] - so[clear]) / np.maximum(np.abs(so[clear]), 1e-6)) < 1e-4


def test_constructed_planes_and_runs(oracle):
    """Quadratic peaks (exact answer), runs of partial pairs, a masked run
    and an out-of-grid tile, as in the oracle's own test."""
    R_ = 7
    y, x = np.mgrid[-R_:R_ + 1, -R_:R_ + 1].astype(np.float64)

    def planes(rho):
        out = []
        for p in range(6):
            bx, by = S.PORT_OFFSETS[S.PAIRS[p][1]] - S.PORT_OFFSETS[S.PAIRS[p][0]]
            out.append(1.0 - ((x - rho * bx) ** 2 + (y - rho * by) ** 2) / 400.0)
        return np.stack(out).reshape(6, -1).astype(np.float32)

    a, b = planes(1.25), planes(-0.5)
    corrs = np.concatenate([a[:3], b, a[3:]])
    idx = np.array([(3 << 8) + 0, (3 << 8) + 1, (3 << 8) + 2] + [(7 << 8) + p for p in range(6)] +
                   [(99999 << 8) + 3, (99999 << 8) + 4, (99999 << 8) + 5], np.int32)
    geom = S.geometry(64, 64)
    d, s = _fit_gpu(geom, corrs, idx)
    assert abs(d[3] - 1.25) < 1e-5 and abs(d[7] + 0.5) < 1e-5
    assert np.count_nonzero(~np.isnan(d)) == 2
    d2, _ = _fit_gpu(geom, corrs, idx, pair_mask=0x30)
    assert np.isnan(d2[3]) and abs(d2[7] + 0.5) < 1e-5


def test_plain_method_accuracy_matches_oracle(oracle):
    """Noisy plane scene, per-tile disparity error U[-0.5, 0.5]: the GPU
    method (forward CLT, correlation, fit) and the FP64 oracle method reach
    the same RMS error against the true disparity (within 0.005 px), both
    below 0.25 px on interior tiles."""
    import gpu_runner as R
    from tile_processor_gpu_b200 import api
    W, H = 512, 384
    rng = np.random.default_rng(12)
    g = S.geometry(W, H, image_rows=H + 16)
    imgs, disp = S.plane_scene(rng, W, H, disparity=(0.0, 16.0), texture="detail")
    pit = S.pitched(imgs, W + 64, H + 16)
    kern, extra = S.kernel_tables(rng, g, pool=64, zero_extra=True, psf_offset=0.0)
    tasks, err = S.tasks_grid(g, rng, jitter=0.0, disparity=disp, disparity_error=0.5, return_error=True)
    idx = S.corr_indices_fast(tasks, g)
    TX, TY = W // 8, H // 8
    tx, ty = tasks["txy"] & 0xFFFF, tasks["txy"] >> 16
    inner = (tx >= 3) & (tx < TX - 3) & (ty >= 3) & (ty < TY - 3)
    # GPU
    ga = api.Geometry.from_dict(g)
    im = [torch.from_numpy(pit[k]).to(DEV) for k in range(4)]
    ke = [torch.from_numpy(kern[k]).to(DEV) for k in range(4)]
    ex = [torch.from_numpy(extra[k]).to(DEV) for k in range(4)]
    clt = [torch.zeros(TX * TY * 768, device=DEV) for _ in range(4)]
    P = api.PointerArray
    pe, pk, pi, pc = P(ex), P(ke), P(im), P(clt)
    td = api.tasks_to_device(tasks, DEV)
    api.convert_correct_tiles(ga, pe, pk, pi, td, pc, W + 64, tasks.size, 0)
    idd = torch.from_numpy(idx).to(DEV)
    co = torch.empty((len(idx), 225), device=DEV)
    api.correlate2D(ga, pc, 3, .25, .25, .5, 0.05, len(idx), idd, 225, 7, co)
    po = torch.from_numpy(S.PORT_OFFSETS.reshape(-1)).to(DEV)
    dd = torch.full((TX * TY,), float("nan"), device=DEV)
    ss = torch.full((TX * TY,), float("nan"), device=DEV)
    api.disparity_fit(ga, co, 225, 7, len(idx), idd, po, dd, ss)
    torch.cuda.synchronize()
    got = dd.cpu().numpy()[ty * TX + tx]
    # oracle
    clt_o = oracle.convert_correct_tiles(g, extra, kern, pit, W + 64, tasks)
    co_o = oracle.correlate2D(g, clt_o, 3, .25, .25, .5, 0.05, idx, 225, 7)
    do, _ = oracle.disparity_fit(g, co_o, idx, 7)
    ref = do[ty * TX + tx]
    truth = -err
    rms_g = np.sqrt(np.mean((got[inner] - truth[inner]) ** 2))
    rms_o = np.sqrt(np.mean((ref[inner] - truth[inner]) ** 2))
    assert rms_g < 0.25 and rms_o < 0.25
    assert abs(rms_g - rms_o) < 0.005
