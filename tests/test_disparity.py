"""CPU tests of the disparity fit's oracle: known answers on constructed
correlation tiles, list handling, and the accuracy of the whole plain method
(forward CLT -> pair correlation -> fit) on a plane scene of known
disparity."""
import numpy as np
import pytest

from tile_processor_gpu_b200 import synth as S

R = 7
N = 2 * R + 1
PAIR_B = [(1, 0), (1, 0), (0, 1), (0, 1), (1, 1), (1, -1)]  # port_offsets[j] - port_offsets[i], square quad


def _planes(rho, shape):
    """six (2r+1)^2 tiles peaking at rho * b_p with the given profile"""
    y, x = np.mgrid[-R:R + 1, -R:R + 1].astype(np.float64)
    out = []
    for bx, by in PAIR_B:
        d2 = (x - rho * bx) ** 2 + (y - rho * by) ** 2
        out.append(shape(d2))
    return np.stack(out).astype(np.float32)


GEOM = S.geometry(64, 64)


@pytest.mark.parametrize("rho", [0.0, 0.37, -1.62, 2.9, -4.25])
@pytest.mark.parametrize("mode", [0, 1])
def test_quadratic_peak_is_exact(oracle, rho, mode):
    """Correlations that are quadratic in the offset make S(k) a parabola:
    both parabola fits return rho exactly."""
    c = _planes(rho, lambda d2: 1.0 - d2 / 400.0)
    idx = (5 << 8) + np.arange(6, dtype=np.int32)
    d, s = oracle.disparity_fit(GEOM, c.reshape(6, -1), idx, R, mode=mode)
    assert abs(d[5] - rho) < 1e-5          # float32 planes, curvature 0.03 per unit
    assert abs(s[5] - 1.0) < 1e-5          # fitted peak per pair
    assert np.isnan(d[4]) and np.isnan(d[6])


@pytest.mark.parametrize("rho", [0.3, -2.45])
def test_gaussian_peak_modes(oracle, rho):
    """Gaussian peaks: the 3-point parabola is within 0.05 px, the centroid
    within 0.2 px, and all modes find the right integer neighbourhood."""
    c = _planes(rho, lambda d2: np.exp(-0.5 * d2 / 1.3 ** 2)).reshape(6, -1)
    idx = (9 << 8) + np.arange(6, dtype=np.int32)
    got = [oracle.disparity_fit(GEOM, c, idx, R, mode=m)[0][9] for m in range(3)]
    assert abs(got[0] - rho) < 0.05
    assert abs(got[1] - rho) < 0.12
    assert abs(got[2] - rho) < 0.2


def test_pair_mask_runs_and_range(oracle):
    """A tile's run ends where the next tile starts; masked pairs and
    out-of-grid tiles are skipped; k whose sample leaves the tile is unused."""
    a = _planes(1.25, lambda d2: 1.0 - d2 / 400.0).reshape(6, -1)
    b = _planes(-0.5, lambda d2: 1.0 - d2 / 400.0).reshape(6, -1)
    corrs = np.concatenate([a[:3], b, a[3:]])
    idx = np.array([(3 << 8) + 0, (3 << 8) + 1, (3 << 8) + 2] + [(7 << 8) + p for p in range(6)] +
                   [(99999 << 8) + 3, (99999 << 8) + 4, (99999 << 8) + 5], np.int32)
    d, s = oracle.disparity_fit(GEOM, corrs, idx, R, mode=0)
    assert abs(d[3] - 1.25) < 1e-5 and abs(d[7] + 0.5) < 1e-5
    d2, _ = oracle.disparity_fit(GEOM, corrs, idx, R, mode=0, pair_mask=0x30)   # diagonal pairs only
    assert np.isnan(d2[3]) and abs(d2[7] + 0.5) < 1e-5
    assert np.count_nonzero(~np.isnan(d)) == 2


def test_fit_profile_edges(oracle):
    """Maximum at the edge of the profile: no sub-pixel step beyond it; flat
    or rising profiles stay at the integer maximum."""
    S_ = np.linspace(0.0, 1.0, N)
    assert oracle.fit_profile(S_, mode=0)[0] == R
    v = np.ones(N, np.int32); v[R + 1] = 0
    S2 = -((np.arange(N) - R - 0.3) ** 2)
    assert oracle.fit_profile(S2, v, mode=0)[0] == 0.0      # neighbour unusable -> integer maximum
    assert abs(oracle.fit_profile(S2, mode=0)[0] - 0.3) < 1e-12


def _plane_pipeline(oracle, W, H, err, seed, noise=True):
    rng = np.random.default_rng(seed)
    g = S.geometry(W, H, image_rows=H + 16)
    kw = {} if noise else dict(gain=0.0, read_sigma=0.0)
    imgs, disp = S.plane_scene(rng, W, H, disparity=(0.0, 16.0), texture="detail", **kw)
    pit = S.pitched(imgs, W + 64, H + 16)
    kern, extra = S.kernel_tables(rng, g, pool=64, zero_extra=True, psf_offset=0.0)
    tasks, e = S.tasks_grid(g, rng, jitter=0.0, disparity=disp, disparity_error=err, return_error=True)
    clt = oracle.convert_correct_tiles(g, extra, kern, pit, W + 64, tasks)
    idx = S.corr_indices_fast(tasks, g)
    co = oracle.correlate2D(g, clt, 3, .25, .25, .5, 0.05, idx, 225, 7)
    d, s = oracle.disparity_fit(g, co, idx, 7, mode=0)
    TX, TY = W // 8, H // 8
    tx, ty = tasks["txy"] & 0xFFFF, tasks["txy"] >> 16
    inner = (tx >= 3) & (tx < TX - 3) & (ty >= 3) & (ty < TY - 3)
    return d[ty * TX + tx], -e, inner


def test_plane_scene_accuracy(oracle):
    """One pass of the plain method on the noisy plane scene: residual
    disparity within 0.25 px RMS of the truth on interior tiles (the truth
    spreads 0.29 px RMS), slope of fit on truth above 0.6."""
    got, truth, inner = _plane_pipeline(oracle, 256, 256, 0.5, 7)
    res = got[inner] - truth[inner]
    assert np.sqrt(np.mean(res ** 2)) < 0.25
    assert np.polyfit(truth[inner], got[inner], 1)[0] > 0.6


def test_occlusion_scene_geometry(oracle):
    """Two planes with an occlusion edge (the learned residual's training
    scenes): tasks placed by the per-point disparity function, one pass of
    the plain method, noise-free.  Tiles whose footprint stays on one side
    of the edge match the truth as on a single plane; tiles straddling the
    edge are worse."""
    W = H = 256
    rng = np.random.default_rng(21)
    g = S.geometry(W, H, image_rows=H + 16)
    imgs, dfun = S.occlusion_scene(rng, W, H, disparity=(0.0, 24.0), gain=0.0, read_sigma=0.0)
    pit = S.pitched(imgs, W + 64, H + 16)
    kern, extra = S.kernel_tables(rng, g, pool=64, zero_extra=True, psf_offset=0.0)
    tasks, e = S.tasks_grid(g, rng, jitter=0.0, disparity=dfun, disparity_error=0.5, return_error=True)
    clt = oracle.convert_correct_tiles(g, extra, kern, pit, W + 64, tasks)
    idx = S.corr_indices_fast(tasks, g)
    co = oracle.correlate2D(g, clt, 3, .25, .25, .5, 0.05, idx, 225, 7)
    d, _ = oracle.disparity_fit(g, co, idx, 7, mode=0)
    TX, TY = W // 8, H // 8
    tx, ty = tasks["txy"] & 0xFFFF, tasks["txy"] >> 16
    res = d[ty * TX + tx] + e
    nx, ny, c = dfun.edge
    dist = np.abs(nx * (tx * 8 + 4) + ny * (ty * 8 + 4) - c)
    inner = (tx >= 3) & (tx < TX - 3) & (ty >= 3) & (ty < TY - 3)
    far, near = inner & (dist > 24), inner & (dist < 6)
    assert far.sum() > 100 and near.sum() > 10
    rms_far, rms_near = np.sqrt(np.mean(res[far] ** 2)), np.sqrt(np.mean(res[near] ** 2))
    assert rms_far < 0.2, rms_far
    assert rms_near > rms_far


def test_plane_scene_noise_free(oracle):
    """Without noise one pass is within 0.2 px RMS."""
    got, truth, inner = _plane_pipeline(oracle, 256, 256, 0.5, 8, noise=False)
    assert np.sqrt(np.mean((got[inner] - truth[inner]) ** 2)) < 0.2
