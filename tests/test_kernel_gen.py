"""The CLT kernel-table generator: the oracle's FP64 formula (known answers,
and the convolution it approximates through the forward and inverse CLT),
and tp_psf_to_clt on the GPU against it."""
import numpy as np
import pytest

from tile_processor_gpu_b200 import synth as S

TAPS = np.arange(-7, 8)


def _gauss(sig):
    Y, X = np.meshgrid(TAPS, TAPS, indexing="ij")
    h = np.exp(-0.5 * (X ** 2 + Y ** 2) / sig ** 2)
    return h / h.sum()


def test_centre_tap_is_identity(oracle):
    h = np.zeros((15, 15)); h[7, 7] = 1.0
    k = oracle.psf_to_clt(h)
    assert np.allclose(k[0], 1.0, atol=1e-15) and np.allclose(k[1:], 0.0, atol=1e-15)


def test_two_formulations_agree(oracle):
    """the oracle's direct tap sum and the separable einsum of the synthetic
    input generator"""
    h = S._psf_pool(np.random.default_rng(4), 5)
    assert np.max(np.abs(oracle.psf_to_clt(h) - S.psf_to_clt(h))) < 1e-14


def test_symmetries(oracle):
    """an even kernel has no sine parts; a kernel odd in x only has SC"""
    h = _gauss(0.8)
    k = oracle.psf_to_clt(h)
    assert np.max(np.abs(k[1:])) < 1e-15
    odd = np.zeros((15, 15)); odd[7, 8] = 0.5; odd[7, 6] = -0.5
    k = oracle.psf_to_clt(odd)
    assert np.max(np.abs(k[[0, 2, 3]])) < 1e-15 and np.max(np.abs(k[1])) > 0.1


@pytest.mark.parametrize("sig,bound", [(0.3, 5e-4), (0.5, 1.5e-2)])
def test_inverse_clt_approximates_convolution(oracle, sig, bound):
    """forward CLT with the generated kernel, then the overlap-add inverse:
    each colour's sparse Bayer plane convolved with the kernel, on interior
    pixels, within the measured approximation of the CLT-domain product"""
    from scipy.signal import convolve2d
    W = H = 96
    rng = np.random.default_rng(0)
    g = S.geometry(W, H, border_mode=1)
    x = S.smooth_noise(rng, H, W, scales=(16, 6, 3), weights=(1, .8, .6)).astype(np.float32)
    h = _gauss(sig)
    K = oracle.psf_to_clt(h).astype(np.float32)
    kv, kh = g["kernels_vert"], g["kernels_hor"]
    ker = np.broadcast_to(K, (4, kv * kh * 3, 4, 8, 8)).reshape(4, -1).copy()
    _, extra = S.kernel_tables(rng, g, kind="identity", zero_extra=True)
    clt = oracle.convert_correct_tiles(g, extra, ker, np.stack([x] * 4), W, S.tasks_grid(g, None, jitter=0))
    rbg = np.zeros(3 * (H + 8) * (W + 8))
    oracle.imclt_rbg_all(g, clt[0], rbg, W + 8)
    rbg = rbg.reshape(3, H + 8, W + 8)
    cmap = S.bayer_color_map(H, W)
    sl = np.s_[24:-24, 24:-24]
    for col in range(3):
        ref = convolve2d(np.where(cmap == col, x, 0.0), h, mode="same")
        got = rbg[col, 4:4 + H, 4:4 + W]
        assert np.abs(got[sl] - ref[sl]).max() / np.abs(ref[sl]).max() < bound


@pytest.mark.gpu
def test_gpu_generator_matches_oracle(oracle, native):
    import torch
    from tile_processor_gpu_b200 import api
    rng = np.random.default_rng(7)
    h = np.concatenate([S._psf_pool(rng, 300), rng.standard_normal((20, 15, 15))]).astype(np.float32)
    dev = torch.from_numpy(h).cuda()
    out = torch.full((h.shape[0], 256), -9.0, device="cuda")
    api.psf_to_clt(dev, out)
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(-1, 4, 8, 8)
    want = oracle.psf_to_clt(h.astype(np.float64))
    scale = np.abs(want).reshape(len(h), -1).max(axis=1)[:, None, None, None]
    assert np.max(np.abs(got - want) / scale) < 2e-7     # double accumulation, one float rounding


@pytest.mark.gpu
def test_generated_tables_drive_convert(oracle, native):
    """a camera table made on the GPU gives the same CLT as the same table
    made on the host"""
    import torch
    import gpu_runner as R
    from cases import Case
    from tile_processor_gpu_b200 import api
    c = Case(256, 256, seed=5, border_mode=0)
    rng = np.random.default_rng(8)
    nk = c.geom["kernels_vert"] * c.geom["kernels_hor"] * 3
    h = S._psf_pool(rng, nk).astype(np.float32)
    table_host = oracle.psf_to_clt(h.astype(np.float64)).astype(np.float32).reshape(-1)
    dev_h = torch.from_numpy(h).cuda()
    fr = R.Frame(c)
    api.psf_to_clt(dev_h, fr.kernels[0])
    torch.cuda.synchronize()
    assert np.max(np.abs(fr.kernels[0].cpu().numpy() - table_host)) < 1e-6
