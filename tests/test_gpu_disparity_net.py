"""GPU tests of the learned disparity residual: the tp_mlp_* kernels against
NumPy and the FP64 oracle (GEMM, features, gradients, Adam), and a trained
network against the plain fit on held-out synthetic scenes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


@pytest.mark.parametrize("M,N,K,ta,tb", [(70, 37, 51, 0, 0), (130, 256, 1350, 0, 0), (1350, 256, 97, 1, 0),
                                          (64, 128, 256, 0, 1), (33, 2, 128, 1, 1), (4096, 256, 1350, 0, 0),
                                          (1350, 256, 4096, 1, 0), (256, 128, 4096, 1, 0), (300, 0, 7, 0, 0),
                                          (200, 40, 0, 0, 0)])
@pytest.mark.parametrize("epi", ["plain", "bias_beta", "gelu"])
@pytest.mark.parametrize("tc", [False, True], ids=["simt", "tensor_core"])
def test_gemm(native, oracle, M, N, K, ta, tb, epi, tc):
    """tp_mlp_gemm (FP32 SIMT) and tp_mlp_gemm_tc (split-TF32 tensor-core
    MMAs) against FP64, within 1e-5 of the largest magnitude; the
    tensor-core GEMM's error flag stays clear.  K = 0 gives the epilogue of a
    zero product; N = 0 leaves C alone."""
    import torch
    from tile_processor_gpu_b200 import disparity_net as D
    rng = np.random.default_rng(M * 7 + N)
    A = rng.standard_normal((K, M) if ta else (M, K)).astype(np.float32)
    B = rng.standard_normal((N, K) if tb else (K, N)).astype(np.float32)
    C0 = rng.standard_normal((M, N)).astype(np.float32)
    bias = rng.standard_normal(N).astype(np.float32)
    a, b, c = _dev(A), _dev(B), _dev(C0)
    z = torch.zeros_like(c) if epi == "gelu" else None
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    D.gemm(a, b, c, M, N, K, ta=ta, tb=tb, beta=0.5 if epi == "bias_beta" else 0.0,
           bias=_dev(bias) if epi != "plain" else None, z=z, tc=tc, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    if N == 0:
        return
    ref = (A.T if ta else A).astype(np.float64) @ (B.T if tb else B).astype(np.float64)
    if epi != "plain":
        ref = ref + bias
    if epi == "bias_beta":
        ref = ref + 0.5 * C0
    den = lambda r: np.abs(r).max() or 1.0  # noqa: E731  (K = 0 without bias: an all-zero product)
    if epi == "gelu":
        assert np.max(np.abs(z.cpu().numpy() - ref)) / den(ref) < 1e-5
        ref = oracle.mlp_gelu(ref)
    assert np.max(np.abs(c.cpu().numpy() - ref)) / den(ref) < 1e-5


@pytest.mark.parametrize("tc", [False, True], ids=["simt", "tensor_core"])
def test_gradients_against_oracle(native, oracle, tc):
    import torch
    from tile_processor_gpu_b200 import disparity_net as D
    rng = np.random.default_rng(5)
    p = D.init_params(3)
    for k in p:
        if k.startswith("b"):
            p[k] = rng.normal(0, 0.1, p[k].shape).astype(np.float32)
    rows = 37
    x = rng.normal(0, 0.3, (rows, D.N_IN)).astype(np.float32)
    t = rng.normal(0, 0.5, rows).astype(np.float32)
    w = (rng.random(rows) > 0.2).astype(np.float32)
    net = D.DisparityMLP(p, tc=tc)
    xd = _dev(x)
    out = net.forward(xd, rows)
    loss = net.loss_backward(xd, rows, _dev(t), weight=_dev(w))
    torch.cuda.synchronize()
    net.check()
    ref_out, _ = oracle.mlp_forward(p, x.astype(np.float64))
    ref_loss, ref_g = oracle.mlp_loss_and_grads(p, x.astype(np.float64), t.astype(np.float64), w)
    assert np.max(np.abs(out.cpu().numpy() - ref_out)) / np.abs(ref_out).max() < 1e-5
    assert abs(loss - ref_loss) / abs(ref_loss) < 1e-5
    for k in D.PARAMS:
        gk = net.g[k].cpu().numpy()
        assert np.max(np.abs(gk - ref_g[k])) / np.abs(ref_g[k]).max() < 1e-4, k


def test_adam_step(native):
    import torch
    from tile_processor_gpu_b200 import _native
    from tile_processor_gpu_b200.api import _dptr
    rng = np.random.default_rng(6)
    p, g = rng.standard_normal(1000).astype(np.float32), rng.standard_normal(1000).astype(np.float32)
    m, v = rng.standard_normal(1000).astype(np.float32) * 0.1, rng.random(1000).astype(np.float32) * 0.1
    P, G, Mm, V = _dev(p), _dev(g), _dev(m), _dev(v)
    _native.call("tp_mlp_adam", 1000, _dptr(P), _dptr(G), _dptr(Mm), _dptr(V), 1e-3, 0.9, 0.999, 1e-8, 3, None)
    torch.cuda.synchronize()
    m2 = 0.9 * m + 0.1 * g
    v2 = 0.999 * v + 0.001 * g * g
    p2 = p - 1e-3 * (m2 / (1 - 0.9 ** 3)) / (np.sqrt(v2 / (1 - 0.999 ** 3)) + 1e-8)
    assert np.max(np.abs(P.cpu().numpy() - p2)) < 1e-6


def test_features(native):
    import torch
    import gpu_runner as R
    from cases import Case
    from tile_processor_gpu_b200 import disparity_net as D
    c = Case(128, 128, seed=9, border_mode=1)
    fr = R.Frame(c)
    R.convert(fr)
    idx = c.corr_idx[np.arange(len(c.corr_idx)) % 7 != 3]   # some pairs missing
    co = R.correlate(fr, idx, stride=229)
    feat = torch.full((c.TX * c.TY, D.N_IN), -5.0, device="cuda")
    D.features(fr.g, _dev(co), 229, 7, len(idx), torch.from_numpy(idx).cuda(), feat)
    torch.cuda.synchronize()
    got = feat.cpu().numpy()
    want = np.zeros((c.TX * c.TY, D.N_IN), np.float64)
    seen = np.zeros(c.TX * c.TY, bool)
    for e, code in enumerate(idx):
        want[code >> 8, (code & 0xFF) * 225:(code & 0xFF) * 225 + 225] = co[e, :225]
        seen[code >> 8] = True
    mx = np.abs(want).max(axis=1, keepdims=True)
    want = np.where(mx > 0, want / np.where(mx > 0, mx, 1), 0)
    assert np.max(np.abs(got[seen] - want[seen])) < 1e-6
    assert np.all(got[~seen] == -5.0)


def test_features_irregular_runs(native):
    """Runs the register path does not take: a pair listed twice (the later
    plane is kept, both count in the maximum), pair codes >= 6 (skipped) and
    a run of 40 entries; ordinary runs beside them."""
    import torch
    from tile_processor_gpu_b200 import api, disparity_net as D, synth
    geom = synth.geometry(128, 128)
    g = api.Geometry.from_dict(geom)
    TX, TY, _ = synth.tiles(geom)
    rng = np.random.default_rng(5)
    codes = []
    codes += [(3 << 8) | p for p in (0, 1, 2, 1)]                 # pair 1 twice
    codes += [(4 << 8) | p for p in (0, 6, 7, 5)]                 # codes 6, 7 skipped
    codes += [(5 << 8) | (i % 6) for i in range(40)]              # 40 entries
    codes += [(6 << 8) | p for p in (0, 1, 2, 3, 4, 5)]           # ordinary
    codes += [(7 << 8) | 2]                                       # one entry
    idx = np.array(codes, np.int32)
    stride = 230
    co = rng.normal(0, 1, (len(idx), stride)).astype(np.float32)
    co[len(idx) - 1, :225] *= 50.0
    feat = torch.full((TX * TY, D.N_IN), -5.0, device="cuda")
    D.features(g, torch.from_numpy(co).cuda(), stride, 7, len(idx), torch.from_numpy(idx).cuda(), feat)
    torch.cuda.synchronize()
    got = feat.cpu().numpy()
    for tile in (3, 4, 5, 6, 7):
        want = np.zeros(D.N_IN, np.float64)
        mx = 0.0
        for e, code in enumerate(idx):
            if code >> 8 != tile or (code & 0xFF) >= 6:
                continue
            p = code & 0xFF
            want[p * 225:(p + 1) * 225] = co[e, :225]
            mx = max(mx, float(np.abs(co[e, :225]).max()))
        np.testing.assert_allclose(got[tile], want / mx, rtol=0, atol=1e-6)
    untouched = np.ones(TX * TY, bool)
    untouched[[3, 4, 5, 6, 7]] = False
    assert np.all(got[untouched] == -5.0)


def test_combine_with_fallback(native):
    """tp_mlp_combine: plain + d where s < gate, plain elsewhere; +inf keeps all."""
    import torch
    from tile_processor_gpu_b200 import disparity_net as D
    rng = np.random.default_rng(8)
    n = 100003
    plain = rng.normal(0, 1, n).astype(np.float32)
    out = rng.normal(0, 1, (n, 2)).astype(np.float32)
    net = D.DisparityMLP(seed=0)
    rho = torch.full((n,), -7.0, device="cuda")
    for gate in (0.25, float("inf"), -10.0):
        net.gate = gate
        net.combine(_dev(plain), _dev(out), n, rho)
        torch.cuda.synchronize()
        want = plain + np.where(out[:, 1] < gate, out[:, 0], 0.0).astype(np.float32)
        assert np.array_equal(rho.cpu().numpy(), want)


def test_learned_residual_beats_plain_fit(native):
    """Trained on eight synthetic frames, on a held-out frame the network's
    estimate (plain fit + correction) has a smaller RMS error against the
    true disparity than the plain fit alone, and its stated variance ranks
    the errors (large-variance tiles err more)."""
    import torch
    from tile_processor_gpu_b200 import disparity_net as D
    data = [D.make_samples(1000 + s, 1024, 768) for s in range(8)]
    feats = torch.cat([d[0] for d in data])
    plain = torch.cat([d[1] for d in data])
    truth = torch.cat([d[2] for d in data])
    net = D.DisparityMLP(seed=1)
    D.train(net, feats, plain, truth, epochs=12, batch=2048, lr=1e-3)
    f2, p2, t2 = D.make_samples(5000, 1024, 768)
    rho, logvar = D.predict(net, f2, p2)
    torch.cuda.synchronize()
    a_plain = D.accuracy(p2, t2)
    a_net = D.accuracy(rho, t2)
    err = (rho - t2).abs()
    lo = err[logvar < logvar.median()].mean().item()
    hi = err[logvar >= logvar.median()].mean().item()
    print("\nheld-out: plain %s  learned %s  mean |err| low/high variance %.4f / %.4f" % (a_plain, a_net, lo, hi))
    assert a_net["rmse_px"] < a_plain["rmse_px"]
    assert hi > lo


@pytest.mark.parametrize("rows,ldx", [(200, 1352), (5000, 1352), (40000, 1352), (40000, 1360), (300, 1356),
                                      (129, 1352)])
def test_tensor_core_inference_matches_fp32(native, rows, ldx):
    """tp_mlp_infer_tc (TMA-fed TF32 layer 1, BF16 layer 2, FP32
    accumulation) against the FP32 forward pass: outputs within the rounding
    of the operands.  40000 rows give every CTA two or three tiles (the next
    tile's first blocks load during the epilogues) and a ragged last tile;
    129 rows a last tile of one row.  Columns past 1350 hold 1e30 and must not
    reach the result (the tensor map ends at column 1350)."""
    import torch
    from tile_processor_gpu_b200 import disparity_net as D
    rng = np.random.default_rng(rows + ldx)
    p = D.init_params(7)
    for k in p:
        if k.startswith("b"):
            p[k] = rng.normal(0, 0.1, p[k].shape).astype(np.float32)
    x = rng.uniform(-1, 1, (rows, D.N_IN)).astype(np.float32)
    net = D.DisparityMLP(p)
    xd = _dev(x)
    ref = net.forward(xd, rows).clone()
    xp = torch.full((rows, ldx), 1e30, dtype=torch.float32, device="cuda")
    xp[:, :D.N_IN] = xd
    net.pack()
    out = torch.full((rows, 2), -99.0, device="cuda")
    net.infer_tc(xp, rows, out, ldx=ldx)
    torch.cuda.synchronize()
    assert int(net.tc_err.item()) == 0
    r, o = ref.cpu().numpy(), out.cpu().numpy()
    assert np.all(np.isfinite(o))
    scale = np.abs(r).max(axis=0)
    err = np.abs(o - r).max(axis=0) / scale
    rms = np.sqrt(np.mean((o - r) ** 2)) / np.sqrt(np.mean(r ** 2))
    print("\ntensor-core vs fp32, rows %d ldx %d: max rel err %s, rms rel %.2e" % (rows, ldx, err, rms))
    assert np.all(err < 3e-2)
    assert rms < 1e-2
