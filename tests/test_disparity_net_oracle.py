"""CPU tests pinning the oracle of the learned disparity residual: its
analytic gradients against central finite differences, and the loss of a
known case."""
import numpy as np


def _small(seed):
    from tile_processor_gpu_b200 import disparity_net as D
    rng = np.random.default_rng(seed)
    p = D.init_params(seed)
    p = {k: v.astype(np.float64) for k, v in p.items()}
    for k in p:
        if k.startswith("b"):
            p[k] = rng.normal(0, 0.1, p[k].shape)
    x = rng.normal(0, 0.3, (5, p["W1"].shape[0]))
    t = rng.normal(0, 0.5, 5)
    return p, x, t


def test_gradients_match_finite_differences(oracle):
    p, x, t = _small(1)
    loss, g = oracle.mlp_loss_and_grads(p, x, t)
    rng = np.random.default_rng(2)
    for k in ("W1", "b1", "W2", "b2", "W3", "b3"):
        for _ in range(4):
            i = tuple(rng.integers(0, n) for n in p[k].shape)
            h = 1e-6
            pp = {kk: vv.copy() for kk, vv in p.items()}
            pm = {kk: vv.copy() for kk, vv in p.items()}
            pp[k][i] += h
            pm[k][i] -= h
            fd = (oracle.mlp_loss_and_grads(pp, x, t)[0] - oracle.mlp_loss_and_grads(pm, x, t)[0]) / (2 * h)
            assert abs(fd - g[k][i]) <= 1e-6 * max(1.0, abs(fd)), (k, i, fd, g[k][i])


def test_loss_of_a_known_case(oracle):
    """zero weights: out = b3 = (d, s); loss = 0.5 exp(-s)(d - t)^2 + 0.5 s"""
    p, x, t = _small(3)
    p = {k: np.zeros_like(v) for k, v in p.items()}
    p["b3"] = np.array([0.2, 0.5])
    loss, _ = oracle.mlp_loss_and_grads(p, x, t)
    want = np.mean(0.5 * np.exp(-0.5) * (0.2 - t) ** 2 + 0.25)
    assert abs(loss - want) < 1e-12


def test_fallback_gate_choice():
    """The validation rule of the fallback gate: corrections that help where
    the network is confident and hurt where it is not are kept only below a
    log-variance quantile; a network that helps everywhere keeps them all."""
    import torch
    from tile_processor_gpu_b200 import disparity_net as D
    g = torch.Generator().manual_seed(3)
    n = 20000
    truth = torch.randn(n, generator=g) * 0.3
    plain = truth + torch.randn(n, generator=g) * 0.2
    logvar = torch.rand(n, generator=g) * 4 - 2
    good = truth + torch.randn(n, generator=g) * 0.05
    bad = truth + torch.randn(n, generator=g) * 0.8
    rho = torch.where(logvar < 1.0, good, bad)           # the top quarter of logvar is harmful
    gate, table = D.choose_gate(rho, logvar, plain, truth)
    assert 0.5 < gate <= 1.2, gate
    assert D.accuracy(D.gated(rho, logvar, plain, gate), truth)["rmse_px"] < D.accuracy(rho, truth)["rmse_px"]
    gate2, _ = D.choose_gate(good, logvar, plain, truth)
    assert gate2 == float("inf")


def test_gate_saved_with_the_weights(tmp_path):
    from tile_processor_gpu_b200 import disparity_net as D
    net = D.DisparityMLP(device="cpu", seed=4)
    net.gate = 0.75
    net.save(str(tmp_path / "n.npz"))
    back = D.DisparityMLP.load(str(tmp_path / "n.npz"), device="cpu")
    assert back.gate == 0.75
    assert all(np.array_equal(back.p[k].numpy(), np.float16(net.p[k].numpy()).astype(np.float32) if k.startswith("W")
                              else net.p[k].numpy()) for k in D.PARAMS)
    net.gate = float("inf")
    net.save(str(tmp_path / "m.npz"))
    assert D.DisparityMLP.load(str(tmp_path / "m.npz"), device="cpu").gate == float("inf")
