"""The learned disparity residual: a small MLP on the six correlation planes
of a tile that corrects the plain fit (tp_disparity_fit) and states its
confidence.  Every operation runs in the library's own kernels (tp_mlp_*);
torch tensors only hold device memory.

    x  = the tile's six (2r+1)^2 planes / their largest magnitude   (tp_mlp_features)
    h1 = gelu(x W1 + b1)        1350 -> 256                         (tp_mlp_gemm)
    h2 = gelu(h1 W2 + b2)        256 -> 128
    [d, s] = h2 W3 + b3          128 -> 2
    rho = plain + d, variance exp(s); trained on the Gaussian negative
    log-likelihood (tp_mlp_nll) with Adam (tp_mlp_adam).

The reference has no counterpart (its absent Java caller fits disparity);
training data come from the library's own pipeline on synthetic scenes of
known disparity (`make_samples`).
"""
import ctypes

import numpy as np

from . import _native
from .api import _dptr, _stream

N_IN, N_H1, N_H2, N_OUT = 1350, 256, 128, 2
TC_KPAD = 1376  # layer-1 K of the tensor-core path (1350 padded to 43 blocks of 32)
TC_LDX = 1352  # feature rows on 16-byte boundaries, as the tensor-core inference needs
PARAMS = ("W1", "b1", "W2", "b2", "W3", "b3")
SHAPES = {"W1": (N_IN, N_H1), "b1": (N_H1,), "W2": (N_H1, N_H2), "b2": (N_H2,), "W3": (N_H2, N_OUT),
          "b3": (N_OUT,)}


def _t():
    import torch
    return torch


def init_params(seed=0):
    """He-scaled normal weights, zero biases (host float32)."""
    rng = np.random.default_rng(seed)
    p = {}
    for name in PARAMS:
        shape = SHAPES[name]
        if name.startswith("W"):
            p[name] = (rng.standard_normal(shape) * np.sqrt(2.0 / shape[0])).astype(np.float32)
        else:
            p[name] = np.zeros(shape, np.float32)
    p["W3"] *= 0.1
    return p


def gemm(A, B, C, M, N, K, ta=0, tb=0, beta=0.0, bias=None, z=None, lda=None, ldb=None, ldc=None, ldz=None,
         stream=None, tc=False, err=None):
    """C = beta C + op(A) op(B) (+ bias; with z, z = that and C = gelu(z)):
    tp_mlp_gemm_tc (split-TF32 tensor-core MMAs; err: device int32 set to 1
    if a wait ran out) when tc, else tp_mlp_gemm (FP32 SIMT)."""
    lda = lda if lda is not None else (M if ta else K)
    ldb = ldb if ldb is not None else (K if tb else N)
    ldc = ldc if ldc is not None else N
    ldz = ldz if ldz is not None else N
    args = [int(M), int(N), int(K), _dptr(A), int(lda), int(ta), _dptr(B), int(ldb), int(tb), float(beta), _dptr(C),
            int(ldc), _dptr(bias) if bias is not None else None, _dptr(z) if z is not None else None, int(ldz)]
    if tc:
        _native.call("tp_mlp_gemm_tc", *args, _dptr(err) if err is not None else None, _stream(stream))
    else:
        _native.call("tp_mlp_gemm", *args, _stream(stream))


def features(geom, corrs, corr_stride, corr_radius, num_corr, corr_indices, out, feature_stride=N_IN,
             stream=None):
    """Rows out[tile] of the tiles with correlation entries (others untouched)."""
    _native.call("tp_mlp_features", geom.ptr, _dptr(corrs), int(corr_stride), int(corr_radius), int(num_corr),
                 _dptr(corr_indices), _dptr(out), int(feature_stride), _stream(stream))


def pad_rows(x, ldx=TC_LDX):
    """Copy of feature rows x [rows][>= 1350] with leading dimension ldx
    (zeros past column 1349), for the tensor-core inference."""
    torch = _t()
    out = torch.zeros((x.shape[0], ldx), dtype=torch.float32, device=x.device)
    out[:, :N_IN] = x[:, :N_IN]
    return out


class DisparityMLP:
    """Weights, Adam state and the forward / backward passes on the GPU."""

    def __init__(self, params=None, device="cuda", seed=0, tc=True):
        torch = _t()
        host = params if params is not None else init_params(seed)
        self.p = {k: torch.from_numpy(np.ascontiguousarray(host[k], np.float32)).to(device) for k in PARAMS}
        # the forward and backward GEMMs on the tensor cores (tp_mlp_gemm_tc)
        # or as FP32 SIMT (tp_mlp_gemm); _err is the tensor-core GEMM's flag
        self.tc = tc
        self._err = torch.zeros(1, dtype=torch.int32, device=device) if device != "cpu" else None
        self.g = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.m = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.step_count = 0
        self.device = device
        self._ws = {}

    def _work(self, rows):
        torch = _t()
        if self._ws.get("rows", 0) < rows:
            f = lambda n: torch.empty((rows, n), dtype=torch.float32, device=self.device)
            self._ws = {"rows": rows, "z1": f(N_H1), "h1": f(N_H1), "z2": f(N_H2), "h2": f(N_H2), "out": f(N_OUT),
                        "dout": f(N_OUT), "dh2": f(N_H2), "dz2": f(N_H2), "dh1": f(N_H1), "dz1": f(N_H1),
                        "loss": torch.empty(rows, dtype=torch.float32, device=self.device)}
        return self._ws

    def forward(self, x, rows, ldx=N_IN, stream=None):
        """out [rows][2] = (d, s) for feature rows x (leading dimension ldx);
        keeps the activations for backward."""
        w = self._work(rows)
        p = self.p
        gemm(x, p["W1"], w["h1"], rows, N_H1, N_IN, bias=p["b1"], z=w["z1"], lda=ldx,
             stream=stream, tc=self.tc, err=self._err)
        gemm(w["h1"], p["W2"], w["h2"], rows, N_H2, N_H1, bias=p["b2"], z=w["z2"],
             stream=stream, tc=self.tc, err=self._err)
        gemm(w["h2"], p["W3"], w["out"], rows, N_OUT, N_H2, bias=p["b3"],
             stream=stream, tc=self.tc, err=self._err)
        return w["out"][:rows]

    def loss_backward(self, x, rows, target, weight=None, ldx=N_IN, stream=None):
        """Gradients of the mean NLL over rows with weight 1 (forward must
        have run on the same x); returns the mean loss (host float)."""
        w = self._work(rows)
        p, g = self.p, self.g
        count = float(weight[:rows].sum().item()) if weight is not None else float(rows)
        _native.call("tp_mlp_nll", int(rows), _dptr(w["out"]), _dptr(target),
                     _dptr(weight) if weight is not None else None, 1.0 / max(count, 1.0), _dptr(w["dout"]),
                     _dptr(w["loss"]), _stream(stream))
        # layer 3
        gemm(w["h2"], w["dout"], g["W3"], N_H2, N_OUT, rows, ta=1, lda=N_H2,
             stream=stream, tc=self.tc, err=self._err)
        _native.call("tp_mlp_colsum", int(rows), N_OUT, N_OUT, _dptr(w["dout"]), 1.0, _dptr(g["b3"]),
                     _stream(stream))
        gemm(w["dout"], p["W3"], w["dh2"], rows, N_H2, N_OUT, tb=1, ldb=N_OUT,
             stream=stream, tc=self.tc, err=self._err)
        _native.call("tp_mlp_gelu_backward", int(rows), N_H2, N_H2, _dptr(w["z2"]), _dptr(w["dh2"]), _dptr(w["dz2"]),
                     _stream(stream))
        # layer 2
        gemm(w["h1"], w["dz2"], g["W2"], N_H1, N_H2, rows, ta=1, lda=N_H1,
             stream=stream, tc=self.tc, err=self._err)
        _native.call("tp_mlp_colsum", int(rows), N_H2, N_H2, _dptr(w["dz2"]), 1.0, _dptr(g["b2"]), _stream(stream))
        gemm(w["dz2"], p["W2"], w["dh1"], rows, N_H1, N_H2, tb=1, ldb=N_H2,
             stream=stream, tc=self.tc, err=self._err)
        _native.call("tp_mlp_gelu_backward", int(rows), N_H1, N_H1, _dptr(w["z1"]), _dptr(w["dh1"]), _dptr(w["dz1"]),
                     _stream(stream))
        # layer 1
        gemm(x, w["dz1"], g["W1"], N_IN, N_H1, rows, ta=1, lda=ldx,
             stream=stream, tc=self.tc, err=self._err)
        _native.call("tp_mlp_colsum", int(rows), N_H1, N_H1, _dptr(w["dz1"]), 1.0, _dptr(g["b1"]), _stream(stream))
        return float(w["loss"][:rows].sum().item()) / max(count, 1.0)

    def check(self):
        """Raise if a tensor-core GEMM of this network reported a wait that ran
        out (its flag is cleared for the next step)."""
        if self._err is not None and int(self._err.item()):
            self._err.zero_()
            raise RuntimeError("tp_mlp_gemm_tc: a wait for the tensor cores ran out")

    def adam_step(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, stream=None):
        self.step_count += 1
        for k in PARAMS:
            _native.call("tp_mlp_adam", int(self.p[k].numel()), _dptr(self.p[k]), _dptr(self.g[k]),
                         _dptr(self.m[k]), _dptr(self.v[k]), float(lr), float(beta1), float(beta2), float(eps),
                         int(self.step_count), _stream(stream))

    def pack(self, stream=None):
        """W1^T in TF32 and W2^T in BF16 for the tensor-core inference (after any update)."""
        torch = _t()
        if not hasattr(self, "w1t"):
            self.w1t = torch.empty((N_H1, TC_KPAD), dtype=torch.float32, device=self.device)
            self.w2t = torch.empty((N_H2, N_H1), dtype=torch.bfloat16, device=self.device)
            self.tc_err = torch.zeros(1, dtype=torch.int32, device=self.device)
        _native.call("tp_mlp_pack", _dptr(self.p["W1"]), _dptr(self.p["W2"]), _dptr(self.w1t), _dptr(self.w2t),
                     _stream(stream))

    def infer_tc(self, x, rows, out, ldx=TC_LDX, stream=None):
        """out [rows][2] = (d, s) with layers 1-2 on the tensor cores (TF32 and
        BF16 operands, FP32 accumulation); pack() must have run since the last
        update.  Rows of x must start on 16-byte boundaries (ldx a multiple of
        4): see pad_rows."""
        p = self.p
        _native.call("tp_mlp_infer_tc", int(rows), _dptr(x), int(ldx), _dptr(self.w1t), _dptr(p["b1"]),
                     _dptr(self.w2t), _dptr(p["b2"]), _dptr(p["W3"]), _dptr(p["b3"]), _dptr(out), _dptr(self.tc_err),
                     _stream(stream))
        return out

    def host_params(self):
        return {k: v.cpu().numpy().copy() for k, v in self.p.items()}

    # log-variance above which the plain fit is kept (combine); +inf keeps every correction
    gate = float("inf")

    def combine(self, plain, out, rows, rho, stream=None):
        """rho = plain + d where the log-variance s < self.gate, else plain (tp_mlp_combine)."""
        _native.call("tp_mlp_combine", int(rows), _dptr(plain), _dptr(out), float(self.gate), _dptr(rho),
                     _stream(stream))
        return rho

    def save(self, path):
        arrays = {k: v.astype(np.float16 if k.startswith("W") else np.float32) for k, v in self.host_params().items()}
        arrays["gate"] = np.array(self.gate, np.float32)
        np.savez_compressed(path, **arrays)

    @classmethod
    def load(cls, path, device="cuda"):
        d = np.load(path)
        net = cls({k: d[k].astype(np.float32) for k in PARAMS}, device=device)
        if "gate" in d.files:
            net.gate = float(d["gate"])
        return net


# --------------------------------------------------------------------------- #
# training data from the library's own pipeline
# --------------------------------------------------------------------------- #
def make_samples(seed, width=1024, height=768, disparity=(0.0, 32.0), error=1.0, margin=5, device="cuda", pool=64):
    """One synthetic plane-scene frame through convert, correlate and the plain
    fit.  Returns (features [n][1350], plain residual [n], true residual [n])
    as device tensors for the interior tiles (`margin` tiles from the edges,
    where every camera's footprint stays inside the frame).  pool: PSF
    shapes of the frame's kernel tables."""
    torch = _t()
    from . import api, synth
    rng = np.random.default_rng(seed)
    geom = synth.geometry(width, height, image_rows=height + 16)
    g = api.Geometry.from_dict(geom)
    imgs, disp = synth.plane_scene(rng, width, height, disparity=disparity, texture="detail")
    dstride = width + 64
    pitched = np.zeros((4, height + 16, dstride), np.float32)
    pitched[:, :height, :width] = imgs
    kern, extra = synth.kernel_tables(rng, geom, pool=pool, zero_extra=True, psf_offset=0.0)
    tasks_np, err = synth.tasks_grid(geom, rng, jitter=0.0, disparity=disp, disparity_error=error,
                                     return_error=True)
    TX, TY, _ = synth.tiles(geom)
    images = [torch.from_numpy(pitched[c]).to(device) for c in range(4)]
    kernels = [torch.from_numpy(kern[c]).to(device) for c in range(4)]
    extras = [torch.from_numpy(extra[c]).to(device) for c in range(4)]
    clt = [torch.empty(TY * TX * 768, dtype=torch.float32, device=device) for _ in range(4)]
    P = api.PointerArray
    pi, pk, pe, pc = P(images), P(kernels), P(extras), P(clt)
    tasks = api.tasks_to_device(tasks_np, device)
    api.convert_correct_tiles(g, pe, pk, pi, tasks, pc, dstride, tasks_np.size, 0)
    idx_np = synth.corr_indices_fast(tasks_np, geom)
    idx = torch.from_numpy(idx_np).to(device)
    corrs = torch.empty((idx_np.size, 225), dtype=torch.float32, device=device)
    api.correlate2D(g, pc, 3, .25, .25, .5, 0.05, idx_np.size, idx, 225, 7, corrs)
    po = torch.from_numpy(synth.PORT_OFFSETS.reshape(-1).copy()).to(device)
    dd = torch.zeros(TX * TY, dtype=torch.float32, device=device)
    ss = torch.zeros(TX * TY, dtype=torch.float32, device=device)
    api.disparity_fit(g, corrs, 225, 7, idx_np.size, idx, po, dd, ss)
    feat = torch.zeros((TX * TY, N_IN), dtype=torch.float32, device=device)
    features(g, corrs, 225, 7, idx_np.size, idx, feat)
    tx, ty = tasks_np["txy"] & 0xFFFF, tasks_np["txy"] >> 16
    inner = (tx >= margin) & (tx < TX - margin) & (ty >= margin) & (ty < TY - margin)
    tiles = torch.from_numpy((ty * TX + tx)[inner].astype(np.int64)).to(device)
    truth = torch.from_numpy((-err[inner]).astype(np.float32)).to(device)
    return feat[tiles].contiguous(), dd[tiles].contiguous(), truth


def train(net, feats, plain, truth, epochs=4, batch=4096, lr=1e-3, seed=0, log=None):
    """Minibatch Adam on the NLL of the residual truth - plain."""
    torch = _t()
    n = feats.shape[0]
    target = (truth - plain).contiguous()
    gen = torch.Generator(device="cpu").manual_seed(seed)
    for ep in range(epochs):
        order = torch.randperm(n, generator=gen).to(feats.device)
        total, nb = 0.0, 0
        for b0 in range(0, n - batch + 1, batch):
            sel = order[b0:b0 + batch]
            xb = feats[sel].contiguous()
            tb = target[sel].contiguous()
            net.forward(xb, batch)
            total += net.loss_backward(xb, batch, tb)
            net.adam_step(lr=lr)
            nb += 1
        net.check()
        if log is not None:
            log(ep, total / max(nb, 1))
    return net


def gated(rho, logvar, plain, gate):
    """The estimate with the plain fit kept where logvar >= gate (evaluation
    helper on device tensors; tp_mlp_combine is the library form)."""
    torch = _t()
    return torch.where(logvar < gate, rho, plain)


GATE_QUANTILES = (0.5, 0.6, 0.7, 0.8, 0.85, 0.9, 0.95, 0.97, 0.98, 0.99, 0.995, 0.998, 0.999)


def choose_gate(rho, logvar, plain, truth, quantiles=GATE_QUANTILES):
    """Pick the log-variance gate on validation samples: among +inf and the
    given quantiles of logvar, the one with the fewest > 0.5 px errors whose
    RMS error stays within 0.5% of the best RMS error.  Returns (gate, table)."""
    torch = _t()
    cands = [float("inf")] + [float(torch.quantile(logvar.float().cpu(), q)) for q in quantiles]
    table = []
    for g in cands:
        a = accuracy(gated(rho, logvar, plain, g), truth)
        table.append((g, a["rmse_px"], a["outliers_gt_0.5px"]))
    best_rmse = min(t[1] for t in table)
    ok = [t for t in table if t[1] <= best_rmse * 1.005]
    gate = min(ok, key=lambda t: (t[2], t[1]))[0]
    return gate, table


def predict(net, feats, plain, batch=16384):
    """rho = plain + d and the log-variance s for every row."""
    torch = _t()
    n = feats.shape[0]
    rho = torch.empty(n, dtype=torch.float32, device=feats.device)
    logvar = torch.empty(n, dtype=torch.float32, device=feats.device)
    for b0 in range(0, n, batch):
        rows = min(batch, n - b0)
        out = net.forward(feats[b0:b0 + rows].contiguous(), rows)
        rho[b0:b0 + rows] = plain[b0:b0 + rows] + out[:, 0]
        logvar[b0:b0 + rows] = out[:, 1]
    return rho, logvar


def accuracy(est, truth):
    e = (est - truth).double()
    return {"rmse_px": float(e.pow(2).mean().sqrt().item()), "outliers_gt_0.5px": float((e.abs() > 0.5).double().mean().item())}
