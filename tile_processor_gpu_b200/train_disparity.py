"""Train the learned disparity residual on synthetic scenes of known disparity.

    python -m tile_processor_gpu_b200.train_disparity --frames 800 --holdout 24 \
        --out tile_processor_gpu_b200/data/disparity_mlp.npz

Each frame is a seeded slanted textured plane, or (a third of the frames)
two planes with an occlusion edge, disparity from 0 to 8..64 px across the
frame, shot noise and a read-noise sigma drawn log-uniformly in
[0.001, 0.02], seen through one of eight lenses (kernel tables of 256 PSF
shapes each); its tiles are tasked at the true disparity plus a per-tile
error U[-e, e] px, e drawn per frame in [0.3, 1.2] (--task-error,
--log-error).  The library's own
pipeline (forward CLT, pair correlation, plain fit, features) turns each
frame into samples; the network is trained with its own kernels
(disparity_net).  Eight validation frames choose the log-variance gate above
which the plain fit is kept (the fallback); held-out frames then compare the
plain fit, the network and the gated network, overall and per scene kind,
with both the FP32 and the tensor-core inference.
Scene rendering runs in spawned worker processes (NumPy only).
"""
import argparse
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

W_DEF, H_DEF = 1024, 768


# per-frame task-error bound e (px): uniform in [lo, hi], or log-uniform
TASK_ERROR = {"lo": 0.3, "hi": 1.2, "log": False}


def _frame_draws(seed):
    """per-frame disparity span, task error, lens index, scene kind (a third
    of the frames have an occlusion edge) and read-noise sigma (log-uniform)"""
    r = np.random.default_rng(seed + 7_000_001)
    span = float(r.uniform(8.0, 64.0))
    lo, hi = TASK_ERROR["lo"], TASK_ERROR["hi"]
    e = float(np.exp(r.uniform(np.log(lo), np.log(hi)))) if TASK_ERROR["log"] else float(r.uniform(lo, hi))
    return (span, e, int(r.integers(0, N_LENSES)),
            "occlusion" if r.uniform() < OCCLUSION_FRACTION else "plane",
            float(np.exp(r.uniform(np.log(0.001), np.log(0.02)))))


OCCLUSION_FRACTION = 1.0 / 3.0


N_LENSES = 8


def _render(args):
    seed, width, height = args
    from tile_processor_gpu_b200 import synth
    span, _, _, kind, sigma = _frame_draws(seed)
    rng = np.random.default_rng(seed)
    scene = synth.occlusion_scene if kind == "occlusion" else synth.plane_scene
    imgs, disp = scene(rng, width, height, disparity=(0.0, span), texture="detail", read_sigma=sigma)
    return seed, imgs, disp


def samples_from_scene(seed, imgs, disp, lens, width, height, error=1.0, margin=5, device="cuda"):
    """features, plain residual, true residual (device tensors) of one scene"""
    import torch
    from tile_processor_gpu_b200 import api, synth, disparity_net as D
    geom = synth.geometry(width, height, image_rows=height + 16)
    g = api.Geometry.from_dict(geom)
    rng = np.random.default_rng(seed + 1_000_003)
    tasks_np, err = synth.tasks_grid(geom, rng, jitter=0.0, disparity=disp, disparity_error=error,
                                     return_error=True)
    TX, TY, _ = synth.tiles(geom)
    dstride = width + 64
    pitched = np.zeros((4, height + 16, dstride), np.float32)
    pitched[:, :height, :width] = imgs
    images = [torch.from_numpy(pitched[c]).to(device) for c in range(4)]
    clt = [torch.empty(TY * TX * 768, dtype=torch.float32, device=device) for _ in range(4)]
    P = api.PointerArray
    pi, pc = P(images), P(clt)
    tasks = api.tasks_to_device(tasks_np, device)
    api.convert_correct_tiles(g, lens["p_extra"], lens["p_kernels"], pi, tasks, pc, dstride, tasks_np.size, 0)
    idx_np = synth.corr_indices_fast(tasks_np, geom)
    idx = torch.from_numpy(idx_np).to(device)
    corrs = torch.empty((idx_np.size, 225), dtype=torch.float32, device=device)
    api.correlate2D(g, pc, 3, .25, .25, .5, 0.05, idx_np.size, idx, 225, 7, corrs)
    dd = torch.zeros(TX * TY, dtype=torch.float32, device=device)
    ss = torch.zeros(TX * TY, dtype=torch.float32, device=device)
    api.disparity_fit(g, corrs, 225, 7, idx_np.size, idx, lens["port_offsets"], dd, ss)
    feat = torch.zeros((TX * TY, D.N_IN), dtype=torch.float32, device=device)
    D.features(g, corrs, 225, 7, idx_np.size, idx, feat)
    tx, ty = tasks_np["txy"] & 0xFFFF, tasks_np["txy"] >> 16
    inner = (tx >= margin) & (tx < TX - margin) & (ty >= margin) & (ty < TY - margin)
    tiles = torch.from_numpy((ty * TX + tx)[inner].astype(np.int64)).to(device)
    truth = torch.from_numpy((-err[inner]).astype(np.float32)).to(device)
    return feat[tiles].contiguous(), dd[tiles].contiguous(), truth


def make_lens(width, height, seed=7, device="cuda"):
    import torch
    from tile_processor_gpu_b200 import api, synth
    geom = synth.geometry(width, height, image_rows=height + 16)
    kern, extra = synth.kernel_tables(np.random.default_rng(seed), geom, pool=256, zero_extra=True, psf_offset=0.0)
    kernels = [torch.from_numpy(kern[c]).to(device) for c in range(4)]
    extras = [torch.from_numpy(extra[c]).to(device) for c in range(4)]
    return {"kernels": kernels, "extras": extras, "p_kernels": api.PointerArray(kernels),
            "p_extra": api.PointerArray(extras),
            "port_offsets": torch.from_numpy(synth.PORT_OFFSETS.reshape(-1).copy()).to(device)}


def build_set(seeds, width, height, lenses, workers):
    """features, plain residual, true residual and scene kind (1 = occlusion) per sample"""
    import torch
    feats, plains, truths, kinds = [], [], [], []
    with mp.get_context("spawn").Pool(workers) as pool:
        for seed, imgs, disp in pool.imap(_render, [(s, width, height) for s in seeds]):
            _, err, li, kind, _ = _frame_draws(seed)
            f, p, t = samples_from_scene(seed, imgs, disp, lenses[li], width, height, error=err)
            feats.append(f)
            plains.append(p)
            truths.append(t)
            kinds.append(torch.full_like(t, 1.0 if kind == "occlusion" else 0.0))
    return torch.cat(feats), torch.cat(plains), torch.cat(truths), torch.cat(kinds)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--frames", type=int, default=800)
    ap.add_argument("--holdout", type=int, default=24)
    ap.add_argument("--validation", type=int, default=8, help="frames that choose the fallback gate")
    ap.add_argument("--epochs", type=int, default=14)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--width", type=int, default=W_DEF)
    ap.add_argument("--height", type=int, default=H_DEF)
    ap.add_argument("--workers", type=int, default=max(1, min(16, (os.cpu_count() or 2) - 1)))
    ap.add_argument("--task-error", default="0.3,1.2", help="per-frame task-error bound range lo,hi (px)")
    ap.add_argument("--log-error", action="store_true", help="draw the bound log-uniformly in the range")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                                                  "disparity_mlp.npz"))
    args = ap.parse_args(argv)
    lo, hi = (float(v) for v in args.task_error.split(","))
    TASK_ERROR.update(lo=lo, hi=hi, log=bool(args.log_error))
    import torch
    from tile_processor_gpu_b200 import build, disparity_net as D
    build.build()
    t0 = time.time()
    lenses = [make_lens(args.width, args.height, seed=100 + i) for i in range(N_LENSES)]
    train_seeds = list(range(10_000, 10_000 + args.frames))
    hold_seeds = list(range(90_000, 90_000 + args.holdout))
    val_seeds = list(range(80_000, 80_000 + args.validation))
    feats, plain, truth, _ = build_set(train_seeds, args.width, args.height, lenses, args.workers)
    hf, hp, ht, hk = build_set(hold_seeds, args.width, args.height, lenses, args.workers)
    vf, vp, vt, _ = build_set(val_seeds, args.width, args.height, lenses, args.workers)
    t1 = time.time()
    net = D.DisparityMLP(seed=1)
    log = lambda ep, loss: print("epoch %d loss %.5f" % (ep, loss), file=sys.stderr, flush=True)
    D.train(net, feats, plain, truth, epochs=args.epochs, batch=args.batch, lr=args.lr, log=log)
    torch.cuda.synchronize()
    t2 = time.time()
    # the plain fit as fallback: a log-variance gate chosen on the validation frames
    vrho, vlogvar = D.predict(net, vf, vp)
    net.gate, gate_table = D.choose_gate(vrho, vlogvar, vp, vt)
    del vf
    rho, logvar = D.predict(net, hf, hp)
    rho_g = D.gated(rho, logvar, hp, net.gate)
    net.pack()
    out_tc = torch.empty((hf.shape[0], 2), dtype=torch.float32, device=hf.device)
    net.infer_tc(D.pad_rows(hf), hf.shape[0], out_tc)
    torch.cuda.synchronize()
    fin = lambda v: v if np.isfinite(v) else None  # noqa: E731  (no gate: null)
    report = {"train_tiles": int(feats.shape[0]), "holdout_tiles": int(hf.shape[0]), "frames": args.frames,
              "holdout_frames": args.holdout, "epochs": args.epochs, "frame": "%dx%d" % (args.width, args.height),
              "lenses": N_LENSES, "disparity_span_px": [8, 64], "task_error_px": [lo, hi],
              "task_error_draw": "log-uniform" if args.log_error else "uniform",
              "scenes": "slanted planes; a third two planes with an occlusion edge",
              "read_sigma": "log-uniform in [0.001, 0.02]",
              "validation_frames": args.validation, "gate_logvar": fin(net.gate),
              "gate_table": [{"gate": fin(g), "rmse_px": r, "outliers_gt_0.5px": o} for g, r, o in gate_table],
              "plain": D.accuracy(hp, ht), "learned_fp32": D.accuracy(rho, ht),
              "learned_gated": D.accuracy(rho_g, ht),
              "learned_tensor_core": D.accuracy(hp + out_tc[:, 0], ht),
              "by_scene": {name: {"tiles": int(m.sum().item()), "plain": D.accuracy(hp[m], ht[m]),
                                  "learned": D.accuracy(rho[m], ht[m]), "learned_gated": D.accuracy(rho_g[m], ht[m])}
                           for name, m in (("plane", hk == 0), ("occlusion", hk == 1)) if int(m.sum().item())},
              "seconds": {"data": round(t1 - t0, 1), "train": round(t2 - t1, 1)}}
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    net.save(args.out)
    with open(os.path.splitext(args.out)[0] + ".json", "w") as fh:
        json.dump(report, fh, indent=1)
    print(json.dumps(report))


if __name__ == "__main__":
    main()
