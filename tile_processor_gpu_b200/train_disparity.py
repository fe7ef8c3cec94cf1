"""Train the learned disparity residual on synthetic scenes of known disparity.

    python -m tile_processor_gpu_b200.train_disparity --frames 200 --holdout 8 \
        --out tile_processor_gpu_b200/data/disparity_mlp.npz

Each frame is a seeded slanted textured plane (disparity from 0 to 8..64 px
across the frame, shot and read noise) seen through one of eight lenses
(kernel tables of 256 PSF shapes each), whose tiles are tasked at the true
disparity plus a per-tile error U[-e, e] px, e drawn per frame in [0.3, 1.2].
The library's own pipeline (forward CLT, pair correlation, plain fit,
features) turns each frame into samples; the network
is trained with its own kernels (disparity_net) and evaluated on held-out
seeds against the plain fit, with both the FP32 and the tensor-core inference.
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


def _frame_draws(seed):
    """per-frame disparity span, task error and lens index"""
    r = np.random.default_rng(seed + 7_000_001)
    return float(r.uniform(8.0, 64.0)), float(r.uniform(0.3, 1.2)), int(r.integers(0, N_LENSES))


N_LENSES = 8


def _render(args):
    seed, width, height = args
    from tile_processor_gpu_b200 import synth
    span, _, _ = _frame_draws(seed)
    rng = np.random.default_rng(seed)
    imgs, disp = synth.plane_scene(rng, width, height, disparity=(0.0, span), texture="detail")
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
    import torch
    feats, plains, truths = [], [], []
    with mp.get_context("spawn").Pool(workers) as pool:
        for seed, imgs, disp in pool.imap(_render, [(s, width, height) for s in seeds]):
            _, err, li = _frame_draws(seed)
            f, p, t = samples_from_scene(seed, imgs, disp, lenses[li], width, height, error=err)
            feats.append(f)
            plains.append(p)
            truths.append(t)
    return torch.cat(feats), torch.cat(plains), torch.cat(truths)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--frames", type=int, default=200)
    ap.add_argument("--holdout", type=int, default=8)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--width", type=int, default=W_DEF)
    ap.add_argument("--height", type=int, default=H_DEF)
    ap.add_argument("--workers", type=int, default=max(1, min(16, (os.cpu_count() or 2) - 1)))
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                                                  "disparity_mlp.npz"))
    args = ap.parse_args(argv)
    import torch
    from tile_processor_gpu_b200 import build, disparity_net as D
    build.build()
    t0 = time.time()
    lenses = [make_lens(args.width, args.height, seed=100 + i) for i in range(N_LENSES)]
    train_seeds = list(range(10_000, 10_000 + args.frames))
    hold_seeds = list(range(90_000, 90_000 + args.holdout))
    feats, plain, truth = build_set(train_seeds, args.width, args.height, lenses, args.workers)
    hf, hp, ht = build_set(hold_seeds, args.width, args.height, lenses, args.workers)
    t1 = time.time()
    net = D.DisparityMLP(seed=1)
    log = lambda ep, loss: print("epoch %d loss %.5f" % (ep, loss), file=sys.stderr, flush=True)
    D.train(net, feats, plain, truth, epochs=args.epochs, batch=args.batch, lr=args.lr, log=log)
    torch.cuda.synchronize()
    t2 = time.time()
    rho, logvar = D.predict(net, hf, hp)
    net.pack()
    out_tc = torch.empty((hf.shape[0], 2), dtype=torch.float32, device=hf.device)
    net.infer_tc(D.pad_rows(hf), hf.shape[0], out_tc)
    torch.cuda.synchronize()
    report = {"train_tiles": int(feats.shape[0]), "holdout_tiles": int(hf.shape[0]), "frames": args.frames,
              "holdout_frames": args.holdout, "epochs": args.epochs, "frame": "%dx%d" % (args.width, args.height),
              "lenses": N_LENSES, "disparity_span_px": [8, 64], "task_error_px": [0.3, 1.2],
              "plain": D.accuracy(hp, ht), "learned_fp32": D.accuracy(rho, ht),
              "learned_tensor_core": D.accuracy(hp + out_tc[:, 0], ht),
              "seconds": {"data": round(t1 - t0, 1), "train": round(t2 - t1, 1)}}
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    net.save(args.out)
    with open(os.path.splitext(args.out)[0] + ".json", "w") as fh:
        json.dump(report, fh, indent=1)
    print(json.dumps(report))


if __name__ == "__main__":
    main()
