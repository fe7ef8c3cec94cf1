"""Two more workload shapes, checked against the FP64 oracle.

Precision: per stage, the largest and the RMS error of the CLT coefficients,
the correlation tiles and the texture colours (stable pixels) relative to the
oracle, on an ordinary scene and a high-dynamic-range one (values up to 1e4).

Batched: frames of uneven sizes with sparse, blob-shaped task lists (activity
5% to 100%) through the same calls back to back, each frame checked against
the oracle, then the whole batch captured once in a CUDA graph and replayed,
which must reproduce the eager outputs exactly."""
import json

import numpy as np
import pytest

from cases import Case, blob_mask, rel_err, rms_err

pytestmark = pytest.mark.gpu


def _stage_errors(oracle, c):
    import gpu_runner as R
    import conditioning
    fr = R.Frame(c)
    b = R.convert(fr)
    o = oracle.convert_correct_tiles(c.geom, c.extra, c.kernels, c.pitched, c.dstride, c.tasks)
    out = {"clt_max": max(rel_err(b[k], o[k]) for k in range(4)),
           "clt_rms": max(rms_err(b[k], o[k]) for k in range(4))}
    o64 = [x.astype(np.float64) for x in b]
    fr.set_clt(b)
    cb = R.correlate(fr, c.corr_idx, stride=225)
    co = oracle.correlate2D(c.geom, o64, 3, .25, .25, .5, 0.05, c.corr_idx, 225, 7)
    out["corr_max"], out["corr_rms"] = rel_err(cb, co), rms_err(cb, co)
    tb = R.textures_tiles(fr, c.tex_idx)
    bad, to = conditioning.unstable_mask(oracle, c, o64, c.tex_idx, 0)
    col = tb[:, :3]
    keep = ~bad[:, :3]
    den = np.abs(to[:, :3]).max()
    err = np.abs(col - to[:, :3])[keep] / den
    out["texture_max"] = float(err.max())
    out["texture_rms"] = float(np.sqrt(np.mean(err ** 2)))
    out["texture_stable_fraction"] = float(keep.mean())
    return out


@pytest.mark.parametrize("name,peak", [("ordinary", 1.0), ("hdr1e4", 1e4)])
def test_stage_errors_against_fp64(oracle, name, peak):
    c = Case(512, 384, seed=31, border_mode=0, scene="plane", peak=peak)
    e = _stage_errors(oracle, c)
    print("\nprecision %s %s" % (name, json.dumps({k: float("%.3g" % v) for k, v in e.items()})))
    assert e["clt_max"] < 1e-5 and e["corr_max"] < 1e-5
    assert e["clt_rms"] < 1e-6 and e["corr_rms"] < 1e-6
    assert e["texture_rms"] < 1e-6 and e["texture_stable_fraction"] > 0.99


SIZES = [(320, 240), (640, 480), (256, 256), (800, 600), (512, 384), (1024, 768)]


def _check_rgba(oracle, geom, tasks, TX, TY, clt, port_offsets, rgba, woi, what):
    """The overlapped RGBA image of one frame against the FP64 oracle's on the
    same CLT, on pixels all of whose tiles are stable (as in the small-frame
    parity tests); returns the per-slice record."""
    import conditioning
    from test_gpu_parity import assert_close_on
    stride = rgba.shape[1]
    o, _, _, _, woi_o = oracle.generate_RBGA(geom, tasks, TX, TY, clt, port_offsets, stride, rgba.shape[0] + 8)
    assert np.array_equal(woi, woi_o), what
    h, w = (woi[3] + 1) * 8, (woi[2] + 1) * 8
    txy = tasks["txy"].astype(np.int64)
    textured = (tasks["task"] & 0xF) != 0
    tiles = ((txy & 0xFFFF) + (txy >> 16) * TX)[textured]
    bad, _ = conditioning.unstable_tiles(oracle, geom, port_offsets, clt, tiles)
    codes = (tiles << 8).astype(np.int64)
    m = conditioning.unstable_image_mask(bad.any(axis=1), codes, woi, TX, (h, w), 4)
    assert m.mean() <= 0.01, (what, m.mean())
    b, r = rgba[:4 * h, :w], o[:4 * h, :w]
    assert_close_on(b, r, ~m, 1e-5, 4e-4)
    sl = lambda a: a.reshape(4, h, w)[None]
    return conditioning.stable_errors(sl(b), sl(r), sl(~m))


def _batch():
    rng = np.random.default_rng(77)
    cases = []
    for k, (w, h) in enumerate(SIZES):
        act = rng.uniform(0.05, 1.0)
        m = blob_mask(rng, w // 8, h // 8, act)
        cases.append(Case(w, h, seed=200 + k, border_mode=k & 1, mask=m, scene="plane" if k % 2 else None))
    return cases


def test_batched_uneven_sparse_frames(oracle):
    import torch
    import gpu_runner as R
    from tile_processor_gpu_b200 import api
    cases = _batch()
    frames = [R.Frame(c) for c in cases]
    stride = [(c.TX + 1) * 8 for c in cases]
    outs = []
    for c, fr, st in zip(cases, frames, stride):
        idx = torch.from_numpy(c.corr_idx).cuda()
        tasks = api.tasks_to_device(c.tasks, "cuda")
        corrs = torch.zeros((len(c.corr_idx), 225), device="cuda")
        rgba = torch.zeros(((c.TY + 1) * 8 * 4, st), device="cuda")
        lst = torch.zeros(c.TX * c.TYA, dtype=torch.int32, device="cuda")
        cnt = torch.zeros(8, dtype=torch.int32, device="cuda")
        woi = torch.zeros(4, dtype=torch.int32, device="cuda")
        outs.append(dict(idx=idx, tasks=tasks, corrs=corrs, rgba=rgba, lst=lst, cnt=cnt, woi=woi))

    def run_all():
        for c, fr, o, st in zip(cases, frames, outs, stride):
            api.convert_correct_tiles(fr.g, fr.p_extra, fr.p_kernels, fr.p_images, o["tasks"], fr.p_clt, c.dstride,
                                      c.num_tiles, 0)
            api.correlate2D(fr.g, fr.p_clt, 3, .25, .25, .5, 0.05, len(c.corr_idx), o["idx"], 225, 7, o["corrs"])
            api.generate_RBGA(fr.g, o["tasks"], c.num_tiles, o["lst"], o["cnt"], o["woi"], c.TX, c.TY, fr.p_clt,
                              fr.port_offsets, 3, 0, 10.0, 3.0, 1.5, 10.0, 3.0, 0.294118, 0.117647, 0.588235, 1, 0,
                              st, o["rgba"])

    run_all()
    torch.cuda.synchronize()
    for c, fr, o in zip(cases, frames, outs):
        clt = fr.clt_numpy()
        ref = oracle.convert_correct_tiles(c.geom, c.extra, c.kernels, c.pitched, c.dstride, c.tasks)
        assert max(rel_err(clt[k], ref[k]) for k in range(4)) < 1e-5, (c.W, c.H)
        co = oracle.correlate2D(c.geom, [x.astype(np.float64) for x in clt], 3, .25, .25, .5, 0.05, c.corr_idx,
                                225, 7)
        assert rel_err(o["corrs"].cpu().numpy(), co) < 1e-5, (c.W, c.H)
        _check_rgba(oracle, c.geom, c.tasks, c.TX, c.TY, clt, c.port_offsets, o["rgba"].cpu().numpy(),
                    o["woi"].cpu().numpy(), (c.W, c.H))
    eager = [(o["corrs"].clone(), o["rgba"].clone()) for o in outs]
    # the whole batch as one CUDA graph (the calls' first use on this device is above)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        with torch.cuda.graph(g, stream=side):
            run_all()
    torch.cuda.current_stream().wait_stream(side)
    for o in outs:
        o["corrs"].fill_(7.0)
        o["rgba"].zero_()  # outside the window of interest the buffers keep their first contents
    g.replay()
    torch.cuda.synchronize()
    for (ec, er), o in zip(eager, outs):
        assert torch.equal(ec, o["corrs"]) and torch.equal(er, o["rgba"])
    # per-frame latency over replays of the batch, printed for the record
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    reps = 20
    ev[0].record()
    for _ in range(reps):
        g.replay()
    ev[1].record()
    torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[1]) / reps
    print("\nbatch of %d uneven sparse frames: %.3f ms per batch, %.1f frames/s" % (len(cases), ms,
                                                                                    len(cases) / ms * 1e3))
    del g


def test_bench_batched_frames_vs_oracle(native, oracle):
    """Four of the bench's own 64 batched frames -- the smallest, the largest,
    the sparsest and the densest -- run through the three calls on the
    bench's shared buffers, each checked against the FP64 oracle: CLT and
    correlations within 1e-5, the overlapped RGBA image on stable pixels."""
    import os
    import sys
    import torch
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    pipe = bench.FramePipeline(seed=100, device="cuda:0")
    batch = bench.BatchedFrames(pipe, n=64, seed=11)
    fs = batch.frames
    area = [f["size"][0] * f["size"][1] for f in fs]
    act = [f["activity"] for f in fs]
    pick = sorted({int(np.argmin(area)), int(np.argmax(area)), int(np.argmin(act)), int(np.argmax(act))})
    records = {}
    for k in pick:
        f = fs[k]
        # the CLT buffer is shared by the batch: tiles this frame does not
        # list would keep an earlier frame's coefficients
        for c in pipe.clt:
            c.zero_()
        batch.run_frame(f)
        torch.cuda.synchronize()
        geom, TX, TY = f["geom"], f["TX"], f["TY"]
        n = TX * TY * 768
        clt = [pipe.clt[c][:n].cpu().numpy() for c in range(4)]
        images = np.stack([x.cpu().numpy() for x in f["images"]])
        kernels = [x.cpu().numpy() for x in f["kernels"]]
        extras = [x.cpu().numpy() for x in f["extras"]]
        want = oracle.convert_correct_tiles(geom, extras, kernels, images, f["dstride"], f["tasks_np"])
        what = "frame %d %dx%d activity %.2f" % (k, f["size"][0], f["size"][1], f["activity"])
        e_clt = max(rel_err(clt[c], want[c]) for c in range(4))
        assert e_clt < 1e-5, (what, e_clt)
        idx = f["corr_idx"].cpu().numpy()
        co = oracle.correlate2D(geom, [x.astype(np.float64) for x in clt], 3, .25, .25, .5, bench.FAT_ZERO, idx,
                                pipe.corr_stride, bench.CORR_RADIUS)
        cb = pipe.corrs[:len(idx)].cpu().numpy()
        e_corr = rel_err(cb[:, :225], co[:, :225])
        assert e_corr < 1e-5, (what, e_corr)
        st = f["rgba_stride"]
        rows = (TY + 1) * 8 * 4
        rgba = pipe.rgba.view(-1)[:rows * st].view(rows, st).cpu().numpy()
        rec = _check_rgba(oracle, geom, f["tasks_np"], TX, TY, clt, pipe.port_offsets.cpu().numpy(), rgba,
                          pipe.woi.cpu().numpy(), what)
        records[what] = {"clt_max": e_clt, "corr_max": e_corr, "rgba": rec}
    print("\nbench batched frames vs the FP64 oracle " + json.dumps(records))
