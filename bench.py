"""Benchmark: full-frame quad-camera CLT + correlation + texture, frames/s.

One step = one 2592x1936 quad-camera Bayer frame (78,408 tiles) through the
hot path, on inputs already resident in HBM, through the three drop-in entry
points:
  1. tp_convert_correct_tiles  forward CLT + aberration kernels + shifts
  2. tp_correlate2D            6 camera pairs per tile, 15x15 outputs
  3. tp_generate_RBGA          texture list + overlapped RGBA texture
The same frame through tp_process_frame (one kernel per tile parity with the
tile's CLT kept in shared memory) is timed too and reported as
`fused_frame_ms`.
`value` is whole-job frames/s (N GPUs each process their own frames:
frame-level replicas, weak scaling).  `e2e` is the same pipeline driven
through the public API with host buffers: each step copies the frame's four
images from pinned host memory and reads the correlation tiles and the RGBA
texture back.

One step is `--frames-per-step` passes of that frame (48 by default), so the
timed region of a default run lasts a few seconds and the clock samples taken
during it mean something.

`--impl reference` times the CPU implementation (the FP64 port of the
reference's tile math, all host threads), one whole 2592x1936 frame per step,
and beside it the reference's own CUDA kernels rebuilt for sm_100a on the same
frame (`reference_kernels`, when that build is present).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WIDTH, HEIGHT = 2592, 1936
METRIC = "quad 5MP frames/s (CLT+corr+texture)"
UNIT = "frames/s"
CORR_RADIUS = 7
DISPARITY_ERROR = 0.5
LEARNED_LDX = 1352
FAT_ZERO = 0.05
TEXTURE = dict(colors=3, is_lwir=0, min_shot=10.0, scale_shot=3.0, diff_sigma=1.5, diff_threshold=10.0,
               min_agree=3.0, weight0=0.294118, weight1=0.117647, weight2=0.588235, dust_remove=1, keep_weights=0)
WORKLOAD = ("full-frame quad 2592x1936 Bayer (78,408 tiles): forward CLT + aberration correction, "
            "6-pair correlation (15x15), texture list + overlapped RGBA texture")


TILES = (WIDTH // 8) * (HEIGHT // 8)
CORR_TILES = 6 * TILES
FRAMES_PER_STEP = 48
L2_NOTE = ("per-frame working set 3.7 GB (images, touched kernel tables, CLT, correlations, RGBA) > 126 MB L2: "
           "no flush")
# dense 8x8 mat-vec flops per tile of each stage (2 flop per MAC)
FLOPS_PER_TILE = {"convert": 75776, "correlate": 92016, "texture": 149304}
# FP32 SIMT: 148 SMs x 128 lanes x 2 flop x 1.965 GHz
FP32_NOMINAL_TFLOPS = 74.4


def bench_config(world):
    """the workload both arms report (identical in both)"""
    return {"workload": WORKLOAD, "frame": "%dx%d" % (WIDTH, HEIGHT), "tiles": TILES, "corr_tiles": CORR_TILES,
            "parallelism": "frame replicas x%d" % world, "l2": L2_NOTE}


def dram_traffic():
    """DRAM bytes per frame of each stage (and of the fused frame kernel)
    from the ncu captures recorded with the package (captures, not
    measurements of this run): (per stage, source, fused bytes, fused source)"""
    path = os.path.join(ROOT, "tile_processor_gpu_b200", "data", "dram_traffic.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return (d["bytes_per_frame"], "ncu capture: " + d["command"], d.get("fused_frame_bytes"),
                "ncu capture: " + d["fused_command"] if "fused_command" in d else None)
    except (OSError, ValueError, KeyError):
        return {}, None, None, None


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return rank, world, local, pg


def max_over_ranks(pg, value):
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def blob_mask(rng, tx, ty, fraction):
    """Seeded activity mask of round blobs covering about `fraction` of the tiles."""
    m = np.zeros((ty, tx), dtype=bool)
    target = int(round(fraction * tx * ty))
    yy, xx = np.mgrid[0:ty, 0:tx]
    while m.sum() < target:
        cy, cx = rng.integers(0, ty), rng.integers(0, tx)
        r = rng.uniform(1.5, max(2.0, min(tx, ty) / 4))
        m |= (yy - cy) ** 2 + (xx - cx) ** 2 <= r * r
    return m


class BatchedFrames:
    """The batched workload: `n` quad frames of uneven sizes (multiples of 16
    in 640x480 .. 2592x1936), each a crop of the full-frame scene at a seeded
    offset with its own images, kernel table (the full table's window under
    the crop, kernel centres moved to the crop's coordinates), and a
    compacted task list of the tiles under seeded blobs covering 5% .. 100% of
    the frame (tasks at the true disparity + U[-0.5, 0.5] px).  The frames run
    one after another on one stream and share the CLT, correlation, list and
    RGBA buffers of `pipe` (sized for the full frame)."""

    def __init__(self, pipe, n=64, seed=11):
        from tile_processor_gpu_b200 import api, synth
        torch = pipe.torch
        self.pipe, self.api = pipe, api
        rng = np.random.default_rng(seed)
        full = [h.numpy() for h in pipe.host_images]
        gf = pipe.geom_d
        KHf, KVf = gf["kernels_hor"], gf["kernels_vert"]
        d0, gx, gy = pipe.scene_disparity
        dev = pipe.images[0].device
        self.frames = []
        for _ in range(n):
            w = 16 * int(rng.integers(40, WIDTH // 16 + 1))
            h = 16 * int(rng.integers(30, HEIGHT // 16 + 1))
            ox = 16 * int(rng.integers(0, (WIDTH - w) // 16 + 1))
            oy = 16 * int(rng.integers(0, (HEIGHT - h) // 16 + 1))
            geom = synth.geometry(w, h, image_rows=h + 16)
            TX, TY, TYA = synth.tiles(geom)
            mask = blob_mask(rng, TX, TY, float(rng.uniform(0.05, 1.0)))
            tasks_np = synth.tasks_grid(geom, rng, jitter=0.0, disparity=(d0 + gx * ox + gy * oy, gx, gy),
                                        mask=mask, disparity_error=DISPARITY_ERROR)
            idx = synth.corr_indices_fast(tasks_np, geom)
            dstride = w + 64
            images = []
            for c in range(4):
                x = np.zeros((h + 16, dstride), np.float32)
                x[:, :w] = full[c][oy:oy + h + 16, ox:ox + w]
                images.append(torch.from_numpy(x).to(dev))
            kh, kv, kx0, ky0 = geom["kernels_hor"], geom["kernels_vert"], ox // 16, oy // 16
            kernels, extras = [], []
            for c in range(4):
                kf = pipe.kernels[c].view(KVf, KHf, 3 * 256)
                kernels.append(kf[ky0:ky0 + kv, kx0:kx0 + kh].contiguous().view(-1))
                ef = pipe.extra[c].view(KVf, KHf, 3, 8)[ky0:ky0 + kv, kx0:kx0 + kh].clone()
                ef[..., 2] -= ox
                ef[..., 3] -= oy
                extras.append(ef.contiguous().view(-1))
            self.frames.append(dict(
                g=api.Geometry.from_dict(geom), geom=geom, tasks_np=tasks_np, activity=float(mask.mean()),
                TX=TX, TY=TY, dstride=dstride, size=(w, h),
                num_tiles=int(tasks_np.size), num_corr=int(idx.size), tasks=api.tasks_to_device(tasks_np, dev),
                corr_idx=torch.from_numpy(idx).to(dev), images=images, kernels=kernels, extras=extras,
                p_images=api.PointerArray(images), p_kernels=api.PointerArray(kernels),
                p_extra=api.PointerArray(extras), rgba_stride=(TX + 1) * 8))
        self.tiles = sum(f["num_tiles"] for f in self.frames)
        self.pixels = sum(f["size"][0] * f["size"][1] for f in self.frames)

    def run_frame(self, f, lane=None):
        """the frame's three calls, on the pipe's buffers or on a lane's (its
        own CLT, correlation, list and RGBA buffers)"""
        p, api, t = self.pipe, self.api, TEXTURE
        b = lane if lane is not None else {"p_clt": p.p_clt, "corrs": p.corrs, "tex_indices": p.tex_indices,
                                           "num_tex": p.num_tex, "woi": p.woi, "rgba": p.rgba}
        api.convert_correct_tiles(f["g"], f["p_extra"], f["p_kernels"], f["p_images"], f["tasks"], b["p_clt"],
                                  f["dstride"], f["num_tiles"], 0)
        api.correlate2D(f["g"], b["p_clt"], 3, 0.25, 0.25, 0.5, FAT_ZERO, f["num_corr"], f["corr_idx"],
                        p.corr_stride, CORR_RADIUS, b["corrs"])
        api.generate_RBGA(f["g"], f["tasks"], f["num_tiles"], b["tex_indices"], b["num_tex"], b["woi"], f["TX"],
                          f["TY"], b["p_clt"], p.port_offsets, t["colors"], t["is_lwir"], t["min_shot"],
                          t["scale_shot"], t["diff_sigma"], t["diff_threshold"], t["min_agree"], t["weight0"],
                          t["weight1"], t["weight2"], t["dust_remove"], 0, f["rgba_stride"], b["rgba"])

    def lanes(self, count):
        """`count` buffer sets for frames in flight on separate streams, and
        the frames' lanes: the largest frame first to the lane with the
        fewest tiles so far"""
        torch, p, api = self.pipe.torch, self.pipe, self.api
        out = []
        for _ in range(count):
            clt = [torch.empty_like(c) for c in p.clt]
            out.append({"clt": clt, "p_clt": api.PointerArray(clt), "corrs": torch.empty_like(p.corrs),
                        "tex_indices": torch.empty_like(p.tex_indices), "num_tex": torch.empty_like(p.num_tex),
                        "woi": torch.empty_like(p.woi), "rgba": torch.empty_like(p.rgba)})
        load, assign = [0] * count, [0] * len(self.frames)
        for i in sorted(range(len(self.frames)), key=lambda i: -self.frames[i]["num_tiles"]):
            k = min(range(count), key=lambda j: load[j])
            assign[i] = k
            load[k] += self.frames[i]["num_tiles"]
        return out, assign

    def run_streams(self, origin, streams, lanes, assign):
        """every frame on its lane's stream, forked from and joined back to `origin`"""
        for s in streams:
            s.wait_stream(origin)
        for f, k in zip(self.frames, assign):
            with self.pipe.torch.cuda.stream(streams[k]):
                self.run_frame(f, lanes[k])
        for s in streams:
            origin.wait_stream(s)

    def run_all(self):
        for f in self.frames:
            self.run_frame(f)

    def measure(self, stream, replays=10):
        """Per-frame device time of an eager pass (CUDA events around each
        frame's three calls) and the whole batch replayed from one CUDA graph."""
        torch = self.pipe.torch
        self.run_all()
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in self.frames]
        for f, (a, b) in zip(self.frames, evs):
            a.record(stream)
            self.run_frame(f)
            b.record(stream)
        torch.cuda.synchronize()
        lat = np.array([a.elapsed_time(b) for a, b in evs])
        eager_ms = float(lat.sum())
        side = torch.cuda.Stream()
        side.wait_stream(stream)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.stream(side):
            with torch.cuda.graph(graph, stream=side):
                self.run_all()
        stream.wait_stream(side)
        graph.replay()
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(replays):
            graph.replay()
        g1.record(stream)
        torch.cuda.synchronize()
        graph_ms = g0.elapsed_time(g1) / replays
        del graph
        # the same frames on four streams (own buffers per stream), one graph
        nlanes = 4
        lanes, assign = self.lanes(nlanes)
        streams = [torch.cuda.Stream() for _ in range(nlanes)]
        self.run_streams(stream, streams, lanes, assign)
        torch.cuda.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.stream(side):
            with torch.cuda.graph(graph, stream=side):
                self.run_streams(side, streams, lanes, assign)
        stream.wait_stream(side)
        graph.replay()
        torch.cuda.synchronize()
        g0.record(stream)
        for _ in range(replays):
            graph.replay()
        g1.record(stream)
        torch.cuda.synchronize()
        streams_ms = g0.elapsed_time(g1) / replays
        del graph, lanes
        n = len(self.frames)
        return {"frames": n, "sizes": "%dx%d .. %dx%d" % (min(f["size"][0] for f in self.frames),
                                                         min(f["size"][1] for f in self.frames),
                                                         max(f["size"][0] for f in self.frames),
                                                         max(f["size"][1] for f in self.frames)),
                "activity": "tiles under seeded blobs, 5-100% of each frame",
                "tasks": self.tiles, "megapixels": round(self.pixels / 1e6, 1),
                "graph_ms_per_batch": round(graph_ms, 3), "frames_per_s": round(n / graph_ms * 1e3, 1),
                "tiles_per_s": round(self.tiles / graph_ms * 1e3, 0),
                "eager_ms_per_batch": round(eager_ms, 3),
                "frame_ms": {"p50": round(float(np.percentile(lat, 50)), 4),
                             "p99": round(float(np.percentile(lat, 99)), 4),
                             "max": round(float(lat.max()), 4)},
                "full_frame_equivalent_per_s": round(self.tiles / (self.pipe.TX * self.pipe.TY) / graph_ms * 1e3, 1),
                "streams": {"count": nlanes, "what": "the same frames on %d streams (each with its own CLT, "
                            "correlation, list and RGBA buffers; frames to the stream with the fewest tiles, "
                            "largest first), forked and joined inside one CUDA graph" % nlanes,
                            "graph_ms_per_batch": round(streams_ms, 3),
                            "frames_per_s": round(n / streams_ms * 1e3, 1),
                            "tiles_per_s": round(self.tiles / streams_ms * 1e3, 0),
                            "full_frame_equivalent_per_s": round(
                                self.tiles / (self.pipe.TX * self.pipe.TY) / streams_ms * 1e3, 1)}}


# --------------------------------------------------------------------------- #
# the B200 pipeline
# --------------------------------------------------------------------------- #
class FramePipeline:
    """Device buffers for one frame and the three hot-path calls."""

    def __init__(self, seed=0, device="cuda", size=(WIDTH, HEIGHT)):
        import torch
        from tile_processor_gpu_b200 import api, synth
        self.api, self.torch = api, torch
        rng = np.random.default_rng(seed)
        self.W, self.H = W, H = size
        self.geom_d = synth.geometry(W, H, image_rows=H + 16)
        g = self.g = api.Geometry.from_dict(self.geom_d)
        self.TX, self.TY, self.TYA = synth.tiles(self.geom_d)
        imgs, disp = synth.plane_scene(rng, W, H, disparity=(0.0, 64.0), texture="detail")
        self.scene_disparity = disp
        self.dstride = W + 64
        pitched = np.zeros((4, H + 16, self.dstride), np.float32)
        pitched[:, :H, :W] = imgs
        self.host_images = [torch.from_numpy(pitched[c]).pin_memory() for c in range(4)]
        # centred PSFs without kernel-centre offsets: the cameras carry no
        # shift the scene does not have, so the disparity is measurable
        kern, extra = synth.kernel_tables(rng, self.geom_d, pool=256, zero_extra=True, psf_offset=0.0)
        # tasks at the true disparity plus a per-tile error U[-0.5, 0.5] px:
        # the residual the correlations measure is minus that error
        self.tasks_np, err = synth.tasks_grid(self.geom_d, rng, jitter=0.0, disparity=disp,
                                              disparity_error=DISPARITY_ERROR, return_error=True)
        self.true_residual = -err
        self.num_tiles = int(self.tasks_np.size)
        self.images = [h.to(device) for h in self.host_images]
        self.kernels = [torch.from_numpy(kern[c]).to(device) for c in range(4)]
        self.extra = [torch.from_numpy(extra[c]).to(device) for c in range(4)]
        self.tasks = api.tasks_to_device(self.tasks_np, device)
        self.clt = [torch.empty(self.TY * self.TX * 768, dtype=torch.float32, device=device) for _ in range(4)]
        self.p_images, self.p_kernels = api.PointerArray(self.images), api.PointerArray(self.kernels)
        self.p_extra, self.p_clt = api.PointerArray(self.extra), api.PointerArray(self.clt)
        corr_idx = synth.corr_indices_fast(self.tasks_np, self.geom_d)
        self.num_corr = int(corr_idx.size)
        self.corr_idx = torch.from_numpy(corr_idx).to(device)
        self.corr_size = (2 * CORR_RADIUS + 1) ** 2
        self.corr_stride = self.corr_size
        self.corrs = torch.empty((self.num_corr, self.corr_stride), dtype=torch.float32, device=device)
        # fused path: one slot per (task, pair)
        self.corrs6 = torch.empty((self.num_tiles, 6, self.corr_stride), dtype=torch.float32, device=device)
        self.tex_indices = torch.empty(self.TX * self.TYA, dtype=torch.int32, device=device)
        self.num_tex = torch.empty(8, dtype=torch.int32, device=device)
        self.woi = torch.empty(4, dtype=torch.int32, device=device)
        self.rgba_stride = (self.TX + 1) * 8
        self.rgba_rows = (self.TY + 1) * 8 * (TEXTURE["colors"] + 1)
        self.rgba = torch.empty((self.rgba_rows, self.rgba_stride), dtype=torch.float32, device=device)
        self.port_offsets = torch.from_numpy(synth.PORT_OFFSETS.reshape(-1).copy()).to(device)
        self.disparity = torch.empty(self.TX * self.TY, dtype=torch.float32, device=device)
        self.strength = torch.empty(self.TX * self.TY, dtype=torch.float32, device=device)
        # kernel-table bytes a frame touches (distinct kernel tiles of all jobs)
        self.kernel_tiles_touched = self._touched_kernel_tiles()
        self.host_corrs = torch.empty_like(self.corrs, device="cpu").pin_memory()
        self.host_rgba = torch.empty_like(self.rgba, device="cpu").pin_memory()

    def _touched_kernel_tiles(self):
        gd = self.geom_d
        n = 0
        for cam in range(4):
            cx = self.tasks_np["xy"][:, cam, 0].astype(np.float32)
            cy = self.tasks_np["xy"][:, cam, 1].astype(np.float32)
            kx = np.clip(np.rint(cx / 16 + 1), 0, gd["kernels_hor"] - 1).astype(np.int64)
            ky = np.clip(np.rint(cy / 16 + 1), 0, gd["kernels_vert"] - 1).astype(np.int64)
            n += np.unique(kx + ky * gd["kernels_hor"]).size * 3
        return n

    # stage calls (each is a C ABI call on the current stream); `slot` selects
    # another frame's images and outputs (see add_slot), None the main ones
    def convert(self, slot=None):
        p_images = self.p_images if slot is None else slot["p_images"]
        self.api.convert_correct_tiles(self.g, self.p_extra, self.p_kernels, p_images, self.tasks, self.p_clt,
                                       self.dstride, self.num_tiles, 0)

    def correlate(self, slot=None):
        corrs = self.corrs if slot is None else slot["corrs"]
        self.api.correlate2D(self.g, self.p_clt, 3, 0.25, 0.25, 0.5, FAT_ZERO, self.num_corr, self.corr_idx,
                             self.corr_stride, CORR_RADIUS, corrs)

    def texture(self, slot=None):
        t = TEXTURE
        rgba = self.rgba if slot is None else slot["rgba"]
        self.api.generate_RBGA(self.g, self.tasks, self.num_tiles, self.tex_indices, self.num_tex, self.woi, self.TX,
                               self.TY, self.p_clt, self.port_offsets, t["colors"], t["is_lwir"], t["min_shot"],
                               t["scale_shot"], t["diff_sigma"], t["diff_threshold"], t["min_agree"], t["weight0"],
                               t["weight1"], t["weight2"], t["dust_remove"], 0, self.rgba_stride, rgba)

    # the precision form: the same three calls with their 8x8 transforms on the
    # tensor cores (split FP16 or BF16 operands); the texture call's inverse
    # CLT goes through a tile buffer of the CLT's size
    def precision_stage(self, stage, fmt):
        api, t = self.api, TEXTURE
        if stage == "convert":
            api.convert_correct_tiles_tc(self.g, self.p_extra, self.p_kernels, self.p_images, self.tasks, self.p_clt,
                                         self.dstride, self.num_tiles, 0, fmt=fmt)
        elif stage == "correlate":
            api.correlate2D_tc(self.g, self.p_clt, 3, 0.25, 0.25, 0.5, FAT_ZERO, self.num_corr, self.corr_idx,
                               self.corr_stride, CORR_RADIUS, self.corrs, fmt=fmt)
        else:
            if not hasattr(self, "p_tiles"):
                self.tiles = [self.torch.empty_like(c) for c in self.clt]
                self.p_tiles = api.PointerArray(self.tiles)
            api.generate_RBGA_tc(self.g, self.tasks, self.num_tiles, self.tex_indices, self.num_tex, self.woi,
                                 self.TX, self.TY, self.p_clt, self.port_offsets, t["colors"], t["is_lwir"],
                                 t["min_shot"], t["scale_shot"], t["diff_sigma"], t["diff_threshold"],
                                 t["min_agree"], t["weight0"], t["weight1"], t["weight2"], t["dust_remove"], 0,
                                 self.rgba_stride, self.rgba, self.p_tiles, fmt=fmt)

    def add_slot(self, device):
        """Device images and outputs plus pinned host outputs of one more
        frame in flight (the CLT, tasks and lists are used within one frame's
        compute and stay shared)."""
        torch = self.torch
        images = [torch.empty_like(x) for x in self.images]
        return {"images": images, "p_images": self.api.PointerArray(images),
                "corrs": torch.empty_like(self.corrs), "rgba": torch.empty_like(self.rgba),
                "host_corrs": torch.empty_like(self.corrs, device="cpu").pin_memory(),
                "host_rgba": torch.empty_like(self.rgba, device="cpu").pin_memory()}

    def step_slot(self, slot):
        self.convert(slot)
        self.correlate(slot)
        self.texture(slot)

    def frame(self):
        t = TEXTURE
        self.api.process_frame(self.g, self.p_extra, self.p_kernels, self.p_images, self.dstride, self.tasks,
                               self.num_tiles, self.corrs6, self.corr_stride, self.port_offsets, self.tex_indices,
                               self.num_tex, self.woi, self.rgba_stride, self.rgba, corr_colors=3, scale0=0.25,
                               scale1=0.25, scale2=0.5, fat_zero=FAT_ZERO, corr_radius=CORR_RADIUS,
                               min_shot=t["min_shot"], scale_shot=t["scale_shot"], diff_sigma=t["diff_sigma"],
                               weight0=t["weight0"], weight1=t["weight1"], weight2=t["weight2"],
                               dust_remove=t["dust_remove"])

    def disparity_fit(self):
        self.api.disparity_fit(self.g, self.corrs, self.corr_stride, CORR_RADIUS, self.num_corr, self.corr_idx,
                               self.port_offsets, self.disparity, self.strength)

    def learned_setup(self):
        """the shipped network (tile_processor_gpu_b200/data/disparity_mlp.npz), packed for the tensor cores"""
        from tile_processor_gpu_b200 import disparity_net as D
        torch = self.torch
        path = os.path.join(ROOT, "tile_processor_gpu_b200", "data", "disparity_mlp.npz")
        self.net = D.DisparityMLP.load(path, device=self.corrs.device)
        try:
            with open(os.path.splitext(path)[0] + ".json") as fh:
                self.net_report = json.load(fh)
        except (OSError, ValueError):
            self.net_report = {}
        self.net.pack()
        # rows of 1352 floats start on 16-byte boundaries: 16-byte feature copies in the inference
        self.feat = torch.zeros((self.TX * self.TY, LEARNED_LDX), dtype=torch.float32, device=self.corrs.device)
        self.net_out = torch.zeros((self.TX * self.TY, 2), dtype=torch.float32, device=self.corrs.device)
        self.learned = torch.zeros(self.TX * self.TY, dtype=torch.float32, device=self.corrs.device)

    def learned_features(self):
        from tile_processor_gpu_b200 import disparity_net as D
        D.features(self.g, self.corrs, self.corr_stride, CORR_RADIUS, self.num_corr, self.corr_idx, self.feat,
                   feature_stride=LEARNED_LDX)

    def learned_infer(self):
        """the network's {d, s} per tile and the estimate with the plain fit as fallback"""
        self.net.infer_tc(self.feat, self.TX * self.TY, self.net_out, ldx=LEARNED_LDX)
        self.net.combine(self.disparity, self.net_out, self.TX * self.TY, self.learned)

    def disparity_accuracy(self):
        """RMS error of the fitted residual against the truth on tiles whose
        footprint stays inside every camera's frame (disparity <= 64 px moves
        a camera by <= 32 px: 5 tiles of margin)"""
        tx = self.tasks_np["txy"] & 0xFFFF
        ty = self.tasks_np["txy"] >> 16
        inner = (tx >= 5) & (tx < self.TX - 5) & (ty >= 5) & (ty < self.TY - 5)
        got = self.disparity.cpu().numpy()[ty * self.TX + tx].astype(np.float64)
        res = got[inner] - self.true_residual[inner]
        learned = None
        if hasattr(self, "net_out"):
            tile = ty * self.TX + tx
            lg = self.learned.cpu().numpy()[tile].astype(np.float64)
            lr = lg[inner] - self.true_residual[inner]
            lu = (got + self.net_out.cpu().numpy()[tile, 0].astype(np.float64))[inner] - self.true_residual[inner]
            kept = float(np.mean(self.net_out.cpu().numpy()[tile, 1][inner] < self.net.gate))
            learned = {"rmse_px": round(float(np.sqrt(np.mean(lr ** 2))), 4),
                       "outliers_gt_0.5px": round(float(np.mean(np.abs(lr) > 0.5)), 5),
                       "gate_logvar": self.net.gate if np.isfinite(self.net.gate) else None,
                       "corrected_fraction": round(kept, 4),
                       "ungated": {"rmse_px": round(float(np.sqrt(np.mean(lu ** 2))), 4),
                                   "outliers_gt_0.5px": round(float(np.mean(np.abs(lu) > 0.5)), 5)},
                       "net": "1350-256-128-2 GELU MLP on the six planes, shipped weights (%s synthetic tiles, "
                              "8 lenses, planes and occlusion edges), layer 1 TF32 and layer 2 BF16 tcgen05 MMAs "
                              "(tp_mlp_infer_tc), plain fit kept where the log-variance is above the gate "
                              "(tp_mlp_combine)" % self.net_report.get("train_tiles", "?")}
        return {"rmse_px": round(float(np.sqrt(np.mean(res ** 2))), 4),
                "outliers_gt_0.5px": round(float(np.mean(np.abs(res) > 0.5)), 5),
                "truth_rms_px": round(float(np.sqrt(np.mean(self.true_residual[inner] ** 2))), 4),
                "tiles": int(inner.sum()), "fit": "3-point parabola on the 6-pair profile (tp_disparity_fit mode 0)",
                "learned": learned,
                "truth": "plane scene disparity; task error U[-%.1f, %.1f] px per tile" % (DISPARITY_ERROR,
                                                                                        DISPARITY_ERROR)}

    STAGES = ("convert", "correlate", "texture")
    LAUNCHES = {"convert": 1, "correlate": 1, "texture": 11}  # texture: 6 list kernels, RGBA clear, 4 passes
    FRAME_LAUNCHES = 11  # 6 list kernels, RGBA clear, 4 parity launches

    def step(self):
        self.convert()
        self.correlate()
        self.texture()

    def frame_bytes(self):
        """compulsory HBM bytes of one frame through the fused path: images,
        touched kernel tiles and offsets, tasks, correlation out, RGBA out"""
        T = self.num_tiles
        return (4 * self.W * self.H * 4 + self.kernel_tiles_touched * (1024 + 32) + T * 40 +
                self.num_corr * self.corr_size * 4 + (self.TX + 1) * 8 * (self.TY + 1) * 8 * 4 * 4)

    def algorithmic_bytes(self):
        """compulsory HBM bytes of each drop-in stage of one frame"""
        T = self.num_tiles
        clt = 4 * T * 3 * 1024
        return {
            "convert": 4 * self.W * self.H * 4 + self.kernel_tiles_touched * (1024 + 32) + T * 40 + clt,
            "correlate": clt + self.num_corr * 4 + self.num_corr * self.corr_size * 4,
            "texture": clt + T * 40 + (self.TX + 1) * 8 * (self.TY + 1) * 8 * 4 * 4,
        }


def run_child(child_args, timeout):
    """bench.py --child ... in a subprocess; its last stdout line as JSON (or
    the reason there is none)"""
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--child"] + child_args
    try:
        res = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    except subprocess.TimeoutExpired:
        return {"error": "child %s: no result within %d s" % (child_args[0], timeout)}
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    if res.returncode != 0 or not lines:
        tail = (res.stderr.strip().splitlines() or ["(no output)"])[-1][:200]
        return {"error": "child %s exited %d: %s" % (child_args[0], res.returncode, tail)}
    return json.loads(lines[-1])


def child_precision_timing(args):
    """The precision form (tp_*_tc) on the bench frame, both operand formats:
    per-stage CUDA-event times over `args.steps` frames after two warm-up
    frames."""
    import torch
    size = tuple(int(v) for v in args.frame.split("x"))
    pipe = FramePipeline(seed=100, device="cuda:0", size=size)
    stream = torch.cuda.current_stream()
    pipe.step()
    torch.cuda.synchronize()
    precision = {}
    for name, fmt in (("fp16x2", pipe.api.TC_FP16X2), ("bf16x2", pipe.api.TC_BF16X2)):
        try:
            for _ in range(2):
                for st in pipe.STAGES:
                    pipe.precision_stage(st, fmt)
            torch.cuda.synchronize()
            evp = {st: [] for st in pipe.STAGES}
            for _ in range(args.steps):
                for st in pipe.STAGES:
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                    pipe.precision_stage(st, fmt)
                    b.record(stream)
                    evp[st].append((a, b))
            torch.cuda.synchronize()
            pst = {st: sum(a.elapsed_time(b) for a, b in v) / args.steps for st, v in evp.items()}
            precision[name] = {"frame_ms": round(sum(pst.values()), 4),
                               "frames_per_s": round(1e3 / sum(pst.values()), 1),
                               "stages_ms": {k: round(v, 4) for k, v in pst.items()},
                               "timed_out": pipe.api.tc_status()}
        except Exception as e:  # reported beside the plain path, never instead of it
            precision[name] = {"error": str(e).splitlines()[0][:200]}
    return precision


def child_precision_parity(args):
    """The precision form's per-stage errors against the FP64 oracle on the
    CPU-baseline sample and on the HDR scene (the checker; see sample_parity)"""
    S = cpu_pipeline(args.cpu_sample_tiles)
    hdr = cpu_pipeline(0, size=(1024, 768), peak=1e4, seed=31)
    out = {}
    for name, T in (("sample", S), ("hdr", hdr)):
        w = T["O"].convert_correct_tiles(T["geom"], T["extra"], T["kern"], T["pitched"], T["dstride"], T["tasks"])
        out[name] = {"sample": T["what"], **precision_errors(T, w)}
    return out


def run_b200(args, rank, world, local, pg):
    import torch
    dev = "cuda:%d" % local
    torch.cuda.set_device(local)
    from tile_processor_gpu_b200 import build
    build.build()
    size = tuple(int(v) for v in args.frame.split("x"))
    pipe = FramePipeline(seed=100 + rank, device=dev, size=size)
    stream = torch.cuda.current_stream()
    # launch shapes (grid caps) of the three stage kernels, tuned on this frame
    from tile_processor_gpu_b200 import autotune
    pipe.step()
    torch.cuda.synchronize()
    shapes = None
    if args.shapes:
        # fixed grid caps, e.g. convert=8,correlate=6,textures=4 (no tuning launches)
        for item in args.shapes.split(","):
            k, v = item.split("=")
            autotune.set_shape(k.strip(), int(v))
    elif not args.no_tune:
        shapes = autotune.tune_stages({"convert": pipe.convert, "correlate": pipe.correlate,
                                       "textures": pipe.texture})
    frame_shapes = {k: autotune.get_shape(k) for k in autotune.KERNELS}
    for _ in range(args.warmup * args.frames_per_step):
        pipe.step()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    ev = {s: [] for s in pipe.STAGES}
    F = args.frames_per_step
    barrier(pg)
    torch.cuda.synchronize()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for _ in range(args.steps):
        for _ in range(F):
            for s in pipe.STAGES:
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                getattr(pipe, s)()
                b.record(stream)
                ev[s].append((a, b))
    t_end.record(stream)
    torch.cuda.synchronize()
    barrier(pg)
    clocks = sampler.stop()
    ms = t_start.elapsed_time(t_end)
    ms_max = max_over_ranks(pg, ms)
    frames_timed = args.steps * F
    stage_ms = {s: sum(a.elapsed_time(b) for a, b in ev[s]) / frames_timed for s in pipe.STAGES}

    # the same frame through tp_process_frame (fused per tile), reported beside
    fused_steps = max(3, min(args.steps, 10))
    for _ in range(2):
        pipe.frame()
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(fused_steps):
        pipe.frame()
    f1.record(stream)
    torch.cuda.synchronize()
    fused_ms = f0.elapsed_time(f1) / fused_steps

    # the same step captured once in a CUDA graph and replayed (17 launches)
    graph_ms = None
    try:
        side = torch.cuda.Stream()
        side.wait_stream(stream)
        with torch.cuda.stream(side):
            pipe.step()
        stream.wait_stream(side)
        torch.cuda.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            pipe.step()
        graph.replay()
        torch.cuda.synchronize()
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(fused_steps):
            graph.replay()
        g1.record(stream)
        torch.cuda.synchronize()
        graph_ms = round(g0.elapsed_time(g1) / fused_steps, 4)
        del graph
    except Exception as e:  # capture is optional: the eager step is the measurement
        graph_ms = "capture failed: %s" % str(e).splitlines()[0][:120]

    # the precision form (tensor-core transforms), both operand formats, timed
    # in a child process on its own copy of the frame: whatever happens there
    # cannot cost this line
    precision = run_child(["precision-timing", "--frame", args.frame, "--steps", str(fused_steps)], timeout=900)

    # the disparity fit on the frame's correlations (the consumer of stage 2)
    pipe.step()
    pipe.disparity_fit()
    torch.cuda.synchronize()
    d0 = torch.cuda.Event(enable_timing=True)
    d1 = torch.cuda.Event(enable_timing=True)
    d0.record(stream)
    for _ in range(fused_steps):
        pipe.disparity_fit()
    d1.record(stream)
    torch.cuda.synchronize()
    fit_ms = d0.elapsed_time(d1) / fused_steps
    # the learned residual on the same correlations: features and tensor-core inference
    pipe.learned_setup()
    pipe.learned_features()
    pipe.learned_infer()
    torch.cuda.synchronize()
    l0, l1, l2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    l0.record(stream)
    for _ in range(fused_steps):
        pipe.learned_features()
    l1.record(stream)
    for _ in range(fused_steps):
        pipe.learned_infer()
    l2.record(stream)
    torch.cuda.synchronize()
    disparity = pipe.disparity_accuracy()
    disparity["fit_ms"] = round(fit_ms, 4)
    if disparity.get("learned"):
        disparity["learned"]["features_ms"] = round(l0.elapsed_time(l1) / fused_steps, 4)
        infer_ms = l1.elapsed_time(l2) / fused_steps
        rows = pipe.TX * pipe.TY
        disparity["learned"]["infer_ms"] = round(infer_ms, 4)
        # algorithmic work of one inference: 2 (1350*256 + 256*128 + 128*2) flops and the 1350 FP32 features per row
        disparity["learned"]["infer_tflops"] = round(rows * 2 * (1350 * 256 + 256 * 128 + 128 * 2) / infer_ms / 1e9, 1)
        disparity["learned"]["infer_feature_gbs"] = round(rows * 1350 * 4 / infer_ms / 1e6, 1)
        # what each estimate costs the frame: the stage kernels plus the plain
        # fit, and plus the features and the inference for the learned one
        frame_ms = ms / frames_timed
        learned_ms = fit_ms + disparity["learned"]["features_ms"] + infer_ms
        disparity["per_frame_cost"] = {
            "plain_fit_ms": round(fit_ms, 4), "learned_ms": round(learned_ms, 4),
            "frames_per_s_with_plain_fit": round(1e3 / (frame_ms + fit_ms), 1),
            "frames_per_s_with_learned": round(1e3 / (frame_ms + learned_ms), 1)}

    # ---- the batched workload: 64 uneven sparse frames, one CUDA graph ----
    batched = None
    if not args.no_batched and size == (WIDTH, HEIGHT):
        batch = BatchedFrames(pipe, n=64, seed=11 + rank)
        batch_shapes = None
        if not args.no_tune and not args.shapes:
            batch.run_all()
            batch_shapes = autotune.tune_stages({"convert": batch.run_all, "correlate": batch.run_all,
                                                 "textures": batch.run_all}, repeats=3, warmup=1)
        batched = batch.measure(stream)
        batched["launch_shapes"] = batch_shapes or {k: autotune.get_shape(k) for k in autotune.KERNELS}
        for k, v in frame_shapes.items():
            autotune.set_shape(k, v)

    # ---- end to end through the public API with host buffers ----
    # Every frame: its four images from pinned host memory to the device, the
    # three calls, its correlation tiles and RGBA image back to pinned host
    # memory.  Two frames in flight on three streams (copy in, compute, copy
    # out), so the PCIe transfers of one frame overlap the compute of another;
    # a frame's upload waits for the compute of the frame two before it (same
    # slot), its compute for its upload and for that frame's download.
    e2e_steps = max(4, min(args.steps, 30))
    h2d = sum(h.numel() * 4 for h in pipe.host_images)
    d2h = pipe.corrs.numel() * 4 + pipe.rgba.numel() * 4
    slots = [pipe.add_slot(dev), pipe.add_slot(dev)]
    s_in, s_comp, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    ev = lambda: torch.cuda.Event(enable_timing=False)
    in_done, comp_done, out_done = [ev(), ev()], [ev(), ev()], [ev(), ev()]
    barrier(pg)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s_in)
    s_comp.wait_stream(s_in)
    s_out.wait_stream(s_in)
    for i in range(e2e_steps):
        k = i & 1
        sl = slots[k]
        with torch.cuda.stream(s_in):
            if i >= 2:
                s_in.wait_event(comp_done[k])
            for c in range(4):
                sl["images"][c].copy_(pipe.host_images[c], non_blocking=True)
            in_done[k].record(s_in)
        with torch.cuda.stream(s_comp):
            s_comp.wait_event(in_done[k])
            if i >= 2:
                s_comp.wait_event(out_done[k])
            pipe.step_slot(sl)
            comp_done[k].record(s_comp)
        with torch.cuda.stream(s_out):
            s_out.wait_event(comp_done[k])
            sl["host_corrs"].copy_(sl["corrs"], non_blocking=True)
            sl["host_rgba"].copy_(sl["rgba"], non_blocking=True)
            out_done[k].record(s_out)
    s_out.wait_stream(s_comp)
    s_out.wait_stream(s_in)
    e1.record(s_out)
    torch.cuda.synchronize()
    barrier(pg)
    e2e_ms = max_over_ranks(pg, e0.elapsed_time(e1)) / e2e_steps

    if rank != 0:
        return None
    hbm, peak_kind = peaks()
    algo = pipe.algorithmic_bytes()
    dom = max(stage_ms, key=stage_ms.get)
    achieved = algo[dom] / (stage_ms[dom] * 1e-3) / 1e9
    fps = world * frames_timed / (ms_max * 1e-3)
    flops = FLOPS_PER_TILE[dom] * pipe.num_tiles
    traffic, traffic_source, fused_traffic, fused_source = dram_traffic()
    out = {
        "metric": METRIC, "value": round(fps, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded plane scene, centred PSF kernels)",
        "config": bench_config(world) if size == (WIDTH, HEIGHT) else dict(
            bench_config(world), frame="%dx%d" % size, tiles=pipe.num_tiles, corr_tiles=pipe.num_corr,
            workload="profiling case (not the benchmark workload)"),
        "frames_per_step": F, "ms_per_frame": round(ms_max / frames_timed, 4),
        "path": "tp_convert_correct_tiles + tp_correlate2D + tp_generate_RBGA",
        "stages_ms": {k: round(v, 4) for k, v in stage_ms.items()},
        "fused_frame_ms": round(fused_ms, 4),
        "fused_frame": {"ms": round(fused_ms, 4), "dram_bytes": fused_traffic, "dram_source": fused_source,
                        "staged_dram_bytes": int(sum(traffic.values())) if traffic else None,
                        "compulsory_bytes": int(pipe.frame_bytes()),
                        "hbm_frac_of_measured": round(pipe.frame_bytes() / (fused_ms * 1e-3) / 1e9 / hbm, 4)},
        "precision": {"what": "the same three calls with each stage's 8x8 transforms as tcgen05 GEMMs "
                              "(tp_*_tc: split 16-bit operands, three MMAs per product, FP32 accumulation); "
                              "errors against the FP64 oracle in parity.precision",
                      **precision},
        "graph_frame_ms": graph_ms,
        "disparity": disparity,
        "batched": batched,
        "launch_shapes": shapes or frame_shapes,
        "roofline": {"bound": "hbm", "kernel": "k_textures (%s stage)" % dom, "achieved": round(achieved, 1),
                     "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4), "peak_kind": peak_kind,
                     "algorithmic_bytes": int(algo[dom]), "traffic": int(traffic[dom]) if dom in traffic else None,
                     "traffic_source": traffic_source,
                     "fp32_simt": {"flops": int(flops), "achieved_tflops": round(flops / (stage_ms[dom] * 1e-3) / 1e12, 2),
                                   "nominal_peak_tflops": FP32_NOMINAL_TFLOPS}},
        "e2e": {"value": round(world / (e2e_ms * 1e-3), 3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "frames": e2e_steps,
                "overlap": "two frames in flight: copy-in, compute, copy-out streams"},
        "gpu_launches": int(frames_timed * sum(pipe.LAUNCHES.values())),
        "clocks": clocks,
    }
    if world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"], out["parity"] = cpu_baseline(args.cpu_sample_tiles)
    return out


# --------------------------------------------------------------------------- #
# CPU implementation (the FP64 port of the reference's tile math)
# --------------------------------------------------------------------------- #
def cpu_pipeline(sample_tiles, seed=100, size=None, peak=None):
    """A bounded sample of the workload for the CPU port: a crop of the same
    seeded scene, sized to about `sample_tiles` tiles (or a whole frame of
    `size` = (w, h)), through all three stages (the per-tile work does not
    depend on the frame size).  With seed 100 and the full size this is the
    frame the B200 arm's rank 0 runs.  Returns the inputs and a step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from tile_processor_gpu_b200 import synth
    O.build()
    rng = np.random.default_rng(seed)
    w = WIDTH
    h = max(32, min(HEIGHT, (sample_tiles // (WIDTH // 8)) * 8))
    if size is not None:
        w, h = size
    geom = synth.geometry(w, h, image_rows=h + 16)
    kw = {} if peak is None else {"peak": peak}
    imgs, disp = synth.plane_scene(rng, w, h, disparity=(0.0, 64.0), texture="detail", **kw)
    dstride = w + 64
    pitched = np.zeros((4, h + 16, dstride), np.float32)
    pitched[:, :h, :w] = imgs
    kern, extra = synth.kernel_tables(rng, geom, pool=256, zero_extra=True, psf_offset=0.0)
    tasks = synth.tasks_grid(geom, rng, jitter=0.0, disparity=disp, disparity_error=DISPARITY_ERROR)
    corr_idx = synth.corr_indices_fast(tasks, geom)
    TX, TY, TYA = synth.tiles(geom)

    def step():
        clt = O.convert_correct_tiles(geom, extra, kern, pitched, dstride, tasks)
        O.correlate2D(geom, clt, 3, .25, .25, .5, FAT_ZERO, corr_idx, (2 * CORR_RADIUS + 1) ** 2, CORR_RADIUS)
        O.generate_RBGA(geom, tasks, TX, TY, clt, synth.PORT_OFFSETS, (TX + 1) * 8, (TY + 1) * 8 * 4 + 8)

    full = (w, h) == (WIDTH, HEIGHT)
    return dict(O=O, step=step, ntiles=int(tasks.size), geom=geom, pitched=pitched, kern=kern, extra=extra,
                tasks=tasks, corr_idx=corr_idx, TX=TX, TY=TY, TYA=TYA, dstride=dstride,
                port_offsets=synth.PORT_OFFSETS,
                what=("the whole %dx%d frame (%d tiles)" if full else "%dx%d crop (%d tiles)") % (w, h, tasks.size))


def _gpu_on_sample(S, fmt=None):
    """This library's three calls on a CPU sample's inputs (fmt None: the
    plain path; else the precision form with that operand format): CLT,
    correlations, RGBA image and window as host arrays."""
    import torch
    from tile_processor_gpu_b200 import api
    geom, TX, TY = S["geom"], S["TX"], S["TY"]
    dev = "cuda"
    pa = api.PointerArray
    g = api.Geometry.from_dict(geom)
    images = [torch.from_numpy(S["pitched"][c]).to(dev) for c in range(4)]
    kernels = [torch.from_numpy(np.ascontiguousarray(S["kern"][c])).to(dev) for c in range(4)]
    extras = [torch.from_numpy(np.ascontiguousarray(S["extra"][c])).to(dev) for c in range(4)]
    tasks = api.tasks_to_device(S["tasks"], dev)
    n, idx = S["ntiles"], S["corr_idx"]
    clt = [torch.zeros(TX * TY * 768, dtype=torch.float32, device=dev) for _ in range(4)]
    corrs = torch.zeros((len(idx), 225), dtype=torch.float32, device=dev)
    idx_d = torch.from_numpy(idx).to(dev)
    stride, rows = (TX + 1) * 8, (TY + 1) * 8 * 4
    rgba = torch.zeros((rows, stride), dtype=torch.float32, device=dev)
    lst = torch.zeros(TX * S["TYA"], dtype=torch.int32, device=dev)
    cnt = torch.zeros(8, dtype=torch.int32, device=dev)
    woi_d = torch.zeros(4, dtype=torch.int32, device=dev)
    t = TEXTURE
    po = torch.from_numpy(np.ascontiguousarray(S["port_offsets"], np.float32).reshape(-1)).to(dev)
    targs = (t["colors"], t["is_lwir"], t["min_shot"], t["scale_shot"], t["diff_sigma"], t["diff_threshold"],
             t["min_agree"], t["weight0"], t["weight1"], t["weight2"], t["dust_remove"], 0, stride, rgba)
    if fmt is None:
        api.convert_correct_tiles(g, pa(extras), pa(kernels), pa(images), tasks, pa(clt), S["dstride"], n, 0)
        api.correlate2D(g, pa(clt), 3, .25, .25, .5, FAT_ZERO, len(idx), idx_d, 225, CORR_RADIUS, corrs)
        api.generate_RBGA(g, tasks, n, lst, cnt, woi_d, TX, TY, pa(clt), po, *targs)
    else:
        tiles = [torch.zeros_like(c) for c in clt]
        api.convert_correct_tiles_tc(g, pa(extras), pa(kernels), pa(images), tasks, pa(clt), S["dstride"], n, 0,
                                     fmt=fmt)
        api.correlate2D_tc(g, pa(clt), 3, .25, .25, .5, FAT_ZERO, len(idx), idx_d, 225, CORR_RADIUS, corrs, fmt=fmt)
        api.generate_RBGA_tc(g, tasks, n, lst, cnt, woi_d, TX, TY, pa(clt), po, *targs, pa(tiles), fmt=fmt)
    torch.cuda.synchronize()
    return [c.cpu().numpy() for c in clt], corrs.cpu().numpy(), rgba.cpu().numpy(), woi_d.cpu().numpy()


def _rel(a, b):
    a = np.asarray(a, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _rms(a, b):
    a = np.asarray(a, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2)) / max(np.abs(b).max(), 1e-300))


def _rgba_errors(S, rgba, clt_ref, woi, eps=1e-6):
    """per-slice errors of an RGBA image against the oracle's from clt_ref,
    on pixels whose tiles the oracle's conditioning probe finds stable"""
    import conditioning
    O, geom, TX, TY = S["O"], S["geom"], S["TX"], S["TY"]
    po = np.ascontiguousarray(S["port_offsets"], np.float32).reshape(-1)
    o, _, _, _, woi_o = O.generate_RBGA(geom, S["tasks"], TX, TY, clt_ref, po, rgba.shape[1], rgba.shape[0] + 8)
    h, w = (woi[3] + 1) * 8, (woi[2] + 1) * 8
    txy = S["tasks"]["txy"].astype(np.int64)
    tiles = (txy & 0xFFFF) + (txy >> 16) * TX
    bad, _ = conditioning.unstable_tiles(O, geom, po, clt_ref, tiles, eps=eps)
    m = conditioning.unstable_image_mask(bad.any(axis=1), tiles << 8, woi, TX, (h, w), 4)
    sl = lambda a: a[:4 * h, :w].reshape(4, h, w)[None]
    per = conditioning.stable_errors(sl(rgba), sl(o), sl(~m))
    out = {}
    for nm, r, k in zip(("r", "b", "g", "alpha"), per, range(4)):
        keep = ~m[:h]  # the mask is the same for the four slices
        g_, o_ = sl(rgba)[0, k][keep].astype(np.float64), sl(o)[0, k][keep]
        r["rms"] = float(np.sqrt(np.mean((g_ - o_) ** 2)) / max(np.abs(o_).max(), 1e-300))
        out[nm] = {kk: float("%.3g" % v) for kk, v in r.items()}
    return out, bool(np.array_equal(woi, woi_o))


def precision_errors(T, w):
    """per-stage errors of the precision form (both formats) on sample T
    against the oracle pipeline from the same inputs (w: the oracle's CLT)"""
    from tile_processor_gpu_b200 import api
    out = {}
    co = T["O"].correlate2D(T["geom"], w, 3, .25, .25, .5, FAT_ZERO, T["corr_idx"], 225, CORR_RADIUS)
    for name, fmt in (("fp16x2", api.TC_FP16X2), ("bf16x2", api.TC_BF16X2)):
        clt, corrs, rgba, woi = _gpu_on_sample(T, fmt)
        # stable against perturbations the size of the format's own error
        tex, woi_ok = _rgba_errors(T, rgba, w, woi, eps=1e-6 if fmt == api.TC_FP16X2 else 1e-5)
        out[name] = {"clt": {"max": float("%.3g" % max(_rel(clt[c], w[c]) for c in range(4))),
                             "rms": float("%.3g" % max(_rms(clt[c], w[c]) for c in range(4)))},
                     "corr": {"max": float("%.3g" % _rel(corrs, co)), "rms": float("%.3g" % _rms(corrs, co))},
                     "texture": tex, "window_equal": woi_ok, "timed_out": api.tc_status()}
    return out


def sample_parity(S, hdr=None):
    """This library on the CPU sample's inputs, checked against the FP64
    oracle (the checker).  Plain path: the CLT from the same inputs, the
    correlations and the overlapped RGBA image from this library's CLT
    (isolating each stage).  Precision form (both operand formats): each
    stage fed by the one before it, against the oracle's own pipeline from the
    same inputs.  Texture pixels are compared where the oracle's conditioning
    probe finds them stable (1e-6 input perturbations, 6-digit window tables).
    Errors relative to the oracle's largest magnitude (per RGBA slice).  `hdr`:
    a second, high-dynamic-range sample run the same way."""
    O, geom = S["O"], S["geom"]
    want = O.convert_correct_tiles(geom, S["extra"], S["kern"], S["pitched"], S["dstride"], S["tasks"])
    idx = S["corr_idx"]

    def plain_record(T):
        clt, corrs, rgba, woi = _gpu_on_sample(T)
        w = want if T is S else O.convert_correct_tiles(T["geom"], T["extra"], T["kern"], T["pitched"],
                                                        T["dstride"], T["tasks"])
        co = T["O"].correlate2D(T["geom"], [x.astype(np.float64) for x in clt], 3, .25, .25, .5, FAT_ZERO,
                                T["corr_idx"], 225, CORR_RADIUS)
        tex, woi_ok = _rgba_errors(T, rgba, clt, woi)
        return {"sample": T["what"], "clt_max_rel": float("%.3g" % max(_rel(clt[c], w[c]) for c in range(4))),
                "corr_max_rel": float("%.3g" % _rel(corrs, co)), "window_equal": woi_ok, "texture": tex}, w

    rec, _ = plain_record(S)
    out = {"against": "FP64 oracle (CPU restatement of the reference's tile math)",
           "rule": "texture: overlapped RGBA on pixels whose tiles the oracle's conditioning probe finds stable; "
                   "errors relative to the oracle's largest magnitude (per slice)", **rec}
    if hdr is not None:
        out["hdr"], _ = plain_record(hdr)
    # the precision form, per stage, each fed by the one before it, against
    # the oracle's own pipeline (in a child process: see run_child)
    out["precision"] = run_child(["precision-parity", "--cpu-sample-tiles", str(S["ntiles"])], timeout=900)
    return out


def cpu_baseline(sample_tiles, min_seconds=10.0, max_reps=5):
    """The port on all host threads: repeat the sample until about
    `min_seconds` of CPU work (at most `max_reps` repetitions).  Also returns
    the parity of this library against the oracle on the same sample."""
    S = cpu_pipeline(sample_tiles)
    O, step = S["O"], S["step"]
    reps = 0
    t = time.perf_counter()
    while reps < max_reps and (reps == 0 or time.perf_counter() - t < min_seconds):
        step()
        reps += 1
    dt = (time.perf_counter() - t) / reps
    frames = S["ntiles"] / TILES
    # the small configuration (a whole 256x256 quad frame, 1,024 tiles) as well
    small = cpu_pipeline(0, size=(256, 256))
    small["step"]()
    t = time.perf_counter()
    for _ in range(3):
        small["step"]()
    small_ms = (time.perf_counter() - t) / 3 * 1e3
    rec = {"value": round(frames / dt, 5), "unit": UNIT, "cores": O.get_threads(), "kind": "port",
           "sample": "%s of the scene through all three stages, FP64, %d rep(s); frames = tiles / 78,408" % (
               S["what"], reps),
           "full_frame_ms": round(1e3 * dt / frames, 1), "small_256x256_ms": round(small_ms, 2)}
    parity = None
    try:
        hdr = cpu_pipeline(0, size=(1024, 768), peak=1e4, seed=31)
        parity = sample_parity(S, hdr=hdr)
    except Exception as e:  # the record is informative; the GPU tests are the parity gate
        parity = {"error": str(e).splitlines()[0][:200]}
    return rec, parity


def reference_kernels(S, frames=10, warmup=2):
    """The reference's own CUDA kernels (src/TileProcessor.cuh), compiled for
    sm_100a from the reference checkout (oracle/_ref), on the same frame:
    convert_correct_tiles, correlate2D and generate_RBGA's kernels launched
    back to back on the default stream (the host reads the texture-list counts
    and window back where the reference's dynamic-parallelism driver read them
    on the device), timed with CUDA events; also with the device synchronised
    after every launch, as the reference's harness runs them."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refgpu
    geom = S["geom"]
    if not torch.cuda.is_available():
        return {"unavailable": "no CUDA device"}
    if not refgpu.available(geom):
        return {"unavailable": "reference kernels for %dx%d not built (oracle/Makefile, make ref)" % (
            geom["img_width"], geom["img_height"])}
    dev = "cuda"
    TX, TY, TYA = S["TX"], S["TY"], S["TYA"]
    ptrs = lambda ts: torch.tensor([x.data_ptr() for x in ts], dtype=torch.int64, device=dev)
    images = [torch.from_numpy(S["pitched"][c]).to(dev) for c in range(4)]
    kernels = [torch.from_numpy(np.ascontiguousarray(S["kern"][c])).to(dev) for c in range(4)]
    extras = [torch.from_numpy(np.ascontiguousarray(S["extra"][c])).to(dev) for c in range(4)]
    clt = [torch.zeros(TX * TY * 768, dtype=torch.float32, device=dev) for _ in range(4)]
    p_img, p_ker, p_ext, p_clt = ptrs(images), ptrs(kernels), ptrs(extras), ptrs(clt)
    tasks = torch.from_numpy(np.ascontiguousarray(S["tasks"]).view(np.int32).reshape(-1, 10).copy()).to(dev)
    n, idx = S["ntiles"], torch.from_numpy(S["corr_idx"]).to(dev)
    stride = (2 * CORR_RADIUS + 1) ** 2
    corrs = torch.zeros((len(S["corr_idx"]), stride), dtype=torch.float32, device=dev)
    rstride = (TX + 1) * 8
    rgba = torch.zeros(((TY + 1) * 8 * 4 + 8, rstride), dtype=torch.float32, device=dev)
    lst = torch.zeros(TX * TYA + 256, dtype=torch.int32, device=dev)
    cnt = torch.zeros(8, dtype=torch.int32, device=dev)
    woi = torch.zeros(4, dtype=torch.int32, device=dev)
    po = torch.from_numpy(np.ascontiguousarray(S["port_offsets"], np.float32).reshape(-1)).to(dev)
    t = TEXTURE
    stages = {
        "convert": lambda: refgpu.call(geom, "ref_convert_correct_tiles", p_ext.data_ptr(), p_ker.data_ptr(),
                                       p_img.data_ptr(), tasks.data_ptr(), p_clt.data_ptr(), S["dstride"], n, 0),
        "correlate": lambda: refgpu.call(geom, "ref_correlate2D", p_clt.data_ptr(), 3, .25, .25, .5, FAT_ZERO,
                                         len(S["corr_idx"]), idx.data_ptr(), stride, CORR_RADIUS, corrs.data_ptr()),
        "texture": lambda: refgpu.call(geom, "ref_generate_RBGA", tasks.data_ptr(), n, lst.data_ptr(),
                                       cnt.data_ptr(), woi.data_ptr(), TX, TY, p_clt.data_ptr(), po.data_ptr(),
                                       t["colors"], t["is_lwir"], t["min_shot"], t["scale_shot"], t["diff_sigma"],
                                       t["diff_threshold"], t["min_agree"], t["weight0"], t["weight1"],
                                       t["weight2"], t["dust_remove"], 0, rstride, rgba.data_ptr()),
    }

    def timed(sync):
        refgpu.call(geom, "ref_set_sync", 1 if sync else 0)
        try:
            for _ in range(warmup):
                for f in stages.values():
                    f()
            torch.cuda.synchronize()
            ev = {k: [] for k in stages}
            for _ in range(frames):
                for k, f in stages.items():
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record()
                    f()
                    b.record()
                    ev[k].append((a, b))
            torch.cuda.synchronize()
        finally:
            refgpu.call(geom, "ref_set_sync", 1)
        st = {k: sum(a.elapsed_time(b) for a, b in v) / frames for k, v in ev.items()}
        return {"ms_per_frame": round(sum(st.values()), 4), "frames_per_s": round(1e3 / sum(st.values()), 2),
                "stages_ms": {k: round(v, 4) for k, v in st.items()}}

    out = {"what": "the reference's CUDA kernels compiled for sm_100a (oracle/_ref), same frame, CUDA events, "
                   "%d frames after %d" % (frames, warmup)}
    out["back_to_back"] = timed(False)
    out["synchronised_per_launch"] = timed(True)
    return out


def run_reference(args, rank, world, pg):
    if rank != 0:
        return None
    # one whole frame per step: the frame the B200 arm's rank 0 runs
    S = cpu_pipeline(0, size=(WIDTH, HEIGHT))
    O, step = S["O"], S["step"]
    for _ in range(args.warmup):
        step()
    t = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t) / args.steps
    v = S["ntiles"] / TILES / dt
    out = {
        "metric": METRIC, "value": round(v, 5), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * dt, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded plane scene, centred PSF kernels)",
        "impl": "reference",
        "config": bench_config(world),
        "frames_per_step": 1,
        "cpu_baseline": {"value": round(v, 5), "unit": UNIT, "cores": O.get_threads(), "kind": "port",
                         "sample": "%s per step through all three stages, FP64" % S["what"]},
        "e2e": {"value": round(v, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_reference_kernels:
        try:
            out["reference_kernels"] = reference_kernels(S)
        except Exception as e:  # beside the line, never instead of it
            out["reference_kernels"] = {"unavailable": str(e).splitlines()[0][:200]}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--frames-per-step", type=int, default=FRAMES_PER_STEP,
                    help="passes of the frame in one timed step")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-sample-tiles", type=int, default=20000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-kernels", action="store_true",
                    help="reference arm: skip the rebuilt reference kernels' GPU timing")
    ap.add_argument("--no-batched", action="store_true", help="skip the 64-frame batched workload")
    ap.add_argument("--frame", default="%dx%d" % (WIDTH, HEIGHT),
                    help="frame size WxH of the main workload (other sizes for profiling captures only)")
    ap.add_argument("--no-tune", action="store_true", help="built-in launch shapes instead of tuned ones")
    ap.add_argument("--shapes", default="", help="fixed launch shapes, e.g. convert=8,correlate=6,textures=4")
    ap.add_argument("--child", default="", choices=["", "precision-timing", "precision-parity"],
                    help="internal: one measurement in a subprocess of the main arm")
    args = ap.parse_args()
    if args.child:
        fn = child_precision_timing if args.child == "precision-timing" else child_precision_parity
        print(json.dumps(fn(args)))
        return
    if args.impl == "reference":
        # CPU arm: rank 0 alone runs it, the other ranks exit without work
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
        if rank == 0:
            print(json.dumps(run_reference(args, rank, world, None)))
        return
    rank, world, local, pg = dist_setup(args)
    try:
        out = run_b200(args, rank, world, local, pg)
        if rank == 0 and out is not None:
            print(json.dumps(out))
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
