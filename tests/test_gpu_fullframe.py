"""Full-frame (2592x1936 quad, 78,408 tiles) checks on the bench's own
workload: CLT and correlation parity with the reference kernels rebuilt for
sm_100a, and the stage-by-stage speed of the library against them (CUDA
events; the rebuilt reference synchronises the device after each of its
launches, as its harness does)."""
import os
import sys

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def pipe(native):
    sys.path.insert(0, ROOT)
    import bench
    import refgpu
    p = bench.FramePipeline(seed=100, device="cuda:0")
    if not refgpu.available(p.geom_d):
        pytest.skip("reference kernels for 2592x1936 not built")
    return p


def _time(fn, reps=5):
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def _ref_calls(p):
    import refgpu
    import bench
    t = bench.TEXTURE
    g = p.geom_d
    ref_corrs = torch.empty_like(p.corrs)
    ref_rgba = torch.empty_like(p.rgba)
    ref_tasks = p.api.tasks_to_device(p.tasks_np, "cuda:0")
    idx = torch.empty_like(p.tex_indices)
    cnt = torch.empty_like(p.num_tex)
    woi = torch.empty_like(p.woi)
    idx_big = torch.zeros(p.TX * p.TYA + 256, dtype=torch.int32, device="cuda:0")

    def convert():
        refgpu.call(g, "ref_convert_correct_tiles", p.p_extra.dev.data_ptr(), p.p_kernels.dev.data_ptr(),
                    p.p_images.dev.data_ptr(), ref_tasks.data_ptr(), p.p_clt.dev.data_ptr(), p.dstride,
                    p.num_tiles, 0)

    def correlate():
        refgpu.call(g, "ref_correlate2D", p.p_clt.dev.data_ptr(), 3, 0.25, 0.25, 0.5, bench.FAT_ZERO, p.num_corr,
                    p.corr_idx.data_ptr(), p.corr_stride, bench.CORR_RADIUS, ref_corrs.data_ptr())

    def texture():
        refgpu.call(g, "ref_generate_RBGA", ref_tasks.data_ptr(), p.num_tiles, idx_big.data_ptr(), cnt.data_ptr(),
                    woi.data_ptr(), p.TX, p.TY, p.p_clt.dev.data_ptr(), p.port_offsets.data_ptr(), t["colors"],
                    t["is_lwir"], t["min_shot"], t["scale_shot"], t["diff_sigma"], t["diff_threshold"],
                    t["min_agree"], t["weight0"], t["weight1"], t["weight2"], t["dust_remove"], 0, p.rgba_stride,
                    ref_rgba.data_ptr())

    return convert, correlate, texture, ref_corrs


def test_fullframe_parity_and_speed(pipe):
    p = pipe
    ref_convert, ref_correlate, ref_texture, ref_corrs = _ref_calls(p)
    # parity of the CLT and the correlations on the full frame
    ref_convert()
    torch.cuda.synchronize()
    clt_ref = [c.clone() for c in p.clt]
    p.convert()
    torch.cuda.synchronize()
    for a, b in zip(p.clt, clt_ref):
        err = (a - b).abs().max().item() / b.abs().max().item()
        assert err < 1e-5, err
    ref_correlate()
    p.correlate()
    torch.cuda.synchronize()
    err = (p.corrs - ref_corrs).abs().max().item() / ref_corrs.abs().max().item()
    assert err < 1e-5, err
    # speed, stage by stage
    mine = {"convert": _time(p.convert), "correlate": _time(p.correlate), "texture": _time(p.texture)}
    ref = {"convert": _time(ref_convert), "correlate": _time(ref_correlate), "texture": _time(ref_texture)}
    print("\nfull frame ms  b200 %s  reference-kernels %s  ratio %s" % (
        {k: round(v, 3) for k, v in mine.items()}, {k: round(v, 3) for k, v in ref.items()},
        {k: round(ref[k] / mine[k], 2) for k in mine}))
    for k in mine:
        assert mine[k] < ref[k], (k, mine[k], ref[k])
