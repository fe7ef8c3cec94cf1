"""One frame split by tile rows (sharding.row_bands), the bands run one after
another on one GPU: each band's texture goes through tp_generate_RBGA_rows
with its tasks plus one tile row above and below, and the bands' own rows
plus the 8-row strips they add below themselves are overlap-added into one
image.  It must equal generate_RBGA on the whole frame (to the summation
order of the strip pixels), on a dense frame and on a sparse one whose
window of interest does not start at the frame's corner."""
import numpy as np
import pytest

from cases import Case, blob_mask

pytestmark = pytest.mark.gpu


def _whole_and_bands(case, bands):
    import torch
    import gpu_runner as R
    from tile_processor_gpu_b200 import api, sharding as S
    fr = R.Frame(case)
    R.convert(fr)
    p = R.TEX
    c = case
    stride = (c.TX + 1) * 8 + 40
    rows = (c.TY + 1) * 8 * (p["colors"] + 1)

    def buffers():
        return (torch.zeros(c.TX * c.TYA + 256, dtype=torch.int32, device="cuda"),
                torch.zeros(8, dtype=torch.int32, device="cuda"), torch.zeros(4, dtype=torch.int32, device="cuda"),
                torch.full((rows + 8, stride), 3.0, dtype=torch.float32, device="cuda"))

    args = (p["min_shot"], p["scale_shot"], p["diff_sigma"], p["weight0"], p["weight1"], p["weight2"],
            p["dust_remove"])
    idx, cnt, woi, whole = buffers()
    tasks = api.tasks_to_device(c.tasks, "cuda")
    api.generate_RBGA(fr.g, tasks, c.num_tiles, idx, cnt, woi, c.TX, c.TY, fr.p_clt, fr.port_offsets, p["colors"],
                      p["is_lwir"], p["min_shot"], p["scale_shot"], p["diff_sigma"], p["diff_threshold"],
                      p["min_agree"], p["weight0"], p["weight1"], p["weight2"], p["dust_remove"], 0, stride, whole)
    torch.cuda.synchronize()
    woi_w = woi.cpu().numpy()
    slices = p["colors"] + 1
    wh = (int(woi_w[3]) + 1) * 8
    whole_np = whole.cpu().numpy()[:slices * wh].reshape(slices, wh, stride)
    # the bands, overlap-added in frame pixel coordinates
    frame_rows = (c.TY + 1) * 8
    out = np.zeros((slices, frame_rows, stride + 8 * c.TX), np.float64)
    for first, last, _ in bands:
        if first == last:
            continue
        bt = S.band_tasks(c.tasks, first, last, c.TY)
        if not bt.size:
            continue
        idx, cnt, woi, img = buffers()
        api.generate_RBGA_rows(fr.g, api.tasks_to_device(bt, "cuda"), bt.size, idx, cnt, woi, c.TX, c.TY, fr.p_clt,
                               fr.port_offsets, p["colors"], *args, stride, img, first, last)
        torch.cuda.synchronize()
        wb = woi.cpu().numpy()
        bh = (int(wb[3]) + 1) * 8
        im = img.cpu().numpy()[:slices * bh].reshape(slices, bh, stride)
        r = S.band_image_rows(wb, first, last, c.TY)
        x0, bw = 8 * int(wb[0]), (int(wb[2]) + 1) * 8  # the band's window (the rest of its buffer is not written)
        for part in ("own", "send"):
            l0, g0, n = r[part]
            if n:
                out[:, g0:g0 + n, x0:x0 + bw] += im[:, l0:l0 + n, :bw]
    y0, x0 = 8 * int(woi_w[1]), 8 * int(woi_w[0])
    want = np.zeros_like(out)
    want[:, y0:y0 + wh, x0:x0 + stride] = whole_np
    # compare inside the whole frame's window (the caller's buffer outside it is not written)
    ww = (int(woi_w[2]) + 1) * 8
    sl = (slice(None), slice(y0, y0 + wh), slice(x0, x0 + ww))
    return out[sl], want[sl]


@pytest.mark.parametrize("nbands", [2, 3, 5])
def test_dense_frame_bands(native, nbands):
    from tile_processor_gpu_b200 import sharding as S
    c = Case(256, 192, seed=31)
    got, want = _whole_and_bands(c, S.row_bands(c.TY, nbands))
    scale = np.abs(want).max()
    err = np.abs(got - want).max() / scale
    print("\n%d bands: max |stitched - whole| / max = %.2e" % (nbands, err))
    assert err < 1e-6


def test_sparse_frame_bands(native):
    from tile_processor_gpu_b200 import sharding as S
    rng = np.random.default_rng(4)
    mask = blob_mask(rng, 32, 24, 0.35)
    mask[:3, :] = False
    mask[:, :2] = False
    c = Case(256, 192, seed=32, mask=mask)
    got, want = _whole_and_bands(c, S.row_bands(c.TY, 4))
    err = np.abs(got - want).max() / np.abs(want).max()
    print("\nsparse, 4 bands: max |stitched - whole| / max = %.2e" % err)
    assert err < 1e-6
