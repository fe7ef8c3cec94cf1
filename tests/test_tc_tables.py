"""CPU checks of the tensor-core precision forms' transform tables.

Each stage's four quadrant transforms are 64 x 64 matrices K_q = V_q (x) H_q
of the 8-point DCT-IV / DST-IV / DCT-II / DST-II (the oracle's matrices); the
library stores them split into two 16-bit halves (hi, lo) as 128-byte-
swizzled shared-memory images.  Decoding an image must give back hi + lo = K_q
to the precision of the split, and hi alone must be K_q rounded to the
format."""
import numpy as np
import pytest


def _decode(img, fmt):
    """image -> (hi, lo) float64 [4][64][64] (rows N = (i, j), columns K = (m, n))"""
    import torch
    b = img.astype(np.uint16)
    if fmt == 0:
        vals = b.view(np.float16).astype(np.float64)
    else:
        vals = torch.from_numpy(b.view(np.int16).copy()).view(torch.bfloat16).to(torch.float64).numpy()
    hi = np.zeros((4, 64, 64))
    lo = np.zeros((4, 64, 64))
    for q in range(4):
        for r in range(64):
            for k in range(64):
                off = r * 128 + (((k >> 3) ^ (r & 7)) << 4) + ((k & 7) << 1)
                hi[q, r, k] = vals[(q * 8192 + off) // 2]
                lo[q, r, k] = vals[((4 + q) * 8192 + off) // 2]
    return hi, lo


def _kinds(stage, q):
    if stage == 0:
        return 2 + (q >> 1), 2 + (q & 1)
    if stage == 1:
        return q >> 1, q & 1
    return (0, q) if q < 2 else (None, None)


@pytest.mark.parametrize("stage", [0, 1, 2])
@pytest.mark.parametrize("fmt", [0, 1])
def test_split_tables(native, oracle, stage, fmt):
    from tile_processor_gpu_b200 import api
    hi, lo = _decode(api.tc_table_image(fmt, stage), fmt)
    bits = 11 if fmt == 0 else 8
    for q in range(4):
        kv, kh = _kinds(stage, q)
        if kv is None:
            assert not hi[q].any() and not lo[q].any()
            continue
        K = np.kron(oracle.dtt_matrix(kv), oracle.dtt_matrix(kh))
        # hi is K rounded to the format: relative error below half an ulp
        nz = K != 0
        assert np.all(np.abs(hi[q] - K)[nz] <= np.abs(K[nz]) * 2.0 ** -bits * 1.0001)
        # hi + lo carries about twice the bits
        assert np.abs(hi[q] + lo[q] - K).max() <= np.abs(K).max() * 2.0 ** (-2 * bits) * 2
