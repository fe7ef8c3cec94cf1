"""Generate the golden fixtures from the reference's own kernels.

Runs the reference kernels rebuilt for sm_100a (oracle/_ref/libtp_ref_256x256.so,
built by `make -C oracle ref`) on a seeded 256x256 quad frame and stores small
subsets of every output:

    python tests/golden/make_golden.py OUTDIR        (needs a CUDA GPU)

The inputs are not stored: tests regenerate them from the seed with
tests/cases.py and check them against the stored SHA-256 digests, so any drift
of the generator is caught before outputs are compared.

Stored (float32 unless noted):
  clt      [16 tiles][4 cams][768]     convert_correct_tiles, selected tiles
  corr     [96][225]                   correlate2D of those tiles, 6 pairs, r=7
  corr_r4m [24][81]                    colors=1, r=4, 4 tiles x 6 pairs
  tex      [16][12][256]               textures_accumulate, keep_weights=1
  imclt    [3 colors][2 crops][40][40] imclt_rbg (4 passes, camera 0)
  rgba     [4 slices][2 crops][40][40] generate_RBGA over all tiles
  list_*   (int32)                     prepare_texture_list on a sparse mask
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests"), HERE]

from cases import Case, blob_mask  # noqa: E402

SEED = 11
SEL_TILES = [(0, 0), (31, 0), (0, 31), (31, 31), (15, 0), (0, 15), (31, 15), (15, 31), (30, 30), (1, 1),
             (7, 9), (20, 4), (12, 25), (26, 17), (5, 28), (16, 16)]
CROPS = [(0, 0), (216, 216)]  # (row, col) of the 40x40 crops
MASK_SEED = 12


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def golden_case():
    return Case(256, 256, seed=SEED, border_mode=0)


def sel_tile_ids(case):
    return np.array([ty * case.TX + tx for tx, ty in SEL_TILES], dtype=np.int64)


def sparse_tasks(case):
    rng = np.random.default_rng(MASK_SEED)
    m = blob_mask(rng, case.TX, case.TY, 0.3)
    return case.tasks[m.reshape(-1)].copy()


def input_digest(case):
    return digest(case.pitched, case.kernels, case.extra, case.tasks.view(np.int32))


def main(outdir):
    import torch
    import gpu_runner as R

    case = golden_case()
    fr = R.Frame(case)
    sel = sel_tile_ids(case)
    clt = R.convert(fr, impl="ref")
    out = {"input_sha256": np.array(input_digest(case))}
    out["clt"] = np.stack([np.stack([clt[c].reshape(-1, 768)[t] for c in range(4)]) for t in sel]).astype(np.float32)
    fr.set_clt(clt)
    idx = np.array([(int(t) << 8) | p for t in sel for p in range(6)], dtype=np.int32)
    out["corr"] = R.correlate(fr, idx, impl="ref")[:, :225].astype(np.float32)
    idx4 = idx[:24]
    out["corr_r4m"] = R.correlate(fr, idx4, colors=1, radius=4, impl="ref")[:, :81].astype(np.float32)
    tex_idx = np.array([(int(t) << 8) | (1 << 7) for t in sel], dtype=np.int32)
    out["tex"] = R.textures_tiles(fr, tex_idx, keep_weights=1, impl="ref").reshape(len(sel), 12, 256)
    img, dst = R.imclt_all(fr, impl="ref")
    H = case.H + 8
    out["imclt"] = np.stack([np.stack([img[col * H + r: col * H + r + 40, c: c + 40] for r, c in CROPS])
                             for col in range(3)]).astype(np.float32)
    rb, woi, stride, rows = R.rgba(fr, impl="ref")
    h = (woi[3] + 1) * 8
    out["rgba"] = np.stack([np.stack([rb[s * h + r: s * h + r + 40, c: c + 40] for r, c in CROPS])
                            for s in range(4)]).astype(np.float32)
    out["rgba_woi"] = woi.astype(np.int32)
    # sparse texture list
    st = sparse_tasks(case)
    case_s = Case(256, 256, seed=SEED, border_mode=0)
    case_s.tasks = st
    frs = R.Frame(case_s)
    tasks_o, lidx, counts, lwoi = R.texture_list(frs, impl="ref")
    out["list_task"] = tasks_o["task"].astype(np.int32)
    out["list_counts"] = counts.astype(np.int32)
    out["list_woi"] = lwoi.astype(np.int32)
    quarter = case.TX * (case.TYA >> 2)
    subl = []
    for q in range(4):
        inner = np.sort(lidx[q * quarter: q * quarter + counts[2 * q]])
        border = np.sort(lidx[(q + 1) * quarter - counts[2 * q + 1]: (q + 1) * quarter])
        subl += [inner, border]
    out["list_entries"] = np.concatenate(subl).astype(np.int32)
    os.makedirs(outdir, exist_ok=True)
    path = os.path.join(outdir, "ref_256x256_seed%d.npz" % SEED)
    np.savez_compressed(path, **out)
    print(path, {k: v.shape for k, v in out.items()})
    torch.cuda.synchronize()


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
