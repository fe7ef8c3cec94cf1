"""CPU tests of the C ABI: the library loads, exports every declared entry
point, and rejects invalid arguments on the host before touching a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tp_b200.h")


def declared_functions():
    with open(HEADER) as fh:
        src = fh.read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(tp_\w+)\s*\(", src, flags=re.M)))


def test_exports_every_declared_symbol(native):
    names = declared_functions()
    assert len(names) >= 16
    for n in names:
        assert hasattr(native, n), n


def test_struct_layouts():
    from tile_processor_gpu_b200.synth import TASK_DTYPE
    from tile_processor_gpu_b200._native import TpGeometry
    assert TASK_DTYPE.itemsize == 40          # struct tp_task with NUM_CAMS = 4
    assert ctypes.sizeof(TpGeometry) == 8 * 4


def test_version(native):
    from tile_processor_gpu_b200 import _native
    assert "sm_100a" in _native.version()


def _geom(**kw):
    from tile_processor_gpu_b200 import api
    d = dict(img_width=256, img_height=256)
    d.update(kw)
    return api.Geometry(**d)


def _code(fn):
    from tile_processor_gpu_b200 import _native
    with pytest.raises(_native.TpError) as ei:
        fn()
    return ei.value.code


P = ctypes.c_void_p


def test_rejects_bad_geometry(native):
    from tile_processor_gpu_b200 import _native as N
    fake = P(0x1000)
    for g in (_geom(img_width=250), _geom(img_height=16), _geom(image_rows=100), _geom(border_mode=3),
              _geom(kernels_lstep=0)):
        code = _code(lambda: N.call("tp_correlate2D", g.ptr, fake, 3, 1.0, 1.0, 1.0, 0.1, 4, fake, 225, 7, fake, None))
        assert code == N.TP_ERR_GEOMETRY


def test_rejects_bad_arguments(native):
    from tile_processor_gpu_b200 import _native as N
    g = _geom()
    fake = P(0x1000)
    # correlation radius above 7, colors 2, stride below (2r+1)^2, NULL output
    assert _code(lambda: N.call("tp_correlate2D", g.ptr, fake, 3, 1., 1., 1., .1, 4, fake, 225, 8, fake, None)) == N.TP_ERR_ARG
    assert _code(lambda: N.call("tp_correlate2D", g.ptr, fake, 2, 1., 1., 1., .1, 4, fake, 225, 7, fake, None)) == N.TP_ERR_ARG
    assert _code(lambda: N.call("tp_correlate2D", g.ptr, fake, 3, 1., 1., 1., .1, 4, fake, 224, 7, fake, None)) == N.TP_ERR_ARG
    assert _code(lambda: N.call("tp_correlate2D", g.ptr, fake, 3, 1., 1., 1., .1, 4, fake, 225, 7, None, None)) == N.TP_ERR_ARG
    # convert: negative count, narrow stride, NULL pointer arrays
    assert _code(lambda: N.call("tp_convert_correct_tiles", g.ptr, fake, fake, fake, fake, fake, 256, -1, 0, None)) == N.TP_ERR_ARG
    assert _code(lambda: N.call("tp_convert_correct_tiles", g.ptr, fake, fake, fake, fake, fake, 200, 4, 0, None)) == N.TP_ERR_ARG
    assert _code(lambda: N.call("tp_convert_correct_tiles", g.ptr, None, fake, fake, fake, fake, 256, 4, 0, None)) == N.TP_ERR_ARG
    # imclt: bad color, parity, stride below W + 8
    assert _code(lambda: N.call("tp_imclt_rbg", g.ptr, fake, fake, 3, 0, 0, 300, None)) == N.TP_ERR_ARG
    assert _code(lambda: N.call("tp_imclt_rbg", g.ptr, fake, fake, 0, 2, 0, 300, None)) == N.TP_ERR_ARG
    assert _code(lambda: N.call("tp_imclt_rbg", g.ptr, fake, fake, 0, 0, 0, 260, None)) == N.TP_ERR_ARG
    # textures: zero sigma, too narrow tile stride for keep_weights
    args = (3, 0, 10., 3., 1.5, 10., 3., .3, .1, .6, 1)
    assert _code(lambda: N.call("tp_textures_accumulate", g.ptr, None, fake, 4, fake, fake, 3, 0, 10., 3., 0.0, 10., 3.,
                                .3, .1, .6, 1, 0, 0, None, 1024, fake, None)) == N.TP_ERR_ARG
    assert _code(lambda: N.call("tp_textures_accumulate", g.ptr, None, fake, 4, fake, fake, *args, 1, 0, None, 1024,
                                fake, None)) == N.TP_ERR_ARG
    # a colour count other than 1 or 3 (the texture kernels are built per
    # count); the shot-noise step without a positive min_shot
    for bad in ((2,) + args[1:], (3, 0, 0.0, 3.) + args[4:], (3, 0, -1.0, 3.) + args[4:]):
        assert _code(lambda: N.call("tp_textures_accumulate", g.ptr, None, fake, 4, fake, fake, *bad, 0, 0, None, 1024,
                                    fake, None)) == N.TP_ERR_ARG
    # RGBA output without a window of interest
    assert _code(lambda: N.call("tp_textures_accumulate", g.ptr, None, fake, 4, fake, fake, *args, 0, 300, fake, 0,
                                None, None)) == N.TP_ERR_ARG
    # list extent larger than the tile grid
    assert _code(lambda: N.call("tp_prepare_texture_list", g.ptr, fake, 4, fake, fake, fake, 33, 32, None)) == N.TP_ERR_ARG
    # generate_RBGA stride below (tilesx + 1) * 8
    assert _code(lambda: N.call("tp_generate_RBGA", g.ptr, fake, 4, fake, fake, fake, 32, 32, fake, fake, *args, 0,
                                263, fake, None)) == N.TP_ERR_ARG
    # disparity fit: radius above 7, mode 3, stride below (2r+1)^2, NULL output
    assert _code(lambda: N.call("tp_disparity_fit", g.ptr, fake, 225, 8, 4, fake, fake, 63, 0, fake, fake,
                                None)) == N.TP_ERR_ARG
    assert _code(lambda: N.call("tp_disparity_fit", g.ptr, fake, 225, 7, 4, fake, fake, 63, 3, fake, fake,
                                None)) == N.TP_ERR_ARG
    assert _code(lambda: N.call("tp_disparity_fit", g.ptr, fake, 200, 7, 4, fake, fake, 63, 0, fake, fake,
                                None)) == N.TP_ERR_ARG
    assert _code(lambda: N.call("tp_disparity_fit", g.ptr, fake, 225, 7, 4, fake, fake, 63, 0, None, fake,
                                None)) == N.TP_ERR_ARG
    # no-alloc generate_RBGA: a frame whose list exceeds the library's scratch
    big = _geom(img_width=8192, img_height=8192)
    assert _code(lambda: N.call("tp_generate_RBGA_noalloc", big.ptr, fake, 4, 1024, 1024, fake, fake, *args, 0,
                                8200, fake, None)) == N.TP_ERR_ARG
    assert "scratch" in N.last_error()
    # tensor-core inference: feature rows must start on 16-byte boundaries (TMA strides)
    for ldx, xp in ((1350, fake), (1353, fake), (1352, P(0x1004))):
        assert _code(lambda: N.call("tp_mlp_infer_tc", 10, xp, ldx, fake, fake, fake, fake, fake, fake, fake, None,
                                    None)) == N.TP_ERR_ARG
        assert "16-byte" in N.last_error()
    assert _code(lambda: N.call("tp_mlp_infer_tc", 10, fake, 1349, fake, fake, fake, fake, fake, fake, fake, None,
                                None)) == N.TP_ERR_ARG
    # LPF table index
    v = np.zeros(64, np.float32)
    assert _code(lambda: N.call("tp_set_lpf", 6, v.ctypes.data_as(P))) == N.TP_ERR_ARG
    assert "lpf" in N.last_error()


def test_launch_shapes(native):
    """Grid caps of the stage kernels: defaults, set, reset, bounds."""
    from tile_processor_gpu_b200 import _native as N, autotune as A
    assert [A.get_shape(k) for k in ("convert", "correlate", "textures")] == [8, 8, 7]
    A.set_shape("correlate", 12)
    assert A.get_shape("correlate") == 12
    A.reset()
    assert A.get_shape("correlate") == 8
    for kernel, v in ((3, 4), (-1, 4), (0, 33), (0, -1)):
        assert _code(lambda: N.call("tp_set_launch_shape", kernel, v)) == N.TP_ERR_ARG
    assert _code(lambda: N.call("tp_get_launch_shape", 7)) == N.TP_ERR_ARG
    assert A.get_shape("convert") == 8


def test_tuner_keeps_the_fastest_cap(native, monkeypatch):
    """autotune.tune times the workload under each candidate cap (here a fake
    timer that reads the cap in force) and leaves the fastest one set."""
    from tile_processor_gpu_b200 import autotune as A
    fake_ms = {4: 0.41, 6: 0.43, 8: 0.39, 12: 0.385, 16: 0.40}
    seen = []
    monkeypatch.setattr(A, "time_ms", lambda run, repeats, warmup: (seen.append(A.get_shape("correlate")),
                                                                     fake_ms[A.get_shape("correlate")])[1])
    try:
        best, times = A.tune("correlate", run=lambda: None)
        assert best == 12 and A.get_shape("correlate") == 12
        assert seen == list(A.CANDIDATES["correlate"]) and times == fake_ms
        best, _ = A.tune("correlate", run=lambda: None, candidates=(16, 4))
        assert best == 16 and A.get_shape("correlate") == 16
    finally:
        A.reset()
    assert A.get_shape("correlate") == 8
    # the tuner never steps off the built-in shape: each default is a candidate
    for k in A.KERNELS:
        assert A.get_shape(k) in A.CANDIDATES[k]


def test_zero_work_is_ok_without_gpu(native):
    """Empty lists return before any launch."""
    from tile_processor_gpu_b200 import _native as N
    g = _geom()
    fake = P(0x1000)
    assert N.call("tp_correlate2D", g.ptr, fake, 3, 1., 1., 1., .1, 0, None, 225, 7, None, None) == 0
    assert N.call("tp_convert_correct_tiles", g.ptr, fake, fake, fake, None, fake, 256, 0, 0, None) == 0
    assert N.call("tp_disparity_fit", g.ptr, None, 225, 7, 0, None, None, 63, 0, None, None, None) == 0
    assert N.call("tp_textures_accumulate", g.ptr, None, fake, 0, None, None, 3, 0, 10., 3., 1.5, 10., 3., .3, .1, .6, 1,
                  0, 0, None, 0, None, None) == 0


def test_library_never_ends_the_process(native):
    """Errors come back as status codes: the library imports no function that
    ends the caller's process (a device-only helper called from host code
    compiles to such a call)."""
    import shutil
    import subprocess
    nm = shutil.which("nm")
    if nm is None:
        pytest.skip("nm not available")
    from tile_processor_gpu_b200 import _native
    out = subprocess.run([nm, "-D", "--undefined-only", _native.LIB_PATH], capture_output=True, text=True).stdout
    names = {ln.split()[-1].split("@")[0] for ln in out.splitlines() if ln.strip()}
    assert not names & {"exit", "_exit", "_Exit", "abort", "quick_exit"}, sorted(names & {"exit", "_exit", "abort"})
