"""ctypes binding of libtp_b200.so (the C ABI in include/tp_b200.h).

The shared library is built in-tree by ``tile_processor_gpu_b200.build`` and
loaded from this package directory.  There is no fallback: if the library is
missing or does not load, every entry point raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtp_b200.so")

TP_OK = 0
TP_ERR_ARG = -1
TP_ERR_GEOMETRY = -2
TP_ERR_CUDA = -3
TP_ERR_UNSUPPORTED = -4
TP_ERR_NO_DEVICE = -5

TP_BORDER_REFERENCE = 0
TP_BORDER_CLAMP = 1


class TpGeometry(ctypes.Structure):
    _fields_ = [
        ("img_width", ctypes.c_int),
        ("img_height", ctypes.c_int),
        ("kernels_hor", ctypes.c_int),
        ("kernels_vert", ctypes.c_int),
        ("kernels_lstep", ctypes.c_int),
        ("image_rows", ctypes.c_int),
        ("border_mode", ctypes.c_int),
        ("debug_marks", ctypes.c_int),
    ]


class TpError(RuntimeError):
    def __init__(self, func, code, msg):
        super().__init__("%s failed (%d): %s" % (func, code, msg))
        self.code = code


_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float
_S = ctypes.c_size_t
_G = ctypes.POINTER(TpGeometry)

# name -> argtypes (restype is int for all compute entry points)
SIGNATURES = {
    "tp_convert_correct_tiles": [_G, _P, _P, _P, _P, _P, _S, _I, _I, _P],
    "tp_convert_correct_tiles_tma": [_G, _P, _P, _P, _P, _P, _S, _I, _I, _P],
    "tp_correlate2D": [_G, _P, _I, _F, _F, _F, _F, _S, _P, _S, _I, _P, _P],
    "tp_textures_accumulate": [_G, _P, _P, _S, _P, _P, _I, _I, _F, _F, _F, _F, _F, _F, _F, _F, _I, _I,
                               _S, _P, _S, _P, _P],
    "tp_imclt_rbg": [_G, _P, _P, _I, _I, _I, _S, _P],
    "tp_imclt_rbg_all": [_G, _P, _P, _S, _P],
    "tp_prepare_texture_list": [_G, _P, _I, _P, _P, _P, _I, _I, _P],
    "tp_clear_texture_rbga": [_G, _I, _I, _S, _P, _P],
    "tp_generate_RBGA": [_G, _P, _I, _P, _P, _P, _I, _I, _P, _P, _I, _I, _F, _F, _F, _F, _F, _F, _F, _F, _I,
                         _I, _S, _P, _P],
    "tp_generate_RBGA_noalloc": [_G, _P, _I, _I, _I, _P, _P, _I, _I, _F, _F, _F, _F, _F, _F, _F, _F, _I, _I, _S,
                                 _P, _P],
    "tp_generate_RBGA_rows": [_G, _P, _I, _P, _P, _P, _I, _I, _P, _P, _I, _F, _F, _F, _F, _F, _F, _I, _S, _P,
                              _I, _I, _P],
    "tp_process_frame": [_G, _P, _P, _P, _S, _P, _I, _I, _I, _F, _F, _F, _F, _I, _S, _P, _P, _F, _F, _F, _F, _F,
                         _F, _I, _P, _P, _P, _S, _P, _P, _P],
    "tp_disparity_fit": [_G, _P, _S, _I, _S, _P, _P, _I, _I, _P, _P, _P],
    "tp_psf_to_clt": [_P, _S, _P, _P],
    "tp_tasks_from_portsxy": [_P, _I, _I, _I, _P],
    "tp_corr_indices_from_tasks": [_P, _I, _I, _P],
    "tp_mlp_features": [_G, _P, _S, _I, _S, _P, _P, _S, _P],
    "tp_mlp_gemm": [_I, _I, _I, _P, _I, _I, _P, _I, _I, _F, _P, _I, _P, _P, _I, _P],
    "tp_mlp_gemm_tc": [_I, _I, _I, _P, _I, _I, _P, _I, _I, _F, _P, _I, _P, _P, _I, _P, _P],
    "tp_mlp_gelu_backward": [_I, _I, _I, _P, _P, _P, _P],
    "tp_mlp_colsum": [_I, _I, _I, _P, _F, _P, _P],
    "tp_mlp_nll": [_I, _P, _P, _P, _F, _P, _P, _P],
    "tp_mlp_pack": [_P, _P, _P, _P, _P],
    "tp_mlp_infer_tc": [_I, _P, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "tp_mlp_adam": [_S, _P, _P, _P, _P, _F, _F, _F, _F, _I, _P],
    "tp_mlp_combine": [_S, _P, _P, _F, _P, _P],
    "tp_set_lpf": [_I, _P],
    "tp_get_lpf": [_I, _P],
    "tp_reset_lpf": [],
    "tp_tiles_x": [_G],
    "tp_tiles_y": [_G],
    "tp_tiles_ya": [_G],
    "tp_set_launch_shape": [_I, _I],
    "tp_get_launch_shape": [_I],
    "tp_resident_ctas": [_I],
    "tp_correlate2D_tc": [_G, _P, _I, _F, _F, _F, _F, _S, _P, _S, _I, _P, _I, _P],
    "tp_convert_correct_tiles_tc": [_G, _P, _P, _P, _P, _P, _S, _I, _I, _I, _P],
    "tp_textures_accumulate_tc": [_G, _P, _P, _S, _P, _P, _I, _I, _F, _F, _F, _F, _F, _F, _F, _F, _I, _I,
                                  _S, _P, _S, _P, _P, _I, _P],
    "tp_generate_RBGA_tc": [_G, _P, _I, _P, _P, _P, _I, _I, _P, _P, _I, _I, _F, _F, _F, _F, _F, _F, _F, _F, _I,
                            _I, _S, _P, _P, _I, _P],
    "tp_tc_status": [_P, _I],
    "tp_tc_table_image": [_I, _I, _P],
}
STRING_FUNCS = ("tp_last_error", "tp_version")
# entry points returning a count (long long) instead of a status
COUNT_FUNCS = {"tp_read_floats": [ctypes.c_char_p, _P, _S], "tp_write_floats": [ctypes.c_char_p, _P, _S]}

_lib = None


def load():
    """Load libtp_b200.so once; raise if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libtp_b200.so not built (run tile_processor_gpu_b200.build.build()): %s" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, argtypes in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = ctypes.c_int
    for name in STRING_FUNCS:
        fn = getattr(lib, name)
        fn.argtypes = []
        fn.restype = ctypes.c_char_p
    for name, argtypes in COUNT_FUNCS.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = ctypes.c_longlong
    _lib = lib
    return lib


def call(name, *args):
    """Call a tp_* entry point; raise TpError on a negative status."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc < 0:
        raise TpError(name, rc, lib.tp_last_error().decode())
    return rc


def last_error():
    return load().tp_last_error().decode()


def version():
    return load().tp_version().decode()
