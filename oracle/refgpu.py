"""ctypes wrapper of the reference kernels rebuilt for sm_100a (oracle/_ref/).

TEST INFRASTRUCTURE ONLY.  oracle/Makefile (`make ref`) compiles the
reference's own CUDA sources, in place, with oracle/ref_shim.cu into one
library per frame geometry; this module loads the one matching a geometry and
calls its launchers with device pointers (ints).  `available(geom)` is False
when that library was not built (the parity tests then skip the
reference-kernel leg and keep the oracle leg).
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
_libs = {}

_P, _I, _F, _S = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_size_t
SIGS = {
    "ref_convert_correct_tiles": [_P, _P, _P, _P, _P, _S, _I, _I],
    "ref_correlate2D": [_P, _I, _F, _F, _F, _F, _S, _P, _S, _I, _P],
    "ref_textures_accumulate": [_P, _P, _S, _P, _P, _I, _I, _F, _F, _F, _F, _F, _F, _F, _F, _I, _I, _S, _P, _S, _P],
    "ref_imclt_rbg": [_P, _P, _I, _I, _I, _S],
    "ref_prepare_texture_list": [_P, _I, _P, _P, _P, _I, _I],
    "ref_generate_RBGA": [_P, _I, _P, _P, _P, _I, _I, _P, _P, _I, _I, _F, _F, _F, _F, _F, _F, _F, _F, _I, _I, _S, _P],
    "ref_tilesx": [], "ref_tilesy": [], "ref_tilesya": [], "ref_set_sync": [_I],
}


def path(geom):
    return os.path.join(_HERE, "_ref", "libtp_ref_%dx%d.so" % (geom["img_width"], geom["img_height"]))


def available(geom):
    std = geom["kernels_hor"] == geom["img_width"] // 16 + 2 and geom["kernels_vert"] == geom["img_height"] // 16 + 2
    return std and geom.get("kernels_lstep", 4) == 4 and os.path.exists(path(geom))


def lib(geom):
    p = path(geom)
    if p not in _libs:
        L = ctypes.CDLL(p)
        for n, a in SIGS.items():
            f = getattr(L, n)
            f.argtypes = a
            f.restype = ctypes.c_int
        _libs[p] = L
    return _libs[p]


def call(geom, name, *args):
    rc = getattr(lib(geom), name)(*args)
    if rc != 0:
        raise RuntimeError("%s returned %d" % (name, rc))
