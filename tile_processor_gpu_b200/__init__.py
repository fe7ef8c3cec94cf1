"""B200-native (sm_100a) frequency-domain tile processor.

A from-scratch implementation of the hot path of mfkiwl/tile_processor_gpu
(Bayer tile fetch -> aberration correction and fractional shift in the complex
lapped transform -> pairwise phase correlation -> inverse-CLT textures) behind
the reference's kernel interface.  The compute lives in libtp_b200.so (C ABI:
include/tp_b200.h); this package holds the host-side mirror of the reference's
entry points (`api`), seeded synthetic inputs (`synth`) and the build
(`build`).
"""
from . import synth  # noqa: F401

__all__ = ["api", "synth", "build"]


def __getattr__(name):
    # torch-dependent modules are imported on first use
    if name in ("api", "build"):
        import importlib
        return importlib.import_module(__name__ + "." + name)
    raise AttributeError(name)
