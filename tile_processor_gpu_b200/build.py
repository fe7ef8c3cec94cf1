"""In-tree build of libtp_b200.so for sm_100a (nvcc, no JIT cache).

``python -m tile_processor_gpu_b200.build`` or ``build()`` from Python.  The
library is rebuilt when any source under csrc/ or include/ is newer than it.
"""
import glob
import os
import shutil
import subprocess
import sys

_HERE = os.path.dirname(os.path.abspath(__file__))
_ROOT = os.path.dirname(_HERE)
CSRC = os.path.join(_HERE, "csrc")
OUT = os.path.join(_HERE, "libtp_b200.so")

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]


def nvcc_path():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
                  glob.glob(os.path.join(CSRC, "*.cpp")) + glob.glob(os.path.join(CSRC, "*.inc")) +
                  glob.glob(os.path.join(_ROOT, "include", "*.h")))


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(s) > t for s in sources())


def build(force=False, verbose=False):
    """Compile csrc/tp_api.cu (which includes every kernel) and the host
    helpers csrc/tp_io.cpp into libtp_b200.so."""
    if not force and not needs_build():
        return OUT
    cmd = [nvcc_path()] + ARCH_FLAGS + NVCC_FLAGS + ["-o", OUT + ".tmp", os.path.join(CSRC, "tp_api.cu"),
                                                     os.path.join(CSRC, "tp_io.cpp")]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose:
        print(res.stderr)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
