"""The butterfly forms of the 8-point DCT-II / DST-II / DCT-IV / DST-IV used
by every kernel (tp_common.cuh) against their closed forms in double
precision, on the host: 100,000 random vectors (a fifth of them scaled by
1e4), the error within 1e-6 of the vector's largest element (the plain float
matrix product reaches ~3e-7)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    return None


def test_butterfly_transforms(tmp_path):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc not found")
    exe = str(tmp_path / "host_transforms")
    src = os.path.join(ROOT, "tests", "host_transforms.cu")
    inc = os.path.join(ROOT, "tile_processor_gpu_b200", "csrc")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-I", inc, "-o", exe, src], check=True, capture_output=True)
    res = subprocess.run([exe], capture_output=True, text=True)
    print(res.stdout)
    assert res.returncode == 0, res.stdout
