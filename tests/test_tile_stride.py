"""Host-only check (compiled with nvcc, run on the CPU) that the tile row
strides of the line FFTs leave no shared-memory bank conflict in any access
group of the tiles -- half-warps of complex64, quarter-warps of complex128
(tests/cpp/tile_stride_check.cu)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_tile_strides_are_conflict_free(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    exe = tmp_path / "tile_stride_check"
    subprocess.run([nvcc, "-std=c++17", "-O1", "-I", os.path.join(ROOT, "spectral_upcxx_b200", "csrc"),
                    os.path.join(HERE, "cpp", "tile_stride_check.cu"), "-o", str(exe)],
                   check=True, capture_output=True, timeout=300)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout
    assert r.stdout.count("conflicting accesses: 0") == 12, r.stdout
