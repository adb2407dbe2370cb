"""Host packing of STORM_t rows, checked without a GPU: the threaded bulk
packer (ChunkPack::add_rows) must lay out exactly what the row-by-row
packer (ChunkPack::add_row) does. tests/pack_identity.cu is compiled with
nvcc against the library's headers and libstorm_b200.so and run on the host."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "stormbitmaps-internal_b200")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


@pytest.mark.timeout(600)
def test_bulk_packer_matches_row_by_row(sb):
    if not os.path.exists(NVCC) and shutil.which("nvcc") is None:
        pytest.skip("nvcc not available")
    out = os.path.join(ROOT, "_build", "pack_identity")
    os.makedirs(out, exist_ok=True)
    exe = os.path.join(out, "pack_identity")
    subprocess.run([NVCC if os.path.exists(NVCC) else "nvcc", "-std=c++17", "-O2",
                    "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", os.path.join(ROOT, "include"), "-I", os.path.join(PKG, "csrc"),
                    os.path.join(ROOT, "tests", "pack_identity.cu"), "-o", exe,
                    "-L", PKG, "-lstorm_b200", "-Xlinker", "-rpath", "-Xlinker", PKG],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("identical"), r.stdout + r.stderr
