"""Builds and runs the host-only C++ checks under tests/ (*.cu compiled with
nvcc against the library's headers and libstorm_b200.so; no GPU needed)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "stormbitmaps-internal_b200")


def nvcc():
    p = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    if os.path.exists(p):
        return p
    p = shutil.which("nvcc")
    if p is None:
        pytest.skip("nvcc not available")
    return p


def run_host_check(name, timeout=300):
    """Compile tests/<name>.cu, run it, return its stdout (asserts exit 0)."""
    out = os.path.join(ROOT, "_build", name)
    os.makedirs(out, exist_ok=True)
    exe = os.path.join(out, name)
    subprocess.run([nvcc(), "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", os.path.join(ROOT, "include"), "-I", os.path.join(PKG, "csrc"),
                    os.path.join(ROOT, "tests", name + ".cu"), "-o", exe,
                    "-L", PKG, "-lstorm_b200", "-Xlinker", "-rpath", "-Xlinker", PKG],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout
