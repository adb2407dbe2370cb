"""Build libstorm_b200.so (all CUDA + host sources) for sm_100a, in-tree.

    python stormbitmaps-internal_b200/build.py [--verbose] [--ptxas-info]

Each csrc/*.cu / *.cpp is compiled to an object under _build/ (parallel,
skipped when up to date), then linked with nvcc into
stormbitmaps-internal_b200/libstorm_b200.so with the CUDA runtime linked
statically, so the library loads next to any PyTorch build.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build", "storm_b200")
LIB = os.path.join(HERE, "libstorm_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include")]
CUFLAGS = ARCH + COMMON + ["-lineinfo", "--expt-relaxed-constexpr"]


def _sources():
    out = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".cu", ".cpp")):
            out.append(os.path.join(CSRC, f))
    return out


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + [
        os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))
    ]


def _obj(src):
    return os.path.join(BUILD, os.path.basename(src) + ".o")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, ptxas_info=False, verbose=False):
    obj = _obj(src)
    if not _stale(obj, [src] + _headers()):
        return obj, ""
    cmd = [NVCC] + CUFLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC] + COMMON + ["-x", "c++", "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose=False, ptxas_info=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, ptxas_info, verbose), srcs))
    objs = [o for o, _ in results]
    if ptxas_info:
        for _, err in results:
            if err:
                print(err)
    if _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs + ["-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    a = ap.parse_args()
    if a.ptxas_info:
        for s in _sources():
            o = _obj(s)
            if os.path.exists(o):
                os.remove(o)
    print(build(verbose=a.verbose, ptxas_info=a.ptxas_info))
    sys.exit(0)
