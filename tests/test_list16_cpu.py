"""The list x list count the chunk kernel runs for list chunks that are not
strictly increasing (list16_ref.cuh), checked on the host against the
reference's own STORM_intersect_vector16_cardinality (SSE4.2 build, from
oracle/_ref) on seeded lists with repeats, unsorted entries and leading
zeros (tests/list16_check.cu); skipped when the reference is not built."""
import os

import pytest

from harness import ROOT, nvcc
import subprocess


@pytest.mark.timeout(600)
def test_blocked_list_count_matches_reference():
    ref = os.path.join(ROOT, "oracle", "_ref", "libstorm_ref.so")
    if not os.path.exists(ref):
        pytest.skip("reference library not built (oracle/_ref)")
    out = os.path.join(ROOT, "_build", "list16_check")
    os.makedirs(out, exist_ok=True)
    exe = os.path.join(out, "list16_check")
    subprocess.run([nvcc(), "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", os.path.join(ROOT, "stormbitmaps-internal_b200", "csrc"),
                    os.path.join(ROOT, "tests", "list16_check.cu"), "-o", exe, "-ldl"],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([exe, ref], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("identical"), r.stdout
