"""Writes tests/golden/corpus.stormbin and tests/golden/corpus.stormpack with
the reference's OWN tools, so the loaders are pinned to what the reference
writes rather than to a restatement of its layout:

  * STORMBIN: tools/sets2bin.py (adjacency input: one set per line),
  * STORMPACK: tools/pack.cpp compiled from the reference sources, run on
    that STORMBIN file (stride 1, card_max_array 32: every stored
    representation appears -- bitmap, u16 array, u16 runs, full, empty);
  * tests/golden/threshold_hits.json: the reference's thresholded mode,
    bench/bench_threshold.cpp compiled with kernels/*.cpp, run on the
    STORMBIN file at several Jaccard thresholds; its CSV line's hit count
    (pairs i < j with |Xi & Xj| > 0 and Jaccard >= t) per threshold.

The sets are regenerated from the same seed by corpus_sets() in the tests.
Run in a container that has the reference tree (REF below); the outputs are
committed. Test infrastructure only.
"""
import glob
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

REF = os.environ.get("STORM_REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))
UNIVERSE = 5008
THRESHOLDS = (0.0, 0.001, 0.01, 0.05, 0.1, 0.3, 0.6)


def corpus_sets():
    """Seeded rows over a 5008-bit universe: sparse rows, dense rows, short
    runs, one full row. (An empty row cannot be expressed in the adjacency
    input; the STORMPACK file gets one from pack.cpp only if a row is empty.)"""
    g = np.random.Generator(np.random.PCG64(20261204))
    rows = []
    for k in range(60):
        kind = k % 4
        if kind == 0:
            card = int(g.integers(1, 30))
        elif kind == 1:
            card = int(g.integers(200, 2500))
        elif kind == 2:
            start = int(g.integers(0, UNIVERSE - 40))
            rows.append(np.arange(start, start + int(g.integers(8, 30)), dtype=np.uint32))
            continue
        else:
            card = int(g.integers(31, 120))
        rows.append(np.sort(g.choice(UNIVERSE, size=card, replace=False)).astype(np.uint32))
    rows.append(np.arange(UNIVERSE, dtype=np.uint32))
    return rows


def main():
    rows = corpus_sets()
    with tempfile.TemporaryDirectory() as tmp:
        adj = os.path.join(tmp, "sets.txt")
        with open(adj, "w") as f:
            for r in rows:
                f.write(" ".join(str(int(x)) for x in r) + "\n")
        binf = os.path.join(HERE, "corpus.stormbin")
        subprocess.run([sys.executable, os.path.join(REF, "tools", "sets2bin.py"), adj, "-o", binf,
                        "--format", "adjacency", "--universe", str(UNIVERSE)], check=True)
        exe = os.path.join(tmp, "pack")
        subprocess.run(["g++", "-O2", "-std=c++17", "-I", REF, os.path.join(REF, "tools", "pack.cpp"),
                        os.path.join(REF, "kernels", "storm_repr.cpp"), "-o", exe], check=True)
        subprocess.run([exe, binf, os.path.join(HERE, "corpus.stormpack"), "1", "32"], check=True)
        thr = os.path.join(tmp, "bench_threshold")
        srcs = sorted(glob.glob(os.path.join(REF, "kernels", "*.cpp")))
        subprocess.run(["g++", "-O2", "-std=c++17", "-march=native", "-I", REF,
                        os.path.join(REF, "bench", "bench_threshold.cpp")] + srcs + ["-o", thr], check=True)
        hits = {}
        for t in THRESHOLDS:
            out = subprocess.run([thr, "--file", binf, "--rows", "1000", "--t", repr(t), "--repeats", "1", "--csv"],
                                 check=True, capture_output=True, text=True).stdout.strip().splitlines()[-1]
            fields = out.split(",")    # corpus,t,N,pairs,hits,candidates,...,correct
            assert fields[-1] == "1", out
            hits[repr(t)] = int(fields[4])
        with open(os.path.join(HERE, "threshold_hits.json"), "w") as f:
            json.dump(hits, f, indent=1)


if __name__ == "__main__":
    main()
