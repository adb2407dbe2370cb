"""All-pairs exact intersection cardinality on B200: the benchmark.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (one "step"): every pair i <= j of the large dense configuration --
N = 65536 rows x M = 262144 bits, bit iid Bernoulli(p) with p drawn per row
uniformly in [0.05, 0.5], packed as u64 (2 GiB in), u32 |Xi & Xj| for all
i <= j out (2,147,516,416 pairs, 8.6 GB) -- through the STORM_contiguous_t
interface of libstorm_b200.so.  Inputs are seeded synthetic data generated
on the GPU.  Metric: exact pairs per second (and ns per pair).

    value  device-resident: rows already in HBM, output stays in HBM; the
           timed region is the all-pairs call (CUDA events, max over ranks).
    e2e    through the C ABI with HOST buffers: each step takes the rows
           from pinned host memory and returns the whole triangle into
           pinned host memory, in one call
           (STORM_contig_pairw_intersect_matrix_from_host, copies and tiles
           overlapped); the same through add + matrix calls is reported
           beside it (e2e.two_calls).

Multi-GPU (torchrun): every rank runs its own instance (seed + rank); the
rows of different ranks are independent, so there is no data-path
collective ("scaling": "weak").  `--impl reference` times the reference's own
CPU kernel (oracle/_ref, built from the reference sources) on the host cores,
on a bounded row sample of the same workload, on rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes as C
import importlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_ROWS, M_BITS, P_RANGE, SEED = 65536, 262144, (0.05, 0.5), 0x5EED2
L2_BYTES = 126 * 1000 * 1000
# DRAM bytes per launch of the tensor-core kernel on the 65536 x 262144 workload:
# one ncu capture at 16384 x 262144 (10.710 GB read + 0.525 GB written), scaled
# by the pairs ratio 16 (tiles, and the rows they re-read, grow with the pairs).
TS_TRAFFIC_BENCH_WORKLOAD = 11.2358e9 * 16
METRIC = "exact pairs/sec & ns/pair on 1 B200: learned-batched vs plain GPU vs CPU"


# --------------------------------------------------------------- workload
def bernoulli_rows_gpu(n, m, p, seed, device, chunk=1024):
    """[n, ceil(m/64)] int64 rows (bit patterns of u64 words) generated on the
    GPU: row r's bits are iid Bernoulli(p_r), p_r = p or U[p[0], p[1]]."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    w = (m + 63) // 64
    out = torch.empty((n, w), dtype=torch.int64, device=device)
    shifts = torch.arange(64, device=device, dtype=torch.int64)
    for r0 in range(0, n, chunk):
        r1 = min(n, r0 + chunk)
        if isinstance(p, tuple):
            pr = p[0] + (p[1] - p[0]) * torch.rand((r1 - r0, 1), generator=g, device=device)
        else:
            pr = torch.full((r1 - r0, 1), float(p), device=device)
        bits = torch.rand((r1 - r0, w * 64), generator=g, device=device) < pr
        if w * 64 > m:
            bits[:, m:] = False
        out[r0:r1] = (bits.view(r1 - r0, w, 64).to(torch.int64) << shifts).sum(dim=-1)
        del bits
    return out


def pairs_of(n):
    return n * (n + 1) // 2


def haplotype_rows_gpu(n_sites, n_hap, block, seed, device, chunk=4096):
    """Haplotype-like matrix: per site an allele count k with P(k) ~ 1/k on
    [1, n_hap - 1]; carriers are whole contiguous blocks of `block`
    haplotypes, ceil(k / block) distinct blocks at random, the last selected
    block (in haplotype order) filled only up to k carriers.  Returns
    [n_sites, ceil(n_hap/64)] int64 on the device."""
    import torch
    g = np.random.Generator(np.random.PCG64(seed))
    ks = np.arange(1, n_hap, dtype=np.float64)
    pk = 1.0 / ks
    pk /= pk.sum()
    kk = g.choice(ks.astype(np.int64), size=n_sites, p=pk)
    n_blocks = (n_hap + block - 1) // block
    w = (n_hap + 63) // 64
    tg = torch.Generator(device=device)
    tg.manual_seed(seed)
    out = torch.empty((n_sites, w), dtype=torch.int64, device=device)
    shifts = torch.arange(64, device=device, dtype=torch.int64)
    hap = torch.arange(w * 64, device=device)
    blk_of = (hap // block).clamp(max=n_blocks - 1)
    off_in = hap % block
    for r0 in range(0, n_sites, chunk):
        r1 = min(n_sites, r0 + chunk)
        k = torch.from_numpy(kk[r0:r1]).to(device)
        nb = torch.clamp((k + block - 1) // block, max=n_blocks)
        keys = torch.rand((r1 - r0, n_blocks), generator=tg, device=device)
        rank = keys.argsort(dim=1).argsort(dim=1)               # random rank of each block
        sel = rank < nb[:, None]
        ordinal = torch.cumsum(sel.to(torch.int32), dim=1)      # 1-based order among selected blocks
        last_fill = (k - block * (nb - 1))[:, None]              # carriers in the last selected block
        bits = sel[:, blk_of] & ((ordinal[:, blk_of] < nb[:, None]) | (off_in[None, :] < last_fill))
        bits &= hap[None, :] < n_hap
        out[r0:r1] = (bits.view(r1 - r0, w, 64).to(torch.int64) << shifts).sum(dim=-1)
    return out


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (200 ms period)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, name in enumerate(names):
                if len(s) > 5 + k and s[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


_TENSOR8 = {}


def tensor8_peak(device, size=8192, reps=10, loop_s=2.0):
    """Dense 8-bit tensor-core throughput measured on this GPU, the
    denominator of the tensor-core kernels' roofline: cuBLASLt GEMMs of
    size^3 with s8 x s8 -> s32 (torch._int_mm) and e4m3 x e4m3 -> bf16
    (torch._scaled_mm), each as the best of `reps` single calls (burst) and as
    a back-to-back loop of about loop_s seconds (sustained); TOPS = 2 size^3 /
    time.  Library calls outside every timed region of this benchmark.  The
    roofline divides by the largest of the burst figures and twice the
    measured bf16 rate, so a slow library path cannot inflate the fraction."""
    if "res" in _TENSOR8:
        return _TENSOR8["res"]
    import torch
    res = {"gemm": f"{size}^3"}

    def time_fn(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        best = None
        for _ in range(reps):
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            t = e0.elapsed_time(e1)
            best = t if best is None else min(best, t)
        n_loop = max(10, int(loop_s * 1e3 / max(best, 1e-3)))
        e0.record()
        for _ in range(n_loop):
            fn()
        e1.record()
        e1.synchronize()
        ops = 2.0 * size ** 3
        return ops / (best * 1e-3) / 1e12, ops * n_loop / (e0.elapsed_time(e1) * 1e-3) / 1e12

    g = torch.Generator(device=device)
    g.manual_seed(8)
    try:
        a = torch.randint(-128, 127, (size, size), dtype=torch.int8, device=device, generator=g)
        bt = torch.randint(-128, 127, (size, size), dtype=torch.int8, device=device, generator=g)
        best = None
        for b in (bt.t(), bt):   # column-major B first (the IMMA layout), then row-major
            try:
                r = time_fn(lambda: torch._int_mm(a, b))
            except Exception:
                continue
            if best is None or r[0] > best[0]:
                best = r
        if best:
            res["int8_tops"], res["int8_tops_sustained"] = round(best[0], 1), round(best[1], 1)
        del a, bt
    except Exception as e:
        res["int8_error"] = f"{type(e).__name__}: {e}"
    try:
        a = torch.randn((size, size), device=device, generator=g).to(torch.float8_e4m3fn)
        bt = torch.randn((size, size), device=device, generator=g).to(torch.float8_e4m3fn)
        one = torch.tensor(1.0, device=device)
        r = time_fn(lambda: torch._scaled_mm(a, bt.t(), scale_a=one, scale_b=one, out_dtype=torch.bfloat16))
        res["fp8_tflops"], res["fp8_tflops_sustained"] = round(r[0], 1), round(r[1], 1)
        del a, bt
    except Exception as e:
        res["fp8_error"] = f"{type(e).__name__}: {e}"
    torch.cuda.empty_cache()
    _TENSOR8["res"] = res
    return res


def tensor_peak_tops(device):
    """(peak TOPS, source text) for the int8 tensor-core roofline."""
    peaks, src = measured_peaks()
    t8 = tensor8_peak(device)
    cands = {f"2 x bf16_tflops {src}": 2.0 * peaks["bf16_tflops"]}
    if t8.get("int8_tops"):
        cands["cuBLASLt int8 GEMM measured (burst)"] = t8["int8_tops"]
    if t8.get("fp8_tflops"):
        cands["cuBLASLt fp8 GEMM measured (burst)"] = t8["fp8_tflops"]
    name = max(cands, key=cands.get)
    return cands[name], f"{name}: {cands[name]:.1f} (largest of {json.dumps({k: round(v, 1) for k, v in cands.items()})})"


# ------------------------------------------------------ distributed setup
def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def init_dist(world, backend, timeout_s=180.0):
    """Process group for N > 1 (None at N = 1). The timeout bounds every
    collective: a rank that never arrives (it failed between steps) ends the
    others' next collective with an error instead of a hang."""
    import torch.distributed as dist
    if world > 1 and not dist.is_initialized():
        import datetime
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist if world > 1 else None


def max_over_ranks(value, dist, device):
    """Max of a float over ranks (all ranks call it in the same order)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, dist, device):
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ------------------------------------------------------------ CPU baseline
def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def reference_sample(host_rows: np.ndarray, target_s: float, threads: int):
    """Time the reference's AND+popcount kernel (oracle/_ref) over whole rows
    of the triangle, starting at row 0, sized to ~target_s seconds.
    Returns (pairs/s, pairs, seconds, rows)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    R = ol.reference()
    if R is None:
        return None
    n, w = host_rows.shape
    rows = np.ascontiguousarray(host_rows)
    ptr = rows.ctypes.data_as(ol.u64p)
    # calibrate on a few rows
    r1 = max(1, min(n, 2 * threads))
    t0 = time.perf_counter()
    R.ref_contig_matrix_mt(ptr, n, w, 0, r1, None, threads)
    dt = time.perf_counter() - t0
    pairs_cal = sum(n - i for i in range(r1))
    rate = pairs_cal / max(dt, 1e-9)
    want_pairs = rate * target_s
    rows_needed = max(1, min(n, int(want_pairs / n) + 1))
    t0 = time.perf_counter()
    R.ref_contig_matrix_mt(ptr, n, w, 0, rows_needed, None, threads)
    dt = time.perf_counter() - t0
    pairs = sum(n - i for i in range(rows_needed))
    return pairs / dt, pairs, dt, rows_needed


# ------------------------------------------------- mixed-density forms
def zipf_sets_gpu(n, universe, s, lo, hi, seed, device):
    """Rows with cardinality P(k) ~ k^-s on [lo, hi], elements uniform without
    replacement, sorted u32 (generated on the GPU in batches, returned as
    numpy arrays)."""
    cards = zipf_cards(n, s, lo, hi, seed)
    out = []
    for b, (r0, r1) in enumerate(batch_plan(cards, 1 << 27)):
        vals, offs = uniform_rows_batch(cards[r0:r1], universe, seed * 1000003 + b, device)
        host = vals.cpu().numpy().view(np.uint32)
        out.extend(host[int(offs[k]):int(offs[k + 1])].copy() for k in range(r1 - r0))
    return out


def mixed_density_forms(sb, device, n=4096, universe=1 << 20, tile=64, samples=1024):
    """Config-3-shaped corpus (Zipf(1.1) cardinalities, clipped like the full
    configuration relative to the universe: [16, universe/4]) through the kernel
    layer: plain per-tile GPU launches with the reference's cost model, the
    batched persistent graph launch with the cost model, the batched launch
    with the learned selector, and the reference's own CPU driver on a row
    sample.  Counts of every GPU form are checked against each other."""
    t_gen = time.perf_counter()
    sets = zipf_sets_gpu(n, universe, 1.1, 16, universe // 4, 0xC0F3, device)
    t_gen = time.perf_counter() - t_gen
    r = sb.StormRows(universe)
    for v in sets:
        r.add(v)
    t_up = time.perf_counter()
    r.upload()   # positions to HBM, every representation built on the device
    t_up = time.perf_counter() - t_up
    pairs = n * (n - 1) // 2
    out = {"workload": f"{n} rows over 2^{universe.bit_length() - 1}, card ~ Zipf(1.1) on [16, 2^"
                       f"{(universe // 4).bit_length() - 1}], uniform w/o replacement; tile {tile}",
           "pairs": pairs, "generate_s": round(t_gen, 2), "upload_and_device_build_s": round(t_up, 4),
           "values": int(sum(len(v) for v in sets))}
    def best_of(policy, exec_, reps=3, tile=tile):
        times, s = [], None
        for _ in range(reps):
            s, st = r.allpairs_sum(policy, tile, exec_=exec_)
            times.append(st["ns_total"])
        return s, min(times), st

    forms = {}
    # the reference's default constants (Apple M4, storm_cost.cpp:482-496) before any calibration
    r.set_dense_block(0.0)
    s0, ns0, st0 = best_of(sb.POLICY_PERTILE, sb.EXEC_PER_TILE)
    forms["plain_per_tile_default_model"] = {"pairs_per_s": pairs / (ns0 * 1e-9), "ms": ns0 * 1e-6,
                                             "launches": st0["launches"], "cell_pairs": st0["cell_pairs"]}
    t0 = time.perf_counter()
    sel = r.train_selector(tile=tile, samples=samples, epochs=400, seed=7)   # also calibrates the cost model
    out["train_s"] = round(time.perf_counter() - t0, 2)
    out["selector"] = {k: (round(v, 4) if isinstance(v, float) else v) for k, v in sel.items()}
    out["selector"].update({k: round(v, 4) for k, v in r.last_training().items()})
    ref_sum = s0
    for name, pol, ex, dense in (("plain_per_tile_cost_model", sb.POLICY_PERTILE, sb.EXEC_PER_TILE, 0.0),
                                 ("batched_cost_model", sb.POLICY_PERTILE, sb.EXEC_BATCHED, 0.0),
                                 ("batched_learned", sb.POLICY_LEARNED, sb.EXEC_BATCHED, 0.0),
                                 ("batched_learned_tensor_block", sb.POLICY_LEARNED, sb.EXEC_BATCHED,
                                  DENSE_BLOCK_DEFAULT),
                                 ("batched_all_bitmap", sb.POLICY_ALLBITMAP, sb.EXEC_BATCHED, 0.0)):
        r.set_dense_block(dense)
        s, ns, st = best_of(pol, ex)
        if ref_sum is None:
            ref_sum = s
        if s != ref_sum:
            raise RuntimeError(f"{name}: sum {s} != {ref_sum}")
        forms[name] = {"pairs_per_s": pairs / (ns * 1e-9), "ms": ns * 1e-6, "launches": st["launches"],
                       "cell_pairs": st["cell_pairs"]}
    # Autotuned: tile x dense-block threshold timed on this corpus (the
    # learned selector keeps its training tile), best kept for tile-0 calls.
    for name, pol in (("batched_cost_model_autotuned", sb.POLICY_PERTILE),
                      ("batched_learned_autotuned", sb.POLICY_LEARNED)):
        t_tile, t_dens, _ = r.autotune(pol, sb.EXEC_BATCHED)
        s, ns, st = best_of(pol, sb.EXEC_BATCHED, tile=0)
        if s != ref_sum:
            raise RuntimeError(f"{name}: sum {s} != {ref_sum}")
        forms[name] = {"pairs_per_s": pairs / (ns * 1e-9), "ms": ns * 1e-6, "launches": st["launches"],
                       "tile": t_tile, "dense_block_min_density": t_dens, "cell_pairs": st["cell_pairs"]}
    out["forms"] = forms
    out["plain_per_tile_cost_model_is"] = "the cost model calibrated on this GPU's cell timings (training split)"
    out["learned_autotuned_over_plain"] = (forms["batched_learned_autotuned"]["pairs_per_s"] /
                                           forms["plain_per_tile_cost_model"]["pairs_per_s"])
    out["calibrated_over_default_per_tile"] = (forms["plain_per_tile_cost_model"]["pairs_per_s"] /
                                               forms["plain_per_tile_default_model"]["pairs_per_s"])
    out["learned_over_plain"] = forms["batched_learned"]["pairs_per_s"] / forms["plain_per_tile_cost_model"]["pairs_per_s"]
    out["learned_tensor_block_over_plain"] = (forms["batched_learned_tensor_block"]["pairs_per_s"] /
                                              forms["plain_per_tile_cost_model"]["pairs_per_s"])
    out["learned_over_batched_cost_model"] = (forms["batched_learned"]["pairs_per_s"] /
                                              forms["batched_cost_model"]["pairs_per_s"])
    # The reference's own kernel-layer driver (storm::allpairs_sum, PerTile, default model) on a sample.
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    R = ol.reference()
    if R is not None:
        g = np.random.Generator(np.random.PCG64(11))
        pick = np.sort(g.choice(n, size=min(n, 384), replace=False))
        sub = [sets[i] for i in pick]
        offs = np.zeros(len(sub) + 1, np.uint64)
        for k, v in enumerate(sub):
            offs[k + 1] = offs[k] + len(v)
        vals = np.ascontiguousarray(np.concatenate(sub), dtype=np.uint32)
        st = np.zeros(4, np.uint64)
        t0 = time.perf_counter()
        R.ref_allpairs_sum(vals.ctypes.data_as(ol.u32p), offs.ctypes.data_as(ol.u64p), len(sub), universe, 2, tile,
                           st.ctypes.data_as(ol.u64p))
        dt = time.perf_counter() - t0   # includes build_row of the sample (the reference times it too)
        sp = len(sub) * (len(sub) - 1) // 2
        out["cpu_reference_per_tile"] = {"pairs_per_s": sp / dt, "cores": 1,
                                         "sample": f"{len(sub)} random rows ({sp} pairs), storm::allpairs_sum "
                                                   f"PerTile incl. build_row, single thread as shipped"}
    r.close()
    return out


def run_sets_gpu(n, universe, mean_runs, mean_len, seed, device):
    """Run-clustered rows: Poisson(mean_runs) runs per row, start uniform,
    length Geometric(mean mean_len); the row is the union (sorted u32)."""
    import torch
    g = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(n):
        k = int(g.poisson(mean_runs))
        if k == 0:
            out.append(np.zeros(0, np.uint32))
            continue
        starts = torch.from_numpy(g.integers(0, universe, size=k)).to(device)
        lens = torch.from_numpy(g.geometric(1.0 / mean_len, size=k)).to(device)
        pos = torch.repeat_interleave(starts, lens) + (torch.arange(int(lens.sum().item()), device=device) -
                                                       torch.repeat_interleave(torch.cumsum(lens, 0) - lens, lens))
        pos = torch.unique(pos[pos < universe])
        out.append(pos.to(torch.int64).cpu().numpy().astype(np.uint32))
    return out


def bernoulli_sets_gpu(n, universe, density, seed, device):
    import torch
    g = np.random.Generator(np.random.PCG64(seed))
    tg = torch.Generator(device=device)
    tg.manual_seed(seed)
    out = []
    for k in g.binomial(universe, density, size=n):
        perm = torch.randperm(universe, generator=tg, device=device)[: int(k)]
        out.append(torch.sort(perm).values.to(torch.int64).cpu().numpy().astype(np.uint32))
    return out


# ------------------------------------------- full-size STORM_t corpora
def zipf_cards(n, s, lo, hi, seed):
    """Row cardinalities with P(k) ~ k^-s on [lo, hi] (the same draw as
    zipf_sets_gpu for the same seed)."""
    g = np.random.Generator(np.random.PCG64(seed))
    ks = np.arange(lo, hi + 1, dtype=np.float64)
    pk = ks ** (-s)
    pk /= pk.sum()
    return g.choice(ks.astype(np.int64), size=n, p=pk)


def batch_plan(sizes, max_values):
    """Consecutive row ranges [r0, r1) holding at most max_values values
    (a single larger row gets a range of its own)."""
    out, r0, acc = [], 0, 0
    for r, k in enumerate(sizes):
        if r > r0 and acc + int(k) > max_values:
            out.append((r0, r))
            r0, acc = r, 0
        acc += int(k)
    if r0 < len(sizes):
        out.append((r0, len(sizes)))
    return out


def uniform_rows_batch(cards, universe, seed, device):
    """Rows r of one batch: cards[r] distinct positions uniform without
    replacement over [0, universe), sorted.  Positions are drawn with
    repeats (enough draws that the expected distinct count exceeds the
    cardinality by several standard deviations; rows left short draw again),
    repeats are removed, and a uniformly random subset of the wanted size is
    kept (random priorities, the lowest per row).  Returns (values int32 on
    the device, offsets numpy u64 from 0)."""
    import torch
    U = int(universe)
    nb = len(cards)
    k = torch.as_tensor(np.asarray(cards, np.int64), device=device)
    if nb == 0:
        return torch.zeros(0, dtype=torch.int32, device=device), np.zeros(1, np.uint64)
    if float(k.max().item()) > 0.5 * U:
        raise ValueError("uniform_rows_batch: density above 1/2")
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    kd = k.to(torch.float64)
    dens = kd / U
    m = torch.where(k > 0, torch.ceil(-U * torch.log1p(-dens) + 6.0 * torch.sqrt(kd) + 32.0),
                    torch.zeros_like(kd)).to(torch.int64)
    rid = torch.arange(nb, device=device, dtype=torch.int64)
    key = torch.unique(torch.repeat_interleave(rid, m) * U +
                       torch.randint(0, U, (int(m.sum().item()),), generator=g, device=device))
    for _ in range(64):
        cnt = torch.bincount(key // U, minlength=nb)
        short = cnt < k
        if not bool(short.any()):
            break
        extra = torch.where(short, 2 * (k - cnt) + 64, torch.zeros_like(k))
        more = torch.repeat_interleave(rid, extra) * U + torch.randint(0, U, (int(extra.sum().item()),),
                                                                       generator=g, device=device)
        key = torch.unique(torch.cat([key, more]))
    else:
        raise RuntimeError("uniform_rows_batch: rows stayed short")
    krow = key // U
    pr = torch.rand(key.numel(), generator=g, device=device, dtype=torch.float64)
    order = torch.argsort(krow.to(torch.float64) * 2.0 + pr)
    start = torch.cumsum(cnt, 0) - cnt
    rank = torch.arange(key.numel(), device=device) - start[krow[order]]
    keep = order[rank < k[krow[order]]]
    key = torch.sort(key[keep]).values
    vals = (key % U).to(torch.int32)
    offs = np.zeros(nb + 1, np.uint64)
    offs[1:] = np.cumsum(np.asarray(cards, np.uint64))
    return vals, offs


def run_rows_batch(starts, lens, nrun, universe, device):
    """Rows of one batch as unions of runs [start, start + len) clipped to
    the universe: nrun[r] runs for row r, starts/lens their concatenation.
    Returns (values int32 on the device, offsets numpy u64 from 0)."""
    import torch
    U = int(universe)
    nb = len(nrun)
    st = torch.as_tensor(np.asarray(starts, np.int64), device=device)
    ln = torch.as_tensor(np.asarray(lens, np.int64), device=device)
    rr = torch.repeat_interleave(torch.arange(nb, device=device), torch.as_tensor(np.asarray(nrun, np.int64),
                                                                                     device=device))
    tot = int(ln.sum().item())
    run_of = torch.repeat_interleave(torch.arange(st.numel(), device=device), ln)
    first = torch.cumsum(ln, 0) - ln
    pos = st[run_of] + (torch.arange(tot, device=device) - first[run_of])
    ok = pos < U
    key = torch.unique(rr[run_of][ok] * U + pos[ok])
    cnt = torch.bincount(key // U, minlength=nb).cpu().numpy()
    offs = np.zeros(nb + 1, np.uint64)
    offs[1:] = np.cumsum(cnt.astype(np.uint64))
    return (key % U).to(torch.int32), offs


class FullCorpus:
    """One of the full-size STORM_t configurations, generated on the GPU
    batch by batch, each batch from its own seed, so that any batch can be
    made again on its own.  kind:
      "zipf"      N rows over `universe`, card ~ Zipf(s) on [lo, hi] (P(k) ~
                  k^-s restricted to the range), uniform without replacement;
      "runs"      N rows over `universe`, Poisson(mean_runs) runs per row,
                  start uniform, length Geometric(mean mean_len);
      "bernoulli" N rows over `universe`, every bit iid Bernoulli(density):
                  card ~ Binomial, positions uniform without replacement;
      "bits"      the same distribution made as packed bitmaps (every bit
                  drawn), for densities whose value lists would be larger.
    batch(b) -> (r0, r1, values int32 on the device, offsets numpy u64), or
    for "bits" (r0, r1, words int64 [rows, universe / 64] on the device,
    None)."""

    def __init__(self, kind, n, universe, seed, device, max_values=1 << 28, **kw):
        self.kind, self.n, self.universe, self.seed, self.device = kind, n, int(universe), seed, device
        g = np.random.Generator(np.random.PCG64(seed))
        self.density = kw.get("density")
        if kind == "zipf":
            self.cards = zipf_cards(n, kw.get("s", 1.1), kw["lo"], kw["hi"], seed)
            sizes = self.cards
        elif kind == "bernoulli":
            self.cards = g.binomial(self.universe, self.density, size=n).astype(np.int64)
            sizes = self.cards
        elif kind == "bits":
            self.cards = None
            sizes = np.full(n, self.universe // 32, np.int64)      # u64 words, in 32-bit units
        elif kind == "runs":
            self.nrun = g.poisson(kw["mean_runs"], size=n).astype(np.int64)
            tot = int(self.nrun.sum())
            self.starts = g.integers(0, self.universe, size=tot)
            self.lens = g.geometric(1.0 / kw["mean_len"], size=tot).astype(np.int64)
            self.run0 = np.zeros(n + 1, np.int64)
            self.run0[1:] = np.cumsum(self.nrun)
            sizes = np.zeros(n, np.int64)
            nz = self.nrun > 0
            sizes[nz] = np.add.reduceat(self.lens, self.run0[:-1][nz]) if tot else 0
            self.cards = None
        else:
            raise ValueError(kind)
        self.plan = batch_plan(sizes, max_values)

    def batch(self, b):
        import torch
        r0, r1 = self.plan[b]
        if self.kind == "runs":
            a, z = int(self.run0[r0]), int(self.run0[r1])
            vals, offs = run_rows_batch(self.starts[a:z], self.lens[a:z], self.nrun[r0:r1], self.universe,
                                        self.device)
            return r0, r1, vals, offs
        if self.kind == "bits":
            g = torch.Generator(device=self.device)
            g.manual_seed(self.seed * 1000003 + b)
            w = self.universe // 64
            out = torch.empty((r1 - r0, w), dtype=torch.int64, device=self.device)
            shifts = torch.arange(64, device=self.device, dtype=torch.int64)
            for q0 in range(0, r1 - r0, 16):
                q1 = min(r1 - r0, q0 + 16)
                bits = torch.rand((q1 - q0, self.universe), generator=g, device=self.device) < self.density
                out[q0:q1] = (bits.view(q1 - q0, w, 64).to(torch.int64) << shifts).sum(dim=-1)
                del bits
            return r0, r1, out, None
        vals, offs = uniform_rows_batch(self.cards[r0:r1], self.universe, self.seed * 1000003 + b, self.device)
        return r0, r1, vals, offs

    def batch_of(self, row):
        """Index of the batch holding `row`."""
        for b, (r0, r1) in enumerate(self.plan):
            if r0 <= row < r1:
                return b
        raise IndexError(row)


def full_corpus(name, device):
    """The full-size configurations run through STORM_t."""
    if name == "config3":
        return FullCorpus("zipf", 100000, 1 << 24, 0xC0F3, device, s=1.1, lo=16, hi=1 << 22)
    if name == "config4":
        return FullCorpus("runs", 50000, 1 << 26, 0xC0F4, device, mean_runs=200, mean_len=256)
    if name == "config5b_0.01":
        return FullCorpus("bernoulli", 20000, 1 << 24, 0xC05B, device, density=0.01)
    if name == "config5b_0.17":
        return FullCorpus("bits", 20000, 1 << 24, 0xC05C, device, density=0.17, max_values=1 << 27)
    raise ValueError(name)


FULL_CORPORA = {
    "config3": "100000 rows over 2^24, card ~ Zipf(1.1) on [16, 2^22], uniform w/o replacement (5.0e9 pairs)",
    "config4": "50000 rows over 2^26, Poisson(200) runs of Geometric(mean 256) length (1.25e9 pairs)",
    "config5b_0.01": "20000 rows over 2^24, Bernoulli(0.01) (2.0e8 pairs)",
    "config5b_0.17": "20000 rows over 2^24, Bernoulli(0.17) (2.0e8 pairs)",
}


def _batch_hist_and_cards(corpus, vals_or_words, offs):
    """(value histogram of the batch over the universe, per-row counts)."""
    import torch
    if offs is not None:
        return torch.bincount(vals_or_words, minlength=corpus.universe), np.diff(offs.astype(np.int64))
    w = vals_or_words
    shifts = torch.arange(64, device=w.device, dtype=torch.int64)
    h = torch.zeros(corpus.universe, dtype=torch.int64, device=w.device)
    cards = torch.zeros(w.shape[0], dtype=torch.int64, device=w.device)
    for q0 in range(0, w.shape[0], 16):
        bits = ((w[q0:q0 + 16, :, None] >> shifts) & 1).view(-1, corpus.universe)
        h += bits.sum(dim=0)
        cards[q0:q0 + 16] = bits.sum(dim=1)
        del bits
    return h, cards.cpu().numpy()


def _batch_row_sums(corpus, vals_or_words, offs, hist):
    """Per row of the batch: sum over its values v of hist[v]."""
    import torch
    if offs is not None:
        nb = len(offs) - 1
        seg = torch.repeat_interleave(torch.arange(nb, device=hist.device),
                                      torch.as_tensor(np.diff(offs.astype(np.int64)), device=hist.device))
        out = torch.zeros(nb, dtype=torch.int64, device=hist.device)
        out.index_add_(0, seg, hist[vals_or_words.to(torch.int64)])
        return out
    w = vals_or_words
    shifts = torch.arange(64, device=w.device, dtype=torch.int64)
    hf = hist.to(torch.float64)
    out = torch.zeros(w.shape[0], dtype=torch.int64, device=w.device)
    for q0 in range(0, w.shape[0], 8):
        bits = ((w[q0:q0 + 8, :, None] >> shifts) & 1).view(-1, corpus.universe).to(torch.float64)
        out[q0:q0 + 8] = torch.round(bits @ hf).to(torch.int64)   # exact: every partial sum < 2^53
        del bits
    return out


def load_full_corpus(sb, corpus, on_batch=None, row_sums=True, keep_limit=100 << 30):
    """Generates every batch in row order and appends it to a new STORM_t
    (STORM_add_rows for value lists, STORM_add_bitmap_rows for bitmaps, from
    host memory), accumulating the value histogram on the device; calls
    on_batch(r0, r1, host values or words, offsets or None) per batch.  With
    row_sums, also returns every row's sum over its values v of (rows
    holding v) -- from batches kept on the device when they fit keep_limit,
    else from a second pass that makes each batch again.  Returns a dict:
    storm, hist, cards, want_row (or None), gen_s, add_s."""
    import torch
    st = sb.Storm()
    hist = torch.zeros(corpus.universe, dtype=torch.int64, device=corpus.device)
    cards = np.zeros(corpus.n, np.int64)
    t_gen = t_add = 0.0
    kept, kept_bytes, keep = [], 0, row_sums
    for b in range(len(corpus.plan)):
        t0 = time.perf_counter()
        r0, r1, x, offs = corpus.batch(b)
        h, c = _batch_hist_and_cards(corpus, x, offs)
        hist += h
        cards[r0:r1] = c
        host = x.cpu().numpy()
        t1 = time.perf_counter()
        if offs is not None:
            st.add_rows(host.view(np.uint32), offs)
        else:
            st.add_bitmap_rows(host.view(np.uint64))
        t2 = time.perf_counter()
        t_gen += t1 - t0
        t_add += t2 - t1
        if on_batch is not None:
            on_batch(r0, r1, host.view(np.uint32) if offs is not None else host.view(np.uint64), offs)
        if keep:
            kept_bytes += x.numel() * x.element_size()
            if kept_bytes <= keep_limit:
                kept.append((r0, r1, x, offs))
            else:
                keep, kept = False, []
        del x, host
    want_row = None
    if row_sums:
        want_row = torch.zeros(corpus.n, dtype=torch.int64, device=corpus.device)
        if keep:
            for r0, r1, x, offs in kept:
                want_row[r0:r1] = _batch_row_sums(corpus, x, offs, hist)
            kept = []
        else:
            for b in range(len(corpus.plan)):
                r0, r1, x, offs = corpus.batch(b)
                want_row[r0:r1] = _batch_row_sums(corpus, x, offs, hist)
                del x
    torch.cuda.empty_cache()
    return {"storm": st, "hist": hist, "cards": cards, "want_row": want_row, "gen_s": t_gen, "add_s": t_add}


def triangle_row_sums(d_tri, n):
    """Per row i of the full symmetric matrix held as a packed device
    triangle (i <= j): the upper part of row i plus column i above the
    diagonal; and the diagonal.  Returns (row sums int64, diagonal int64),
    both on the device."""
    import torch
    dev = d_tri.device
    ii = np.arange(n + 1, dtype=np.int64)
    S = ii * n - (ii * (ii - 1)) // 2                  # start of row i; S[n] = n(n+1)/2
    got = torch.zeros(n, dtype=torch.int64, device=dev)
    diag = torch.zeros(n, dtype=torch.int64, device=dev)
    i = 0
    while i < n:
        i1 = int(np.searchsorted(S, S[i] + (1 << 27), side="right")) - 1   # rows whose entries fit the step
        i1 = min(n, max(i + 1, i1))
        a, b = int(S[i]), int(S[i1])
        seg = d_tri[a:b].to(torch.int64) & 0xFFFFFFFF
        lens = torch.as_tensor(n - ii[i:i1], device=dev)
        rows = torch.repeat_interleave(torch.arange(i, i1, device=dev), lens)
        first = torch.as_tensor(S[i:i1] - a, device=dev)
        cols = rows + (torch.arange(b - a, device=dev) - torch.repeat_interleave(first, lens))
        got.index_add_(0, rows, seg)
        off = cols != rows
        got.index_add_(0, cols[off], seg[off])
        diag[i:i1] = seg[first]
        del seg, rows, cols, off
        i = i1
    return got, diag


def engine_roofline(eng, device):
    """Per STORM_t engine of the last call: device ms, the planner's
    prediction, and the engine's roofline -- the tensor cores against the
    measured 8-bit tensor peak, the panel and the postings (bytes they must
    move) against the measured HBM bandwidth."""
    peaks, src = measured_peaks()
    tpk, _ = tensor_peak_tops(device)
    out = {}
    for name, (ms, pred, work) in eng.items():
        if ms <= 0 and work <= 0:
            continue
        e = {"ms": round(ms, 3), "predicted_ms": round(pred, 3)}
        if ms > 0 and work > 0:
            if name == "tensor":
                e.update({"tops_int8": work / (ms * 1e-3) / 1e12, "frac_of_tensor_peak": work / (ms * 1e-3) / 1e12 / tpk})
            elif name in ("panel", "postings"):
                gbs = work / (ms * 1e-3) / 1e9
                e.update({"alg_bytes": work, "GBps": gbs, "frac_of_hbm": gbs / peaks["hbm_gbs"],
                          "hbm_peak_source": src})
            else:
                e.update({"pairs": work})
        out[name] = e
    return out


def storm_t_full(device, names=tuple(FULL_CORPORA), cpu_seconds=2.0):
    """The sparse and mixed-density configurations at full size through
    STORM_t: rows generated on the GPU and appended from host memory
    (STORM_add_rows / STORM_add_bitmap_rows), then
      e2e       the first per-pair call into a host buffer (packs the rows,
                uploads them, computes, copies the triangle back);
      device    per-pair counts into HBM, device time of the call (best of 2);
      sum_only  the reference's STORM_pairw_intersect_cardinality;
    every triangle checked against the value-histogram identities (every
    row's sum, the diagonal, the total) before it is reported; and the
    reference's own STORM_pairw_intersect_cardinality on 1 core plus a
    harness over all host threads, on a prefix of the rows."""
    import torch
    import importlib
    sb = importlib.import_module("stormbitmaps-internal_b200")
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    R = ol.reference()
    out = {}
    for name in names:
        torch.cuda.empty_cache()
        t0 = time.perf_counter()
        corpus = full_corpus(name, device)
        prefix = {}

        def keep_prefix(r0, r1, host, offs):
            if r0 == 0:
                prefix["host"], prefix["offs"] = host.copy(), None if offs is None else offs.copy()

        res = load_full_corpus(sb, corpus, on_batch=keep_prefix)
        st, hist, cards = res["storm"], res["hist"], res["cards"]
        n = corpus.n
        tri = n * (n + 1) // 2
        r = {"workload": FULL_CORPORA[name], "rows": n, "pairs_i_le_j": tri, "values": int(cards.sum()),
             "generate_s": round(res["gen_s"], 1), "STORM_add_rows_s": round(res["add_s"], 1)}
        want_sum = int((hist * (hist - 1) // 2).sum().item())
        # end to end: the first per-pair call into host memory
        host_out = torch.empty(tri, dtype=torch.int32, pin_memory=True)
        t1 = time.perf_counter()
        _, s_e2e = st.matrix(host_out.numpy().view(np.uint32))
        r["e2e"] = {"first_matrix_call_s": round(time.perf_counter() - t1, 3),
                    "pairs_per_s": tri / (time.perf_counter() - t1), "d2h_bytes": tri * 4,
                    "call": "STORM_pairw_intersect_matrix (pack + upload + all pairs + copy back)",
                    "transfers": st.last_transfer_ms()}
        del host_out
        d_tri = torch.empty(tri, dtype=torch.int32, device=device)
        best, sums = None, {s_e2e}
        for _ in range(2):
            sums.add(st.matrix_device(d_tri.data_ptr(), tri))
            ms = st.last_kernel_ms()
            best = ms if best is None else min(best, ms)
        r["device"] = {"ms": round(best, 2), "pairs_per_s": tri / (best * 1e-3), "ns_per_pair": best * 1e6 / tri,
                       "tensor_rows": st.last_dense()[0], "postings_rows": st.last_postings_rows(),
                       "panel_rows": st.last_panel_rows()}
        r["engines"] = engine_roofline(st.last_engine_ms(), device)
        r["engines"]["plan_ms"] = round(st.last_plan_ms(), 3)
        got_row, diag = triangle_row_sums(d_tri, n)
        ok = (bool(torch.equal(diag.cpu(), torch.as_tensor(cards))) and
              int((got_row != res["want_row"]).sum().item()) == 0 and sums == {want_sum})
        r["checked"] = {"identities_hold": ok, "sum_i_lt_j": want_sum}
        del d_tri, got_row, diag
        torch.cuda.empty_cache()
        best = None
        for _ in range(2):
            v = st.pairw_intersect_cardinality()
            ms = st.last_kernel_ms()
            best = ms if best is None else min(best, ms)
            r["checked"]["identities_hold"] &= v == want_sum
        r["sum_only_ms"] = round(best, 2)
        st.close()
        if R is not None and prefix.get("offs") is not None:
            vals_p, offs_p = prefix["host"], prefix["offs"]
            for label, mt in (("cpu_reference", False), ("cpu_reference_all_threads", True)):
                k = 64
                while True:
                    k = min(k, len(offs_p) - 1)
                    v = np.ascontiguousarray(vals_p[:int(offs_p[k])], dtype=np.uint32)
                    o = np.ascontiguousarray(offs_p[:k + 1], dtype=np.uint64)
                    sec = C.c_double(0.0)
                    if mt:
                        R.ref_storm_sum_mt(v.ctypes.data_as(ol.u32p), o.ctypes.data_as(ol.u64p), k, cpu_threads(),
                                           C.byref(sec))
                    else:
                        R.ref_storm_sum_timed(v.ctypes.data_as(ol.u32p), o.ctypes.data_as(ol.u64p), k, C.byref(sec))
                    if sec.value >= cpu_seconds or k == len(offs_p) - 1:
                        break
                    k *= 2
                rate = (k * (k - 1) // 2) / max(sec.value, 1e-9)
                r[label] = {"pairs_per_s": rate, "cores": cpu_threads() if mt else 1,
                            "sample": f"first {k} rows ({k * (k - 1) // 2} pairs i < j, {sec.value:.2f} s), " +
                                      ("project harness over the reference's per-pair "
                                       "STORM_bitmap_cont_intersect_cardinality_premade" if mt else
                                       "STORM_pairw_intersect_cardinality as shipped")}
                r["device_over_" + label] = r["device"]["pairs_per_s"] / rate
        r["seconds"] = round(time.perf_counter() - t0, 1)
        out[name] = r
        del res, prefix
    return out


ENGINE_CASES = ("default", "panel", "postings", "tensor", "runs")


def engine_case(engine, device, n=4096, universe=1 << 24, calls=3):
    """One STORM_t engine on its own, for profiling and for its roofline: a
    config-3-shaped corpus (n rows over `universe`, Zipf(1.1) cards on [16,
    universe / 4]) with every plain row given to `engine` (panel: all in the
    transposed panel; postings: the list rows by postings, rows with bitmap
    chunks on the chunk kernel; tensor: all on the tensor cores) or the
    default plan; per call the device time and each engine's measured and
    predicted time and algorithmic work. "runs": a config-4-shaped corpus
    (8192 rows over 2^26, Poisson(200) runs of Geometric(256) length) under
    the default plan, which gives it to the run form of the postings."""
    import torch
    import importlib
    sb = importlib.import_module("stormbitmaps-internal_b200")
    if engine == "runs":
        n, universe = 8192, 1 << 26
        # generated on the host so that a profiler sees only this library's launches
        sets = run_sets_gpu(n, universe, 200, 256, 0xC0F4, torch.device("cpu"))
        shape = f"{n} rows over 2^26, Poisson(200) runs of Geometric(mean 256) length"
    else:
        sets = zipf_sets_gpu(n, universe, 1.1, 16, universe // 4, 0xC0F3, device)
        shape = f"{n} rows over 2^{universe.bit_length() - 1}, Zipf(1.1) on [16, 2^{(universe // 4).bit_length() - 1}]"
    st = sb.Storm()
    vals = np.ascontiguousarray(np.concatenate(sets), dtype=np.uint32)
    offs = np.zeros(n + 1, np.uint64)
    offs[1:] = np.cumsum([len(v) for v in sets])
    st.add_rows(vals, offs)
    if engine == "panel":
        st.set_panel(2)
    elif engine == "postings":
        st.set_dense_block(0.0)
        st.set_sparse_postings(1)
        st.set_panel(0)
    elif engine == "tensor":
        st.set_dense_block(1e-12)
        st.set_sparse_postings(0)
        st.set_panel(0)
    tri = n * (n + 1) // 2
    d_tri = torch.empty(tri, dtype=torch.int32, device=device)
    res = {"engine": engine, "workload": shape, "calls": []}
    sums = set()
    for _ in range(calls):
        sums.add(st.matrix_device(d_tri.data_ptr(), tri))
        res["calls"].append({"ms": round(st.last_kernel_ms(), 3), "plan_ms": round(st.last_plan_ms(), 3),
                             "rows": {"tensor": st.last_dense()[0], "panel": st.last_panel_rows(),
                                      "postings": st.last_postings_rows()},
                             "postings_form": st.last_postings_form(),
                             "engines": engine_roofline(st.last_engine_ms(), device)})
    res["same_sum"] = len(sums) == 1
    st.close()
    return res


# The library's default tensor-core dense-block threshold (rows whose sparse
# form is at least 2^-14 of the universe).
DENSE_BLOCK_DEFAULT = 1.0 / 16384


def forms_on(sb, sets, universe, tile=64, samples=1024, with_plain=True):
    """Learned selector trained on this corpus (held-out regret), then the
    batched learned form against the batched and per-tile cost-model forms."""
    r = sb.StormRows(universe)
    for v in sets:
        r.add(v)
    t_up = time.perf_counter()
    r.upload()   # positions to HBM, every representation built on the device
    t_up = time.perf_counter() - t_up
    n = len(sets)
    pairs = n * (n - 1) // 2
    sel = r.train_selector(tile=tile, samples=samples, epochs=400, seed=7)
    lt = r.last_training()
    res = {"rows": n, "pairs": pairs, "upload_and_device_build_s": round(t_up, 4),
           "regret_learned": round(sel["regret_mlp"], 4),
           "regret_cost_model_calibrated": round(lt["regret_calibrated_model"], 4),
           "fallback_model": "calibrated" if lt["kept_calibrated_model"] else "reference default",
           "regret_cost_model_default": round(lt["regret_default_model"], 4),
           "train_accuracy": round(sel["train_accuracy"], 3)}
    sums = set()
    dflt = DENSE_BLOCK_DEFAULT
    for name, pol, ex, dense in (("batched_learned", sb.POLICY_LEARNED, sb.EXEC_BATCHED, dflt),
                                 ("batched_learned_no_tensor_block", sb.POLICY_LEARNED, sb.EXEC_BATCHED, 0.0),
                                 ("batched_cost_model", sb.POLICY_PERTILE, sb.EXEC_BATCHED, dflt)) + (
            (("plain_per_tile_cost_model", sb.POLICY_PERTILE, sb.EXEC_PER_TILE, 0.0),) if with_plain else ()):
        r.set_dense_block(dense)
        best = None
        for _ in range(2):   # a second call only where the first is short enough for set-up to matter
            s, st = r.allpairs_sum(pol, tile, exec_=ex)
            best = st["ns_total"] if best is None else min(best, st["ns_total"])
            sums.add(s)
            if best > 2e9:
                break
        res[name + "_pairs_per_s"] = pairs / (best * 1e-9)
    if len(sums) != 1:
        raise RuntimeError(f"forms disagree: {sums}")
    r.close()
    return res


def config5a_full(sb, device, steps=3):
    """Config 5a at full size: 200,000 sites x 20,000 haplotypes (1/k allele
    counts in 32-haplotype blocks), 2.0e10 pairs i <= j, the 80 GB triangle
    kept in HBM; rows resident, device time per call; checksum = the sum."""
    import torch
    torch.cuda.empty_cache()
    n, m = 200000, 20000
    rows = haplotype_rows_gpu(n, m, 32, 0xC05A, device)
    torch.cuda.synchronize()
    c = sb.StormContig(m)
    rc = sb.lib().STORM_contig_add_bitmaps(c.h, C.cast(rows.data_ptr(), sb.u64p), n, rows.shape[1])
    if rc < 0:
        raise sb.StormError(rc, "STORM_contig_add_bitmaps")
    del rows
    tri = n * (n + 1) // 2
    out = torch.empty(tri, dtype=torch.int32, device=device)
    c.matrix_device(out.data_ptr(), tri)        # warm-up
    ms, sums = [], set()
    for _ in range(steps):
        sums.add(c.matrix_device(out.data_ptr(), tri))
        ms.append(c.last_kernel_ms())
    k = statistics.median(ms)
    peak, _ = tensor_peak_tops(device)
    tops = 2.0 * tri * m / (k * 1e-3) / 1e12
    res = {"workload": "200000 sites x 20000 haplotypes, P(k) ~ 1/k, 32-haplotype carrier blocks; "
                       "80 GB u32 triangle in HBM", "pairs_i_le_j": tri, "ms": round(k, 2),
           "pairs_per_s": tri / (k * 1e-3), "checksum_sum_i_lt_j": sums.pop() if len(sums) == 1 else None,
           "kernel": {sb.KERNEL_POPC: "bb_popc_kernel", sb.KERNEL_MMA: "bb_mma_ts_kernel",
                      sb.KERNEL_MMA_DB: "bb_mma_ts2_kernel"}.get(c.last_kernel(), "?"),
           "roofline": {"achieved_tops_int8": tops, "peak": peak, "frac": tops / peak}}
    del out
    c.close()
    torch.cuda.empty_cache()
    return res


def autotune_config1(sb, device):
    """The contiguous autotuner on the config 1 geometry (4096 rows x 65536
    bits, Bernoulli(0.5)): per-candidate device times and the kept choice."""
    import torch
    rows = bernoulli_rows_gpu(4096, 65536, 0.5, 0xC001, device)
    torch.cuda.synchronize()
    c = sb.StormContig(65536)
    rc = sb.lib().STORM_contig_add_bitmaps(c.h, C.cast(rows.data_ptr(), sb.u64p), 4096, 1024)
    if rc < 0:
        raise sb.StormError(rc, "STORM_contig_add_bitmaps")
    k, sched, times = c.autotune()
    names = ("tcgen05_ts_tiles", "tcgen05_ts_stream_k", "tcgen05_db_tiles", "tcgen05_db_stream_k", "tcgen05_ss",
             "popc", "tcgen05_cta_pair_tiles")
    c.close()
    cand = [(sb.KERNEL_MMA, sb.SCHED_TILES), (sb.KERNEL_MMA, sb.SCHED_STREAM_K), (sb.KERNEL_MMA_DB, sb.SCHED_TILES),
            (sb.KERNEL_MMA_DB, sb.SCHED_STREAM_K), (sb.KERNEL_MMA_SS, sb.SCHED_AUTO), (sb.KERNEL_POPC, sb.SCHED_AUTO),
            (sb.KERNEL_MMA_2CTA, sb.SCHED_TILES)]
    tops = {nm: round(2.0 * 4096 * 4097 / 2 * 65536 / (t * 1e-3) / 1e12, 1) for nm, t in zip(names, times) if t > 0}
    return {"workload": "4096 rows x 65536 bits, Bernoulli(0.5)",
            "candidates_ms": {nm: round(t, 4) for nm, t in zip(names, times)},
            "candidates_tops_int8": tops,
            "kept": names[cand.index((k, sched))] if (k, sched) in cand else f"kernel {k} schedule {sched}"}


def config45_forms(device, full_sweep=False):
    """Config-4-shaped run-clustered rows and the config-5b density sweep
    (N = 20000 up to density 1e-3, fewer rows above), each with the learned
    selector's held-out regret against the measured-best cell, beside the
    calibrated and the reference default cost model's."""
    import importlib
    sb = importlib.import_module("stormbitmaps-internal_b200")
    out = {}
    t0 = time.perf_counter()
    sets = run_sets_gpu(2048, 1 << 26, 200, 256, 0xC0F4, device)
    out["runs_2^26"] = forms_on(sb, sets, 1 << 26)
    out["runs_2^26"]["workload"] = "2048 rows over 2^26, Poisson(200) runs of Geometric(mean 256) length"
    sweep = {}
    # N = 20000 (config 5b's row count) where the kernel layer's per-pair
    # cells finish within a minute; fewer rows beyond
    # (the default run keeps 1e-5 and 1e-3 at N = 20000 and 1e-2; --all-forms runs every density)
    grid = ((1e-6, 20000), (1e-5, 20000), (1e-4, 20000), (1e-3, 20000), (1e-2, 1024), (0.17, 256))
    for d, n in (grid if full_sweep else ((1e-5, 20000), (1e-3, 20000), (1e-2, 1024))):
        t1 = time.perf_counter()
        sets = (sparse_bernoulli_sets_gpu(n, 1 << 24, d, int(1e7 * d) + 5, device) if d <= 1e-3 else
                bernoulli_sets_gpu(n, 1 << 24, d, int(1e7 * d) + 5, device))
        sweep[f"{d:g}"] = forms_on(sb, sets, 1 << 24, samples=512, with_plain=False)
        sweep[f"{d:g}"]["seconds"] = round(time.perf_counter() - t1, 1)
    out["density_sweep_2^24"] = sweep
    out["seconds"] = round(time.perf_counter() - t0, 1)
    return out


def chunk_alg_bytes(sets):
    """Algorithmic bytes of the chunked all-pairs sum: over pairs i < j and the
    65536-bit chunks both rows hold, the bytes of both chunks (bitmap 8192 B
    when it holds >= 4096 values, else a u16 list of 2 B per value) --
    sum over chunks c of (rows holding c - 1) x (bytes of c over those rows)."""
    n_c, s_c = {}, {}
    ids_all, sz_all = [], []
    for v in sets:
        if len(v) == 0:
            continue
        ids, cnt = np.unique(np.asarray(v, np.uint32) >> 16, return_counts=True)
        ids_all.append(ids)
        sz_all.append(np.where(cnt >= 4096, 8192, 2 * cnt).astype(np.float64))
    if not ids_all:
        return 0.0
    ids = np.concatenate(ids_all)
    sz = np.concatenate(sz_all)
    m = int(ids.max()) + 1
    n_c = np.bincount(ids, minlength=m).astype(np.float64)
    s_c = np.bincount(ids, weights=sz, minlength=m)
    return float(np.sum(np.maximum(n_c - 1, 0) * s_c))


def sparse_bernoulli_sets_gpu(n, universe, density, seed, device, chunk_rows=2048):
    """Rows of about Bernoulli(density) over [0, universe) for small densities,
    generated in bulk on the GPU: Binomial(universe, density) draws per row,
    uniform positions, sorted, repeats within a row removed (about k^2 / 2U
    per row of k values). Sorted u32 numpy arrays."""
    import torch
    g = np.random.Generator(np.random.PCG64(seed))
    tg = torch.Generator(device=device)
    tg.manual_seed(seed)
    cards = g.binomial(universe, density, size=n)
    out = []
    for r0 in range(0, n, chunk_rows):
        k = torch.from_numpy(cards[r0:r0 + chunk_rows].astype(np.int64)).to(device)
        row = torch.repeat_interleave(torch.arange(len(k), device=device), k)
        pos = torch.randint(0, universe, (int(k.sum().item()),), generator=tg, device=device)
        key = torch.unique(row * universe + pos)                  # sorted, repeats removed
        rr = (key // universe).cpu().numpy()
        vv = (key % universe).to(torch.int64).cpu().numpy().astype(np.uint32)
        cuts = np.searchsorted(rr, np.arange(len(k) + 1))
        out.extend(vv[cuts[i]:cuts[i + 1]] for i in range(len(k)))
    return out


STORM_T_CASES = ("zipf_2^24", "runs_2^26", "haplotypes_20000", "bernoulli_1e-06_2^24_N20000",
                 "bernoulli_1e-05_2^24_N20000", "bernoulli_0.0001_2^24_N20000", "bernoulli_0.001_2^24_N20000",
                 "bernoulli_0.01_2^24", "bernoulli_0.17_2^24")
STORM_T_DEFAULT_CASES = ("zipf_2^24", "bernoulli_1e-06_2^24_N20000", "bernoulli_1e-05_2^24_N20000",
                         "bernoulli_0.0001_2^24_N20000", "bernoulli_0.001_2^24_N20000")


def storm_t_forms(device, cpu_seconds=2.0, only=None):
    """STORM_t (the reference's chunked rows, storm.h:158-178) all-pairs on
    config-3/4/5-shaped corpora: per-pair counts (the packed triangle, i <= j)
    by the chunk kernel alone (the plain per-pair GPU form, at N <= 4096) and
    by the default plan (tensor cores for the heavy rows' pairs, value
    postings for pairs of light rows, chunk kernel for the rest), the default
    plan's sum-only call, and the reference's STORM_pairw_intersect_
    cardinality on 1 core over a prefix of the rows (all-pairs call only)."""
    import ctypes as C
    import importlib
    sb = importlib.import_module("stormbitmaps-internal_b200")
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    R = ol.reference()
    corpora = [
        ("zipf_2^24", lambda: zipf_sets_gpu(4096, 1 << 24, 1.1, 16, 1 << 22, 0xC0F3, device),
         "config 3 shape, N reduced: 4096 rows over 2^24, card ~ Zipf(1.1) on [16, 2^22]"),
        ("runs_2^26", lambda: run_sets_gpu(8192, 1 << 26, 200, 256, 0xC0F4, device),
         "config 4 shape, N reduced: 8192 rows over 2^26, Poisson(200) runs of Geometric(mean 256)"),
        ("haplotypes_20000", lambda: [np.flatnonzero(np.unpackbits(r.view(np.uint8), bitorder="little"))
                                      .astype(np.uint32) for r in
                                      haplotype_rows_gpu(8192, 20000, 32, 0xC0F5, device).cpu().numpy()],
         "config 5a shape, N reduced: 8192 sites x 20000 haplotypes, P(k) ~ 1/k, 32-haplotype carrier blocks"),
    ]
    for d in (1e-6, 1e-5, 1e-4, 1e-3):
        corpora.append((f"bernoulli_{d:g}_2^24_N20000",
                        (lambda d=d: sparse_bernoulli_sets_gpu(20000, 1 << 24, d, int(1e7 * d) + 5, device)),
                        f"config 5b at full N: 20000 rows over 2^24, Bernoulli({d:g})"))
    for d, nn in ((1e-2, 2048), (0.17, 1024)):
        corpora.append((f"bernoulli_{d:g}_2^24",
                        (lambda d=d, nn=nn: bernoulli_sets_gpu(nn, 1 << 24, d, int(1e7 * d) + 5, device)),
                        f"config 5b, N reduced: {nn} rows over 2^24, Bernoulli({d:g})"))
    assert [c[0] for c in corpora] == list(STORM_T_CASES)
    out = {}
    for name, make, desc in corpora:
        if only is not None and name not in ((only,) if isinstance(only, str) else only):
            continue
        t0 = time.perf_counter()
        sets = make()
        n = len(sets)
        pairs = n * (n + 1) // 2
        s = sb.Storm()
        t_add = time.perf_counter()
        for v in sets:
            s.add(v)
        t_add = time.perf_counter() - t_add
        res = {"workload": desc, "pairs_i_le_j": pairs}
        sums = set()
        forms = [("gpu_default", -1.0, -1)]
        if n <= 4096:
            forms.insert(0, ("gpu_chunk_kernel", 0.0, 0))
        buf = np.zeros(pairs, np.uint32)
        # End to end through the C ABI: the first per-pair call packs the rows,
        # uploads them and copies the triangle back to host memory.
        t_e2e = time.perf_counter()
        _, v = s.matrix(buf)
        t_e2e = time.perf_counter() - t_e2e
        sums.add(v)
        res["e2e"] = {"STORM_add_s": round(t_add, 3), "first_matrix_call_s": round(t_e2e, 3),
                      "pairs_per_s_incl_pack_upload_download": pairs / t_e2e,
                      "d2h_bytes": pairs * 4, "transfers": s.last_transfer_ms()}
        res["setup_s"] = round(time.perf_counter() - t0, 1)
        for form, thr, post in forms:
            s.set_dense_block(thr)
            s.set_sparse_postings(post)
            best = None
            for _ in range(2):
                _, v = s.matrix(buf)
                sums.add(v)
                ms = s.last_kernel_ms()
                best = ms if best is None else min(best, ms)
            res[form] = {"pairs_per_s": pairs / (best * 1e-3), "ms": round(best, 3),
                         "tensor_rows": s.last_dense()[0], "postings_rows": s.last_postings_rows()}
        best = None
        for _ in range(2):
            sums.add(s.pairw_intersect_cardinality())
            ms = s.last_kernel_ms()
            best = ms if best is None else min(best, ms)
        res["gpu_default_sum_only_ms"] = round(best, 3)
        # The planner against single-engine plans on the same rows: regret =
        # default / the fastest plan measured - 1 (chunk kernel alone only
        # where it finishes in seconds).
        plans = {"tensor_rows_only": (1e-12, 0, 0), "panel_only": (-1.0, -1, 2), "postings_only": (0.0, 1, 0)}
        if n <= 4096:
            plans["chunk_kernel_only"] = (0.0, 0, 0)
        plan_ms = {"default": res["gpu_default"]["ms"]}
        for pname, (thr, post, pan) in plans.items():
            s.set_dense_block(thr)
            s.set_sparse_postings(post)
            s.set_panel(pan)
            best = None
            for _ in range(2):
                _, v = s.matrix(buf)
                sums.add(v)
                ms = s.last_kernel_ms()
                best = ms if best is None else min(best, ms)
                if best > 2000:
                    break
            plan_ms[pname] = round(best, 3)
        s.set_dense_block(-1.0)
        s.set_sparse_postings(-1)
        s.set_panel(-1)
        fastest = min(plan_ms, key=plan_ms.get)
        res["plans"] = {"ms": plan_ms, "fastest": fastest,
                        "default_regret": round(plan_ms["default"] / plan_ms[fastest] - 1.0, 4)}
        s.close()
        if len(sums) != 1:
            raise RuntimeError(f"{name}: forms disagree {sums}")
        alg = chunk_alg_bytes(sets)
        res["alg_bytes"] = alg
        for form, _, _ in forms:
            res[form]["alg_GBps"] = alg / (res[form]["ms"] * 1e-3) / 1e9
        if R is not None:
            k, rate, secs = 64, None, 0.0
            while True:
                k = min(k, n)
                vals = np.ascontiguousarray(np.concatenate(sets[:k]), dtype=np.uint32)
                offs = np.zeros(k + 1, np.uint64)
                offs[1:] = np.cumsum([len(x) for x in sets[:k]])
                sec = C.c_double(0.0)
                R.ref_storm_sum_timed(vals.ctypes.data_as(ol.u32p), offs.ctypes.data_as(ol.u64p), k, C.byref(sec))
                secs = sec.value
                rate = (k * (k - 1) // 2) / max(secs, 1e-9)
                if secs >= cpu_seconds or k == n:
                    break
                k *= 2
            res["cpu_reference"] = {"pairs_per_s": rate, "cores": 1,
                                    "sample": f"first {k} rows ({k * (k - 1) // 2} pairs i < j, {secs:.2f} s), "
                                              f"STORM_pairw_intersect_cardinality as shipped (all-pairs call only)"}
            res["gpu_default_over_cpu"] = res["gpu_default"]["pairs_per_s"] / rate
            threads = cpu_threads()
            k, rate_mt, secs = 64, None, 0.0
            while True:
                k = min(k, n)
                vals = np.ascontiguousarray(np.concatenate(sets[:k]), dtype=np.uint32)
                offs = np.zeros(k + 1, np.uint64)
                offs[1:] = np.cumsum([len(x) for x in sets[:k]])
                sec = C.c_double(0.0)
                R.ref_storm_sum_mt(vals.ctypes.data_as(ol.u32p), offs.ctypes.data_as(ol.u64p), k, threads,
                                   C.byref(sec))
                secs = sec.value
                rate_mt = (k * (k - 1) // 2) / max(secs, 1e-9)
                if secs >= cpu_seconds or k == n:
                    break
                k *= 2
            res["cpu_reference_all_threads"] = {
                "pairs_per_s": rate_mt, "cores": threads,
                "sample": f"first {k} rows ({k * (k - 1) // 2} pairs i < j, {secs:.2f} s), project harness: "
                          f"the reference's per-pair STORM_bitmap_cont_intersect_cardinality_premade over "
                          f"{threads} threads"}
            res["gpu_default_over_cpu_all_threads"] = res["gpu_default"]["pairs_per_s"] / rate_mt
        if "gpu_chunk_kernel" in res:
            res["gpu_default_over_chunk_kernel"] = (res["gpu_default"]["pairs_per_s"] /
                                                    res["gpu_chunk_kernel"]["pairs_per_s"])
        out[name] = res
        del sets
    return out


TENSOR_KERNELS = ("bb_mma_kernel", "bb_mma_ts_kernel", "bb_mma_ts2_kernel", "bb_mma_2cta_kernel")


def north_star_summary(line):
    """The figures the target names, compactly: the tensor-core kernel's
    fraction of the measured 8-bit peak on the headline workload and on the
    4096 x 65536 configuration; learned-batched vs plain per-tile vs the
    reference CPU driver on the mixed-density corpus, with the selectors'
    regret; each full-size STORM_t configuration's device rate, CPU rate and
    identity check."""
    def g(d, *path):
        for k in path:
            if not isinstance(d, dict) or k not in d:
                return None
            d = d[k]
        return d

    def r3(x):
        return None if x is None else float(f"{x:.4g}")

    ns = {"headline_frac": r3(g(line, "roofline", "frac")), "headline_e2e_pairs_per_s": r3(g(line, "e2e", "value"))}
    at = line.get("autotune_config1")
    if isinstance(at, dict) and "candidates_tops_int8" in at:
        peak = g(line, "roofline", "peak")
        best = max(at["candidates_tops_int8"].values()) if at["candidates_tops_int8"] else None
        ns["config1_best_tops"] = r3(best)
        ns["config1_frac"] = r3(best / peak) if best and peak else None
        ns["config1_kept"] = at.get("kept")
    md = line.get("mixed_density")
    if isinstance(md, dict) and "forms" in md:
        f = md["forms"]
        ns["mixed_density"] = {
            "learned_batched": r3(g(f, "batched_learned_tensor_block", "pairs_per_s")),
            "learned_batched_autotuned": r3(g(f, "batched_learned_autotuned", "pairs_per_s")),
            "plain_per_tile_calibrated": r3(g(f, "plain_per_tile_cost_model", "pairs_per_s")),
            "plain_per_tile_default": r3(g(f, "plain_per_tile_default_model", "pairs_per_s")),
            "cpu_reference": r3(g(md, "cpu_reference_per_tile", "pairs_per_s")),
            "regret_mlp": g(md, "selector", "regret_mlp"),
            "regret_calibrated": g(md, "selector", "regret_calibrated_model"),
            "regret_default": g(md, "selector", "regret_default_model")}
    full = line.get("storm_t_full")
    if isinstance(full, dict):
        for name, r in full.items():
            if isinstance(r, dict) and "device" in r:
                ns[name] = {"device_pairs_per_s": r3(g(r, "device", "pairs_per_s")),
                            "ms": g(r, "device", "ms"),
                            "cpu_1core": r3(g(r, "cpu_reference", "pairs_per_s")),
                            "cpu_all": r3(g(r, "cpu_reference_all_threads", "pairs_per_s")),
                            "exact": g(r, "checked", "identities_hold")}
            elif isinstance(r, dict):
                ns[name] = r
    c5 = line.get("config5a_full")
    if isinstance(c5, dict) and "pairs_per_s" in c5:
        ns["config5a"] = {"pairs_per_s": r3(c5["pairs_per_s"]), "frac": r3(g(c5, "roofline", "frac"))}
    stf = line.get("storm_t")
    if isinstance(stf, dict):
        regret = {name: g(r, "plans", "default_regret") for name, r in stf.items() if isinstance(r, dict)}
        regret = {k: v for k, v in regret.items() if v is not None}
        if regret:
            ns["storm_t_plan_regret"] = regret
    return ns


# ------------------------------------------------------------------ arms
def run_reference_arm(args):
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    import torch
    threads = cpu_threads()
    if not torch.cuda.is_available():
        print(json.dumps({"impl": "reference", "unavailable": "no CUDA device to generate the seeded workload"}))
        return 0
    rows = bernoulli_rows_gpu(args.rows, args.bits, P_RANGE, SEED, torch.device("cuda", 0)).cpu().numpy().view(np.uint64)
    per_step_s = max(2.0, 60.0 / max(1, args.steps + args.warmup))
    for _ in range(args.warmup):
        if reference_sample(rows, min(per_step_s, 3.0), threads) is None:
            print(json.dumps({"impl": "reference",
                              "unavailable": "oracle/_ref/libstorm_ref.so was not built from the reference"}))
            return 0
    rates, total_pairs, total_s, last_rows = [], 0, 0.0, 0
    for _ in range(args.steps):
        rate, pairs, dt, nrows = reference_sample(rows, per_step_s, threads)
        rates.append(rate)
        total_pairs += pairs
        total_s += dt
        last_rows = nrows
    value = total_pairs / total_s
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total_s / args.steps,     # the timed sample of each step
        "ms_per_step_full_triangle_extrapolated": 1e3 * pairs_of(N_ROWS) / value,
        "pairs_per_step_sampled": total_pairs // args.steps,
        "ns_per_pair": 1e9 / value, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64 (AND + popcount)", "data": "synthetic (seeded, generated on the GPU, copied to host)",
        "config": {"workload": f"dense all-bitmap XX^T: {N_ROWS} rows x {M_BITS} bits, p~U[0.05,0.5], u32 i<=j out",
                   "rows": N_ROWS, "bits": M_BITS, "pairs": pairs_of(N_ROWS),
                   "sampled": f"rows 0..{last_rows} of the triangle per step (every j >= i)"},
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": threads, "kind": "reference",
                         "sample": f"{last_rows} rows x all j>=i per step, reference kernel "
                                   f"STORM_get_intersect_count_func({M_BITS // 64}) on {threads} threads, "
                                   f"the reference's cache-blocked traversal (16-row blocks)"},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_b200_arm(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    dist = init_dist(world, "nccl")
    sb = importlib.import_module("stormbitmaps-internal_b200")

    n, m = args.rows, args.bits
    tri = pairs_of(n)
    rows_d = bernoulli_rows_gpu(n, m, P_RANGE, SEED + rank, device)
    w = rows_d.shape[1]
    c = sb.StormContig(m)
    c.set_kernel({"auto": sb.KERNEL_AUTO, "popc": sb.KERNEL_POPC, "mma": sb.KERNEL_MMA,
                  "mma_ss": sb.KERNEL_MMA_SS, "mma_db": sb.KERNEL_MMA_DB, "mma_2cta": sb.KERNEL_MMA_2CTA}[args.kernel])
    c.set_schedule({"auto": sb.SCHED_AUTO, "tiles": sb.SCHED_TILES, "stream_k": sb.SCHED_STREAM_K}[args.schedule])
    rc = sb.lib().STORM_contig_add_bitmaps(c.h, C.cast(rows_d.data_ptr(), sb.u64p), n, w)
    if rc < 0:
        raise sb.StormError(rc, "STORM_contig_add_bitmaps")
    c.upload()
    out_d = torch.empty(tri, dtype=torch.int32, device=device)
    stream = torch.cuda.ExternalStream(c.stream(), device=device)

    # ---- device-resident timing ----
    for _ in range(args.warmup):
        c.matrix_device(out_d.data_ptr(), tri)
    kernel_ms = []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    # Working sets smaller than twice L2 (126 MB) get an L2 flush between
    # steps (a 256 MiB write on the library's stream), timed outside the
    # per-step events; larger ones stream from HBM anyway.
    fits_l2 = n * w * 8 + tri * 4 < 2 * L2_BYTES
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device) if fits_l2 else None
    step_ms = []
    with ClockSampler(local) as clocks:
        if flush is None:
            ev0.record(stream)
        for _ in range(args.steps):
            if flush is not None:
                with torch.cuda.stream(stream):
                    flush.zero_()
                ev0.record(stream)
            s = c.matrix_device(out_d.data_ptr(), tri)
            kernel_ms.append(c.last_kernel_ms())
            if flush is not None:
                ev1.record(stream)
                ev1.synchronize()
                step_ms.append(ev0.elapsed_time(ev1))
        if flush is None:
            ev1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    elapsed_ms = sum(step_ms) if flush is not None else ev0.elapsed_time(ev1)
    elapsed_ms = max_over_ranks(elapsed_ms, dist, device)
    launches = args.steps * c.last_launches()
    kernel_used = {sb.KERNEL_POPC: "bb_popc_kernel", sb.KERNEL_MMA: "bb_mma_ts_kernel",
                   sb.KERNEL_MMA_SS: "bb_mma_kernel", sb.KERNEL_MMA_DB: "bb_mma_ts2_kernel",
                   sb.KERNEL_MMA_2CTA: "bb_mma_2cta_kernel"}.get(c.last_kernel(), "?")
    ms_per_step = elapsed_ms / args.steps
    value = world * tri / (ms_per_step / 1e3)

    # ---- end to end through the C ABI with host buffers ----
    host_in = torch.empty((n, w), dtype=torch.int64, pin_memory=True)
    host_in.copy_(rows_d)
    del rows_d
    host_out = torch.empty(tri, dtype=torch.int32, pin_memory=True)
    L = sb.lib()

    def one_call():
        # STORM_contig_pairw_intersect_matrix_from_host: upload, tiles and
        # copy-back overlapped in one call
        ssum = C.c_uint64(0)
        rc = L.STORM_contig_pairw_intersect_matrix_from_host(c.h, C.cast(host_in.data_ptr(), sb.u64p), n, w,
                                                             C.cast(host_out.data_ptr(), sb.u32p), tri,
                                                             C.byref(ssum))
        if rc < 0:
            raise sb.StormError(rc, "STORM_contig_pairw_intersect_matrix_from_host")
        return int(ssum.value)

    def two_calls():
        # the reference's own shape: add the rows, then the all-pairs call
        L.STORM_contig_clear(c.h)
        rc = L.STORM_contig_add_bitmaps(c.h, C.cast(host_in.data_ptr(), sb.u64p), n, w)
        if rc < 0:
            raise sb.StormError(rc, "STORM_contig_add_bitmaps")
        ssum = C.c_uint64(0)
        rc = L.STORM_contig_pairw_intersect_matrix(c.h, C.cast(host_out.data_ptr(), sb.u32p), tri, C.byref(ssum))
        if rc < 0:
            raise sb.StormError(rc, "STORM_contig_pairw_intersect_matrix")
        return int(ssum.value)

    def timed(fn):
        ms = []
        for it in range(1 + max(1, args.e2e_steps)):
            if dist:
                dist.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            got = fn()
            torch.cuda.synchronize()
            dt = (time.perf_counter() - t0) * 1e3
            if got != s:
                raise RuntimeError(f"device-resident sum {s} != host-buffer sum {got}")
            if it > 0:   # the first iteration (re)allocates the handle's buffers
                ms.append(dt)
        return max_over_ranks(statistics.median(ms), dist, device)

    e2e_two_ms = timed(two_calls)
    e2e_step_ms = timed(one_call)
    e2e_value = world * tri / (e2e_step_ms / 1e3)
    # Self-check of the timed output: two whole rows of the triangle against the oracle.
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    host_rows = host_in.numpy().view(np.uint64)
    host_tri = host_out.numpy().view(np.uint32)
    for i in (0, n // 3):
        base = int(sb.tri_index(n, i, i))
        if not np.array_equal(host_tri[base: base + n - i], ol.contig_row(host_rows, i)):
            raise RuntimeError(f"row {i} of the triangle differs from the oracle")

    # ---- thresholded form (pairs with Jaccard >= t): filter fused into the
    # tensor-core epilogue, no triangle written
    thresh = None
    if args.forms and rank == 0 and world == 1:   # single-GPU characterisation forms
        t_j = 0.3
        try:
            tms, hits = [], 0
            for _ in range(3):
                _, _, _, hits = c.threshold(t_j, cap=1 << 25)
                tms.append(c.last_kernel_ms())
            thresh = {"jaccard_min": t_j, "ms": round(min(tms), 3), "pairs_per_s": tri / (min(tms) * 1e-3),
                      "hits": hits, "hit_fraction": hits / tri, "triangle_bytes_not_written": tri * 4,
                      "vs_full_triangle_kernel_ms": round(statistics.median(kernel_ms), 3)}
        except Exception as e:   # reported, never silently dropped
            thresh = {"error": f"{type(e).__name__}: {e}"}

    # ---- roofline of the dominant kernel ----
    k_ms = statistics.median(kernel_ms)
    if kernel_used in TENSOR_KERNELS:
        ops = 2.0 * tri * m                      # u8 MACs = pairs x row bits, 2 ops each
        achieved = ops / (k_ms / 1e3) / 1e12
        peak, peak_src = tensor_peak_tops(device)
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TOPS (int8)",
                "frac": achieved / peak, "peak_source": peak_src, "tensor8_measured": tensor8_peak(device),
                "algorithmic": f"pairs(i<=j) x {m} bit-MACs x 2 ops", "traffic": args.traffic}
        if args.traffic is None and (n, m) == (N_ROWS, M_BITS) and kernel_used == "bb_mma_ts_kernel":
            roof["traffic"] = TS_TRAFFIC_BENCH_WORKLOAD
            roof["traffic_source"] = ("dram__bytes_read.sum + dram__bytes_write.sum of one launch at 16384 x 262144 "
                                      "(11.24 GB, profiles/bb_mma_ts_dram_16384x262144.md) x 16 (pairs ratio)")
    else:
        ops = 2.0 * tri * m
        achieved = ops / (k_ms / 1e3) / 1e12
        roof = {"bound": "alu", "achieved": achieved, "peak": None, "unit": "Tbit-ops/s", "frac": None,
                "traffic": args.traffic}

    line = {
        "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "ns_per_pair": 1e9 / (value / world),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8 (tcgen05 kind::i8, s32 acc)"
        if kernel_used in TENSOR_KERNELS else "u64 (AND + POPC)",
        "data": "synthetic (seeded Bernoulli rows generated on the GPU)",
        "config": {"workload": f"dense all-bitmap XX^T: {n} rows x {m} bits, p~U[0.05,0.5], u32 i<=j out",
                   "rows": n, "bits": m, "pairs_per_gpu": tri, "kernel": kernel_used, "schedule": args.schedule,
                   "l2": (f"inputs ({n * w * 8 / 1e6:.1f} MB) and outputs ({tri * 4 / 1e6:.1f} MB) fit in twice "
                          f"L2 (126 MB): 256 MiB L2 flush between steps, outside the step events") if fits_l2 else
                         (f"inputs ({n * w * 8 / 2**30:.2f} GiB) and outputs ({tri * 4 / 1e9:.2f} GB) exceed "
                          f"L2 (126 MB); no flush needed"),
                   "parallelism": f"{world} independent instances (weak)"},
        "kernel_ms_median": k_ms,
        "gpu_launches": launches,
        "roofline": roof,
        "clocks": clocks.summary(),
        "e2e": {"value": e2e_value, "unit": "pairs/s", "ms_per_step": e2e_step_ms,
                "h2d_bytes_per_step": int(n * w * 8), "d2h_bytes_per_step": int(tri * 4),
                "call": "STORM_contig_pairw_intersect_matrix_from_host (pinned host rows in, pinned host "
                        "triangle out, overlapped)",
                "two_calls": {"value": world * tri / (e2e_two_ms / 1e3), "ms_per_step": e2e_two_ms,
                              "calls": "STORM_contig_clear + STORM_contig_add_bitmaps + "
                                       "STORM_contig_pairw_intersect_matrix"}},
    }
    if rank == 0 and world == 1 and args.cpu_baseline:   # the CPU baseline is an N=1 figure
        r = reference_sample(host_in.numpy().view(np.uint64), args.cpu_seconds, cpu_threads())
        if r is not None:
            rate, pairs, dt, nrows = r
            line["cpu_baseline"] = {"value": rate, "unit": "pairs/s", "cores": cpu_threads(), "kind": "reference",
                                    "sample": f"rows 0..{nrows} x all j>=i ({pairs} pairs, {dt:.1f} s), reference "
                                              f"AND+popcount kernel via oracle/_ref, cache-blocked traversal"}
        else:
            line["cpu_baseline"] = {"value": None, "unit": "pairs/s", "cores": 0, "kind": "reference",
                                    "sample": "oracle/_ref not built"}
    if thresh is not None:
        line["threshold_form"] = thresh
    if rank == 0 and world == 1 and args.forms:
        # Characterisation forms, each timed (wall seconds in form_seconds).
        # The default run keeps them to a few minutes: the STORM_t table keeps
        # config 5b's densities at N = 20000 and the config-3-shaped corpus
        # (the full-size configurations have their own entries); --all-forms
        # adds the reduced-size duplicates and the whole density sweep.
        secs = {}

        def form(key, fn):
            t1 = time.perf_counter()
            try:
                line[key] = fn()
            except Exception as e:   # reported, never silently dropped
                line[key] = {"error": f"{type(e).__name__}: {e}"}
            secs[key] = round(time.perf_counter() - t1, 1)

        form("mixed_density", lambda: mixed_density_forms(sb, device))
        form("mixed_density_2^24", lambda: mixed_density_forms(sb, device, n=4096, universe=1 << 24,
                                                               samples=1024 if args.all_forms else 256))
        form("configs_4_5", lambda: config45_forms(device, full_sweep=args.all_forms))
        form("storm_t", lambda: storm_t_forms(device, only=None if args.all_forms else STORM_T_DEFAULT_CASES))
        form("storm_t_full", lambda: storm_t_full(device))
        form("autotune_config1", lambda: autotune_config1(sb, device))
        form("config5a_full", lambda: config5a_full(sb, device))
        line["form_seconds"] = secs
    if rank == 0:
        line["north_star"] = north_star_summary(line)   # last, so that the tail of the line keeps it
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--kernel", default="auto", choices=["auto", "popc", "mma", "mma_ss", "mma_db", "mma_2cta"])
    ap.add_argument("--schedule", default="auto", choices=["auto", "tiles", "stream_k"],
                    help="tensor-core work schedule (whole tiles or stream-K; auto picks per launch)")
    ap.add_argument("--rows", type=int, default=N_ROWS)
    ap.add_argument("--bits", type=int, default=M_BITS)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--all-forms", action="store_true",
                    help="also the reduced-size STORM_t corpora and the whole density sweep (longer run)")
    ap.add_argument("--no-forms", dest="forms", action="store_false",
                    help="skip the mixed-density learned/plain/CPU comparison")
    ap.add_argument("--traffic", type=float, default=None,
                    help="dram bytes per launch of the dominant kernel from an ncu capture")
    ap.add_argument("--storm-t-case", default=None, choices=STORM_T_CASES,
                    help="run only this STORM_t corpus of the forms (one JSON line) and exit")
    ap.add_argument("--storm-t-full", default=None, choices=tuple(FULL_CORPORA),
                    help="run only this full-size STORM_t configuration (one JSON line) and exit")
    ap.add_argument("--engine-case", default=None, choices=ENGINE_CASES,
                    help="run one STORM_t engine on a config-3-shaped corpus (one JSON line) and exit")
    ap.add_argument("--mixed-density-only", action="store_true",
                    help="run only the kernel layer's mixed-density forms (one JSON line) and exit")
    ap.add_argument("--mixed-density-batched", action="store_true",
                    help="only the batched cost-model form of that corpus, no selector training (for profiling)")
    args = ap.parse_args()
    if args.mixed_density_batched:
        import torch
        sb = importlib.import_module("stormbitmaps-internal_b200")
        # generated on the host so that a profiler sees only this library's launches
        sets = zipf_sets_gpu(4096, 1 << 20, 1.1, 16, 1 << 18, 0xC0F3, torch.device("cpu"))
        r = sb.StormRows(1 << 20)
        for v in sets:
            r.add(v)
        r.upload()
        res = []
        for _ in range(3):
            s_, st = r.allpairs_sum(sb.POLICY_PERTILE, 64, exec_=sb.EXEC_BATCHED)
            res.append(st["ns_total"] * 1e-6)
        print(json.dumps({"mixed_density_batched_cost_model_ms": res, "sum": s_}), flush=True)
        return 0
    if args.mixed_density_only:
        import torch
        sb = importlib.import_module("stormbitmaps-internal_b200")
        print(json.dumps({"mixed_density": mixed_density_forms(sb, torch.device("cuda", 0))}), flush=True)
        return 0
    if args.engine_case:
        import torch
        print(json.dumps({"engine_case": engine_case(args.engine_case, torch.device("cuda", 0))}), flush=True)
        return 0
    if args.storm_t_full:
        import torch
        print(json.dumps({"storm_t_full": storm_t_full(torch.device("cuda", 0), names=(args.storm_t_full,))}),
              flush=True)
        return 0
    if args.storm_t_case:
        import torch
        print(json.dumps({"storm_t": storm_t_forms(torch.device("cuda", 0), only=args.storm_t_case)}), flush=True)
        return 0
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_b200_arm(args)


if __name__ == "__main__":
    sys.exit(main())
