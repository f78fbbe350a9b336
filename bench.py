#!/usr/bin/env python
"""Benchmark of the GPU spherical harmonic transforms.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]
                    [--workload glq2047|dh2799x16|...]

One step = one forward and one inverse transform of every field of the
workload: MakeGridGLQ then SHExpandGLQ (or the DH pair).  The metric is
transforms/s, one transform being one direction of one field, summed over
all GPUs.  Inputs are seeded synthetic power-law coefficients (no dataset is
involved); nodes and weights come from the GPU PreGLQ.

Prints one JSON line (rank 0).  Multi-GPU runs (torchrun) are independent
replicas: the transforms of a field do not shard across GPUs in this
workload, each rank runs the same per-GPU work and the slowest rank's time
is used (weak scaling).

--impl reference times the reference algorithm on the host cores: the CPU
oracle (a statement-by-statement C restatement of the SHTOOLS Fortran, which
cannot be compiled here) on a bounded sample of ring pairs, all host threads.
"""
import argparse
import concurrent.futures
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "transforms/s at lmax 2047 & 2799: mixed-prec vs FP64 GPU, rel err vs FP64"

WORKLOADS = {
    # the headline workload: plain FP64 GLQ, single field, lmax 2047, 2048 x
    # 4095 grid
    "glq2047": dict(kind="glq", lmax=2047, nfield=1, sampling=1, beta=2.0,
                    seed=2000),
    # 16 DH fields, lmax 2799, sampling 2, FP64 grids
    "dh2799x16": dict(kind="dh", lmax=2799, nfield=16, sampling=2, beta=3.0,
                      seed=5000),
    # 16 DH fields, lmax 1023, sampling 2 (2048 x 4096): the mixed-precision
    # kernels at a size whose P_lm digit table (about 5 GB) profiles quickly
    "dh1023x16": dict(kind="dh", lmax=1023, nfield=16, sampling=2, beta=3.0,
                      seed=5500),
    # 2 DH fields, lmax 2399, sampling 2 (4800 x 9600): the long even-ring
    # FFT build (complex half length 4800) at a size that profiles quickly
    "dh2399x2": dict(kind="dh", lmax=2399, nfield=2, sampling=2, beta=3.0,
                     seed=5700),
    # 2 DH fields, lmax 2799, sampling 2 (5600 x 11200): the radix-10 passes
    # of the long even-ring FFT (half length 5600 = 7 * 10 * 10 * 8)
    "dh2799x2": dict(kind="dh", lmax=2799, nfield=2, sampling=2, beta=3.0,
                     seed=5800),
    # 8 DH fields, lmax 719, sampling 2
    "dh719x8": dict(kind="dh", lmax=719, nfield=8, sampling=2, beta=2.0,
                    seed=3000),
    # complex DH (MakeGridDHC / SHExpandDHC): 8 fields, lmax 719, sampling 2
    "dhc719x8": dict(kind="dhc", lmax=719, nfield=8, sampling=2, beta=2.0,
                     seed=3500),
    # MakeGradientDH: 8 fields, lmax 719, sampling 2
    "gradient719x8": dict(kind="gradient", lmax=719, nfield=8, sampling=2, beta=2.0,
                          seed=3700),
    # MakeGravGridDH: 8 fields, lmax 719, sampling 2, on a
    # rotating ellipsoid with the normal gravity removed
    "gravity719x8": dict(kind="gravity", lmax=719, nfield=8, sampling=2, beta=2.0,
                         seed=3800),
    # SHMultiply: one pair of fields of lmax 1024 and 1023 into lmax 2047 (the
    # GLQ grid of the headline configuration, 2048 x 4095)
    "multiply1024": dict(kind="multiply", lmax=1024, lmax2=1023, nfield=1, sampling=1,
                         beta=2.0, seed=2100),
    # one DH field, lmax 255, sampling 2
    "dh255": dict(kind="dh", lmax=255, nfield=1, sampling=2, beta=2.0,
                  seed=1000),
    # 16 DH fields, lmax 2799, sampling 2, float32 grids and float64
    # coefficients; synthesis, analysis and the adjoint backward of a
    # weighted L2 misfit per step (3 transforms per field)
    "dh2799x16_grad": dict(kind="dh_grad", lmax=2799, nfield=16, sampling=2,
                           beta=3.0, seed=5000),
    # 4096 GLQ fields of lmax ~ U{31..511}, each on its own grid,
    # one persistent Legendre launch per direction, replayed as CUDA graphs
    "glq_uneven4096": dict(kind="glq_batch", lmax=511, lmin=31, nfield=4096,
                           sampling=1, beta=2.0, seed=4000),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--workload", default="glq2047", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="fp64",
                    choices=["fp64", "int8x6", "int8x7", "int8x6-table", "int8x7-table"],
                    help="Legendre sums: FP64, or the INT8 tensor-core error-free split "
                         "with 6 or 7 byte digits (real DH/GLQ workloads): the synthesis "
                         "from the recursion, or (-table) both directions from the "
                         "plan's P_lm digit table")
    ap.add_argument("--no-2799", action="store_true",
                    help="skip the FP64 / mixed-precision comparisons (glq2047 and "
                         "16 DH fields at lmax 2799) that the default workload adds to "
                         "its line")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="use the default Legendre tile shapes instead of tuning "
                         "each plan once before the warm-up (shtools_b200.autotune)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="target duration of the CPU baseline sample")
    return ap.parse_args()


def bench_config(args, w, world):
    """The workload description printed by both arms (identical dictionaries,
    so a reader can match the GPU line with the reference line)."""
    return {"workload": args.workload, "kind": w["kind"], "lmax": w["lmax"],
            "fields_per_gpu": w["nfield"], "sampling": w["sampling"],
            "precision": getattr(args, "precision", "fp64"),
            "step": "synthesis + analysis",
            "parallelism": "replicas" if world > 1 else "single GPU"}


def batch_lmaxes(w):
    """Seeded lmax of every field of a batched workload."""
    import numpy as np
    rng = np.random.default_rng(w["seed"])
    return [int(x) for x in rng.integers(w["lmin"], w["lmax"] + 1, w["nfield"])]


def legendre_flops(w, nsums, L=None):
    """Algorithmic FP64 flops of one Legendre-stage launch that evaluates
    `nsums` coefficient sets on one grid: per ring pair and (l, m), 4 for the
    three-term recursion, once per grid, and 4 for the two multiply-adds of
    each contraction (F_rec + nsums * F_contr, each 2*nlat*N_lm).  One field
    is 8 flops per (pair, l, m)."""
    if w["kind"] == "glq_batch" and L is None:
        from collections import Counter
        cnt = Counter(batch_lmaxes(w))
        return sum(legendre_flops(dict(w, kind="glq"), n, l) for l, n in cnt.items())
    L = w["lmax"] if L is None else L
    nlm = (L + 1) * (L + 2) // 2
    nlat = L + 1 if w["kind"] in ("glq", "glq_batch") else 2 * L + 2
    return 4.0 * (nlat / 2.0) * nlm * (1 + nsums)


def flops_per_transform(w, L=None):
    """Legendre-stage flops of one single-field transform (8 per pair and (l, m))."""
    return legendre_flops(dict(w, kind="glq" if w["kind"] == "glq_batch" else w["kind"]), 1, L)


def fft_classes(lmaxes):
    """Number of FFT kernel classes a GLQ batch launches per FFT stage: the
    ring length (n = 2 lmax + 1, or its Bluestein length, the smallest
    7-smooth number >= 2n - 1, when n has a prime factor above 13) decides
    between radices <= 8 and a factor 11 or 13, and between 128-thread CTAs
    (length <= 512) and larger ones."""
    def smooth7(x):
        for p in (2, 3, 5, 7):
            while x % p == 0:
                x //= p
        return x == 1
    classes = set()
    for L in set(lmaxes):
        n, odd, r = 2 * L + 1, [], 2 * L + 1
        for p in (3, 5, 7, 11, 13):
            while r % p == 0:
                r //= p
                odd.append(p)
        if r == 1:
            length, full = n, any(p > 8 for p in odd)
        else:
            length = 2 * n - 1
            while not smooth7(length):
                length += 1
            full = False
        classes.add((full, length > 512))
    return len(classes)


def power_law(L, seed, beta, cplx=False):
    from shtools_b200.synthetic import power_law_cilm, power_law_cilm_complex
    return (power_law_cilm_complex if cplx else power_law_cilm)(L, seed, beta)


# ---------------------------------------------------------------------------
# CPU baseline: the oracle on all host threads, bounded sample of ring pairs
# ---------------------------------------------------------------------------
def cpu_sample_batch(w, seconds, threads):
    """CPU baseline of a batched workload: the first fields of the seeded
    lmax list (random order, so their mean cost is that of the batch),
    whole synthesis + analysis per field, one field per thread at a time."""
    import numpy as np
    from oracle import oracle as O
    lm = batch_lmaxes(w)

    def run(i):
        L = lm[i]
        c = power_law(L, w["seed"] + i, w["beta"])
        z, wt = O.shglq(L)
        g = O.makegrid_glq(c, zero=z)
        O.shexpand_glq(g, w=wt, zero=z)

    t0 = time.perf_counter()
    run(0)
    t1 = max(time.perf_counter() - t0, 1e-4)
    k = max(threads, min(len(lm), int(seconds * threads / t1)))

    def one_step():
        t0 = time.perf_counter()
        with concurrent.futures.ThreadPoolExecutor(threads) as ex:
            list(ex.map(run, range(k)))
        dt = time.perf_counter() - t0
        return 2.0 * k / dt, dt

    sample = ("first %d of %d fields (seeded lmax in [%d, %d]), whole synthesis + "
              "analysis per field, %d threads" % (k, len(lm), w["lmin"], w["lmax"], threads))
    return one_step, sample, threads


def cpu_sample(w, seconds, threads=None):
    import numpy as np
    from oracle import oracle as O
    L = w["lmax"]
    threads = threads or len(os.sched_getaffinity(0))
    if w["kind"] == "glq_batch":
        return cpu_sample_batch(w, seconds, threads)
    c = power_law(L, w["seed"], w["beta"])
    if w["kind"] == "glq":
        zero, wt = O.shglq(L)
        npair = (L + 2) // 2
        grid = np.random.default_rng(1).standard_normal((L + 1, 2 * L + 1))
    else:
        n = 2 * L + 2
        npair = n // 2 + 1
        grid = np.random.default_rng(1).standard_normal((n, w["sampling"] * n))

    def run(lo, hi):
        if w["kind"] == "glq":
            O.makegrid_glq(c, zero=zero, pair_window=(lo, hi))
            O.shexpand_glq(grid, w=wt, zero=zero, pair_window=(lo, hi))
        else:
            O.makegrid_dh(c, sampling=w["sampling"], pair_window=(lo, hi))
            O.shexpand_dh(grid, sampling=w["sampling"], pair_window=(lo, hi))

    # calibrate: one pair on one thread
    t0 = time.perf_counter()
    run(npair // 3, npair // 3 + 1)
    t1 = max(time.perf_counter() - t0, 1e-4)
    per_thread = max(1, min(npair // threads if threads <= npair else 1,
                            int(seconds / t1)))
    windows = []
    stride = max(1, npair // threads)
    for t in range(threads):
        lo = min(npair - per_thread, (t * stride) % max(1, npair - per_thread + 1))
        windows.append((max(0, lo), max(0, lo) + per_thread))

    def one_step():
        t0 = time.perf_counter()
        with concurrent.futures.ThreadPoolExecutor(threads) as ex:
            list(ex.map(lambda wd: run(*wd), windows))
        dt = time.perf_counter() - t0
        pairs_done = per_thread * threads
        # each (synthesis + analysis) over all pairs is 2 transforms of one field
        transforms = 2.0 * pairs_done / npair
        return transforms / dt, dt

    sample = ("%d ring pairs of %d per thread x %d threads, synthesis+analysis, "
              "single field; transforms/s scaled by the ring fraction"
              % (per_thread, npair, threads))
    return one_step, sample, threads


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clock and clock-event reasons sampled during the timed region.

    Polls NVML every millisecond from a background thread (timed regions of
    a few milliseconds still get samples); falls back to `nvidia-smi -lms`
    when NVML is unavailable.  Reads settings only, changes nothing."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40),
               ("sw_thermal_slowdown", 0x20), ("sw_power_cap", 0x4))

    def __init__(self, index):
        self.index = index
        self.sm = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._nvml = None
        self.proc = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self._physical_index())
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self._nvml = (pynvml, h)
            self._sample()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
        except Exception:
            self._nvml = None
            self._start_smi()
        return self

    def _physical_index(self):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        if vis:
            try:
                return int(vis.split(",")[self.index])
            except (ValueError, IndexError):
                pass
        return self.index

    def _sample(self):
        pynvml, h = self._nvml
        self.sm.append(float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)))
        try:
            r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
        except AttributeError:
            r = pynvml.nvmlDeviceGetCurrentClocksThrottleReasons(h)
        for name, bit in self.REASONS:
            if r & bit:
                self.reasons.add(name)

    def _poll(self):
        while not self._stop.is_set():
            try:
                self._sample()
            except Exception:
                return
            self._stop.wait(0.001)

    def _start_smi(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read_smi, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read_smi(self):
        for line in self.proc.stdout:
            f = [x.strip() for x in line.split(",")]
            try:
                self.sm.append(float(f[0]))
                self.max_mhz = float(f[1])
            except (ValueError, IndexError):
                continue
            for (name, _), v in zip(self.REASONS, f[2:6]):
                if v.lower().startswith("active"):
                    self.reasons.add(name)

    def __exit__(self, *a):
        self._stop.set()
        if self._nvml is not None:
            try:
                self._sample()          # one reading at the end of the region
            except Exception:
                pass
            self.thread.join(timeout=1)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.sm:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [],
                    "samples": 0}
        return {"sm_mhz": statistics.median(self.sm), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.sm),
                "source": "nvml" if self._nvml is not None else "nvidia-smi"}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def fp64_peak(torch, dev):
    """Measured FP64 FMA throughput of this GPU (TFLOP/s), from the probe."""
    import ctypes
    path = os.path.join(ROOT, "shtools_b200", "lib", "libshtc_probe.so")
    lib = ctypes.CDLL(path)
    lib.shtc_probe_dfma.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_void_p]
    props = torch.cuda.get_device_properties(dev)
    blocks = props.multi_processor_count * 8
    iters = 4096
    out = torch.empty(blocks * 256, dtype=torch.float64, device=dev)
    st = torch.cuda.current_stream(dev)
    best = 0.0
    for rep in range(4):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(st)
        rc = lib.shtc_probe_dfma(ctypes.c_void_p(out.data_ptr()), blocks, iters,
                                 ctypes.c_void_p(st.cuda_stream))
        b.record(st)
        b.synchronize()
        assert rc == 0
        ms = a.elapsed_time(b)
        flops = blocks * 256.0 * iters * 16 * 8 * 2
        if rep > 0:
            best = max(best, flops / (ms * 1e-3) / 1e12)
    return best


def max_over_ranks(x, device=None):
    """Max of a float over all ranks of the default process group (the
    slowest replica sets the time); identity without a process group."""
    import torch
    if not (torch.distributed.is_available() and torch.distributed.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def load_traffic(name):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f).get(name)
    except Exception:
        return None


def batch_inputs(torch, b, w, dev):
    """Seeded power-law coefficients of every field, generated on the device
    directly in the batch layout (S(l) = (l+1)^-beta)."""
    flat = b.empty_cilm()
    gen = torch.Generator(device=dev).manual_seed(w["seed"])
    for g, (plan, nf) in enumerate(zip(b.plans, b.counts)):
        D = plan.lc + 1
        o = int(b.cilm_off[g])
        v = flat[o:o + nf * 2 * D * D].view(nf, 2, D, D)
        v.normal_(generator=gen)
        l = torch.arange(D, dtype=torch.float64, device=dev)
        sc = torch.sqrt((l + 1.0) ** (-w["beta"]) / (2 * l + 1.0))
        mask = (l[:, None] >= l[None, :]).to(torch.float64)
        v.mul_(sc[None, None, :, None] * mask)
        v[:, 1, :, 0] = 0.0
    return flat


def run_cuda_batch(args, w, rank, world, local_rank):
    import numpy as np
    import torch
    from shtools_b200 import _lib
    from shtools_b200.batch import Batch

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    lib = _lib.load()
    lm = batch_lmaxes(w)
    b = Batch.glq(lm, device=dev)
    c = batch_inputs(torch, b, w, dev)
    gs, sin_, sout = b.graph("synthesis")
    ga, ain, aout = b.graph("analysis")
    sin_.copy_(c)
    st = torch.cuda.current_stream(dev)

    def step():
        gs.replay()
        ain.copy_(sout)
        ga.replay()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    # round-trip accuracy per degree over all fields (size-independent check)
    err = 0.0
    for i in range(0, len(lm), max(1, len(lm) // 64)):
        x = b.cilm_view(c, i).cpu().numpy()
        y = b.cilm_view(aout, i).cpu().numpy()
        num = np.sqrt(((y - x) ** 2).sum(axis=(0, 2)))
        den = np.sqrt((x ** 2).sum(axis=(0, 2)))
        err = max(err, float((num / np.where(den > 0, den, 1)).max()))
    peak = fp64_peak(torch, dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    torch.cuda.synchronize(dev)
    with ClockSampler(local_rank) as clk:
        for i in range(args.steps):
            flush.fill_(float(i))
            evs[i][0].record(st)
            step()
            evs[i][1].record(st)
        torch.cuda.synchronize(dev)
    total_ms = max_over_ranks(sum(a.elapsed_time(b_) for a, b_ in evs), dev)
    F = w["nfield"]
    value = 2.0 * F * args.steps * world / (total_ms * 1e-3)
    # per-kernel timing (eager, outside the graphs)
    import ctypes
    lib.shtc_timing_enable(1)
    for _ in range(2):
        b.synthesis(c, sout)
        b.analysis(sout, aout)
    torch.cuda.synchronize(dev)
    lib.shtc_timing_enable(0)
    ms = (ctypes.c_double * 6)()
    cnt = (ctypes.c_int * 6)()
    lib.shtc_timing_collect(ms, cnt, 6)
    names = ["pack", "legendre_synth", "fft_c2r", "fft_r2c", "legendre_anal", "unpack"]
    dom = max((1, 4), key=lambda i: ms[i])
    per_launch_ms = ms[dom] / max(1, cnt[dom])
    fl = legendre_flops(w, None)
    achieved = fl / (per_launch_ms * 1e-3) / 1e12
    # end to end: host coefficients in, host coefficients out
    c_host = c.cpu().pin_memory()
    g_host = torch.empty(sout.shape, dtype=torch.float64).pin_memory()
    b_host = torch.empty(aout.shape, dtype=torch.float64).pin_memory()
    a = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    a.record(st)
    e2e_steps = 2
    for _ in range(e2e_steps):
        sin_.copy_(c_host, non_blocking=True)
        gs.replay()
        g_host.copy_(sout, non_blocking=True)
        ain.copy_(g_host, non_blocking=True)
        ga.replay()
        b_host.copy_(aout, non_blocking=True)
    e.record(st)
    torch.cuda.synchronize(dev)
    e2e_ms = max_over_ranks(a.elapsed_time(e), dev)
    return {
        "metric": METRIC, "value": value, "unit": "transforms/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic seeded power-law coefficients, S(l)=(l+1)^-%g" % w["beta"],
        "config": {"workload": args.workload, "kind": "glq batch, uneven lmax",
                   "fields_per_gpu": F, "lmax_range": [w["lmin"], w["lmax"]],
                   "distinct_grids": len(b.plans), "precision": "fp64",
                   "step": "synthesis + analysis of every field, two CUDA graphs",
                   "l2": "flushed between steps (256 MiB write, outside step events)",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "roofline": {"kernel": names[dom], "bound": "fp64", "achieved": achieved,
                     "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak else None,
                     "peak_source": "measured FP64 FMA probe, this run",
                     "flops_per_launch": fl, "traffic": load_traffic(
                         "%s_%s" % (names[dom], args.workload))},
        "stages": {names[i]: {"ms_per_launch": (ms[i] / cnt[i]) if cnt[i] else None,
                              "launches": cnt[i]} for i in range(6)},
        "roundtrip_max_perdeg_err": err,
        "e2e": {"value": 2.0 * F * e2e_steps * world / (e2e_ms * 1e-3),
                "unit": "transforms/s", "steps": e2e_steps,
                "h2d_bytes_per_step": c_host.numel() * 8 + g_host.numel() * 8,
                "d2h_bytes_per_step": g_host.numel() * 8 + b_host.numel() * 8,
                "path": "batch graphs from pinned host buffers"},
        # per step: pack, Legendre and unpack launches, and each FFT stage one
        # launch per FFT class present (radices <= 8 / with 11 or 13)
        "gpu_launches": (int(sum(cnt)) // 2 + 2 * (fft_classes(lm) - 1)) * args.steps,
        "clocks": clk.summary(),
    }


def run_cuda_grad(args, w, rank, world, local_rank):
    """Synthesis to float32 grids, weighted L2 misfit and its adjoint
    backward, analysis to float64 coefficients: three transforms per field
    per step, all through the public torch API."""
    import numpy as np
    import torch
    import shtools_b200 as sht
    from shtools_b200 import _lib

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    lib = _lib.load()
    L, F, s_ = w["lmax"], w["nfield"], w["sampling"]
    c = torch.from_numpy(np.stack([power_law(L, w["seed"] + i, w["beta"])
                                   for i in range(F)])).to(dev)
    d = sht.MakeGridDH(torch.from_numpy(np.stack([power_law(L, w["seed"] + 500 + i,
                                                            w["beta"])
                                                  for i in range(F)])).to(dev),
                       sampling=s_, dtype=torch.float32)
    n = 2 * L + 2
    wt = torch.sin(torch.pi * (torch.arange(n, device=dev, dtype=torch.float32) + 0.5)
                   / n)[:, None]
    st = torch.cuda.current_stream(dev)

    last = {}

    def step(prec=args.precision):
        cr = c.detach().requires_grad_(True)
        g = sht.MakeGridDH(cr, sampling=s_, dtype=torch.float32, precision=prec)
        loss = (wt * (g - d) ** 2).sum()
        loss.backward()
        back = sht.SHExpandDH(g.detach(), sampling=s_, dtype=torch.float64, precision=prec)
        last["g"] = g
        return cr.grad, back

    def perdeg(a, b):
        dd = (a - b).pow(2).sum(dim=(1, 3)).sqrt()
        nn = b.pow(2).sum(dim=(1, 3)).sqrt()
        return float(torch.where(nn > 0, dd / nn, dd).max())

    for _ in range(args.warmup):
        grad, back = step()
    torch.cuda.synchronize(dev)
    mixed_err = None
    if args.precision != "fp64":
        # FP64 on the mixed step's own float32 grid: the analysis of that
        # grid, and the adjoint of the same misfit cotangent, so that the
        # comparison holds the mixed arithmetic alone (two float32 grids
        # would differ by rounding flips at ~1e-7 of the field)
        g32 = last["g"].detach()
        cr64 = c.detach().requires_grad_(True)
        gr = sht.MakeGridDH(cr64, sampling=s_, dtype=torch.float32)
        gr.backward(2.0 * wt * (g32 - d))
        back64 = sht.SHExpandDH(g32, sampling=s_, dtype=torch.float64)
        mixed_err = {"gradient_max_perdeg_rel_err_vs_fp64": perdeg(grad, cr64.grad),
                     "analysis_max_perdeg_rel_err_vs_fp64": perdeg(back, back64),
                     "reference": "FP64 adjoint of the same cotangent and FP64 analysis "
                                  "of the same float32 grid",
                     "status": sht.mixed_status(dev)}
        del gr, back64, cr64
    last.clear()
    bb = back.cpu().numpy()
    cc = c.cpu().numpy()
    num = np.sqrt(((bb - cc) ** 2).sum(axis=(1, 3)))
    den = np.sqrt((cc ** 2).sum(axis=(1, 3)))
    rt_err = float((num / np.where(den > 0, den, 1)).max())
    peak = fp64_peak(torch, dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    torch.cuda.synchronize(dev)
    lib.shtc_timing_enable(1)
    with ClockSampler(local_rank) as clk:
        for i in range(args.steps):
            flush.fill_(float(i))
            evs[i][0].record(st)
            step()
            evs[i][1].record(st)
        torch.cuda.synchronize(dev)
    lib.shtc_timing_enable(0)
    import ctypes
    ms = (ctypes.c_double * 6)()
    cnt = (ctypes.c_int * 6)()
    lib.shtc_timing_collect(ms, cnt, 6)
    total_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in evs), dev)
    value = 3.0 * F * args.steps * world / (total_ms * 1e-3)
    names = ["pack", "legendre_synth", "fft_c2r", "fft_r2c", "legendre_anal", "unpack"]
    dom = max((1, 4), key=lambda i: ms[i])
    per_launch_ms = ms[dom] / max(1, cnt[dom])
    fl = legendre_flops(w, F)
    achieved = fl / (per_launch_ms * 1e-3) / 1e12
    return {
        "metric": METRIC, "value": value, "unit": "transforms/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 (float32 grids)",
        "data": "synthetic seeded power-law coefficients, S(l)=(l+1)^-%g" % w["beta"],
        "config": {"workload": args.workload, "kind": "dh", "lmax": L,
                   "fields_per_gpu": F, "sampling": s_,
                   "precision": ("fp64" if args.precision == "fp64" else args.precision) +
                                " Legendre sums, float32 grids, float64 coefficients",
                   "step": "synthesis + weighted L2 misfit backward (adjoint) + analysis",
                   "l2": "flushed between steps (256 MiB write, outside step events)",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "roofline": {"kernel": names[dom], "bound": "fp64", "achieved": achieved,
                     "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak else None,
                     "peak_source": "measured FP64 FMA probe, this run",
                     "flops_per_launch": fl, "traffic": None},
        "stages": {names[i]: {"ms_per_launch": (ms[i] / cnt[i]) if cnt[i] else None,
                              "launches": cnt[i]} for i in range(6)},
        "roundtrip_max_perdeg_err": rt_err,
        "mixed_vs_fp64": mixed_err,
        "gpu_launches": int(sum(cnt)),
        "clocks": clk.summary(),
    }


# MakeGravGridDH workload parameters: Mars-like GM, reference radius,
# ellipsoid and rotation; total is the gravity disturbance
GRAV = dict(gm=4.2828372e13, r0=3396000.0, a=3395428.0, f=0.00589, omega=7.088218e-5)


def run_cuda_gradient(args, w, rank, world, local_rank):
    """MakeGradientDH (one transform per field, theta and phi grids) or
    MakeGravGridDH (one transform per field, rad, theta, phi, total and pot
    grids) of every field per step, through the public torch API."""
    import numpy as np
    import torch
    import shtools_b200 as sht
    from shtools_b200 import _lib
    from shtools_b200.pipeline import pipelined

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    lib = _lib.load()
    L, F, s_ = w["lmax"], w["nfield"], w["sampling"]
    grav = w["kind"] == "gravity"
    cs = np.stack([power_law(L, w["seed"] + i, w["beta"]) for i in range(F)])
    if grav:
        cs *= 1e-3
        cs[:, 0, 0, 0] = 1.0
        g = GRAV
        step = lambda x: sht.MakeGravGridDH(x, g["gm"], g["r0"], a=g["a"], f=g["f"],
                                            sampling=s_, omega=g["omega"], normal_gravity=1)
    else:
        step = lambda x: sht.MakeGradientDH(x, sampling=s_)
    c_host = torch.from_numpy(cs).pin_memory()
    c = c_host.to(dev)
    st = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        outs0 = step(c)
    torch.cuda.synchronize(dev)
    # size-independent check: the phi component of a zonal field (m = 0) is 0
    zonal = c.clone()
    zonal[:, :, :, 1:] = 0.0
    zero_phi = float(step(zonal)[2 if grav else 1].abs().max().item())
    peak = fp64_peak(torch, dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    torch.cuda.synchronize(dev)
    lib.shtc_timing_enable(1)
    with ClockSampler(local_rank) as clk:
        for i in range(args.steps):
            flush.fill_(float(i))
            evs[i][0].record(st)
            step(c)
            evs[i][1].record(st)
        torch.cuda.synchronize(dev)
    lib.shtc_timing_enable(0)
    import ctypes
    ms = (ctypes.c_double * 6)()
    cnt = (ctypes.c_int * 6)()
    lib.shtc_timing_collect(ms, cnt, 6)
    total_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in evs), dev)
    value = 1.0 * F * args.steps * world / (total_ms * 1e-3)
    # end to end: host coefficients in, every host grid out, pipelined
    outs = [tuple(torch.empty(tuple(o.shape), dtype=o.dtype).pin_memory() for o in outs0)
            for _ in range(2)]
    e2e_steps = max(2, args.steps)
    pipelined(step, [(c_host,)] * 2, outs, device=dev)
    torch.cuda.synchronize(dev)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(st)
    pipelined(step, [(c_host,)] * e2e_steps, [outs[i % 2] for i in range(e2e_steps)],
              device=dev)
    b.record(st)
    torch.cuda.synchronize(dev)
    e2e_ms = max_over_ranks(a.elapsed_time(b), dev)
    names = ["pack", "legendre_synth", "fft_c2r", "fft_r2c", "legendre_anal", "unpack"]
    per_launch_ms = ms[1] / max(1, cnt[1])
    fl = legendre_flops(w, 3 * F)        # three Legendre sums per field, one recursion
    achieved = fl / (per_launch_ms * 1e-3) / 1e12
    if grav:
        kind, what = "dh gravity", ("MakeGravGridDH of every field (rad, theta, phi, "
                                    "total and pot grids; ellipsoid, rotation, "
                                    "normal gravity removed)")
        # pack stage: ring tables, powers, pack; FFT stage: combination (with
        # the centrifugal terms), 4 c2r, magnitude / normal-gravity pass
        launches = 3 * int(cnt[0]) + int(cnt[1]) + 6 * int(cnt[2])
        # the radial factor adds 2 multiplies per (pair, l, m) to the recursion
        fl_note = "recursion + 3 contractions per (pair, l, m); q^l factor not counted"
    else:
        kind, what = "dh gradient", "MakeGradientDH of every field (theta and phi grids)"
        # the FFT stage holds 3 launches (combination, theta c2r, phi c2r)
        launches = int(sum(cnt)) + 2 * int(cnt[2])
        fl_note = "recursion + 3 contractions per (pair, l, m)"
    res = {
        "metric": METRIC, "value": value, "unit": "transforms/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic seeded power-law coefficients, S(l)=(l+1)^-%g" % w["beta"],
        "config": {"workload": args.workload, "kind": kind, "lmax": L,
                   "fields_per_gpu": F, "sampling": s_, "precision": "fp64",
                   "step": what,
                   "l2": "flushed between steps (256 MiB write, outside step events)",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "roofline": {"kernel": "legendre_synth", "bound": "fp64", "achieved": achieved,
                     "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak else None,
                     "peak_source": "measured FP64 FMA probe, this run",
                     "flops_per_launch": fl, "flops_note": fl_note, "traffic": None},
        "stages": {names[i]: {"ms_per_launch": (ms[i] / cnt[i]) if cnt[i] else None,
                              "launches": cnt[i]} for i in range(6)},
        "zonal_field_max_abs_phi": zero_phi,
        "e2e": {"value": 1.0 * F * e2e_steps * world / (e2e_ms * 1e-3),
                "unit": "transforms/s", "steps": e2e_steps,
                "h2d_bytes_per_step": c_host.numel() * 8,
                "d2h_bytes_per_step": sum(o.numel() for o in outs[0]) * 8,
                "path": "public torch API on pinned host buffers, pipelined on 3 streams"},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    return res


def run_cuda_multiply(args, w, rank, world, local_rank):
    """SHMultiply of pairs of fields of degree lmax into degree 2*lmax (two
    GLQ syntheses and one analysis per product), through the public torch
    API."""
    import numpy as np
    import torch
    import shtools_b200 as sht
    from shtools_b200 import _lib
    from shtools_b200.pipeline import pipelined

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    lib = _lib.load()
    L, L2, F = w["lmax"], w["lmax2"], w["nfield"]
    c1h = torch.from_numpy(np.stack([power_law(L, w["seed"] + i, w["beta"])
                                     for i in range(F)])).pin_memory()
    c2h = torch.from_numpy(np.stack([power_law(L2, w["seed"] + 100 + i, w["beta"])
                                     for i in range(F)])).pin_memory()
    c1, c2 = c1h.to(dev), c2h.to(dev)
    st = torch.cuda.current_stream(dev)
    step = lambda a, b: sht.SHMultiply(a, b)
    for _ in range(args.warmup):
        out = step(c1, c2)
    torch.cuda.synchronize(dev)
    # size-independent check: multiplying by the constant field 1 is the identity
    one = torch.zeros((F, 2, 1, 1), dtype=torch.float64, device=dev)
    one[:, 0, 0, 0] = 1.0
    ident = step(c1, one)
    ident_err = float((ident[..., :L + 1, :L + 1] - c1).abs().max().item() /
                      c1.abs().max().item())
    peak = fp64_peak(torch, dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    torch.cuda.synchronize(dev)
    lib.shtc_timing_enable(1)
    with ClockSampler(local_rank) as clk:
        for i in range(args.steps):
            flush.fill_(float(i))
            evs[i][0].record(st)
            step(c1, c2)
            evs[i][1].record(st)
        torch.cuda.synchronize(dev)
    lib.shtc_timing_enable(0)
    import ctypes
    ms = (ctypes.c_double * 6)()
    cnt = (ctypes.c_int * 6)()
    lib.shtc_timing_collect(ms, cnt, 6)
    total_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in evs), dev)
    value = 3.0 * F * args.steps * world / (total_ms * 1e-3)
    outs = [(torch.empty(tuple(out.shape), dtype=out.dtype).pin_memory(),) for _ in range(2)]
    e2e_steps = max(2, args.steps)
    pipelined(step, [(c1h, c2h)] * 2, outs, device=dev)
    torch.cuda.synchronize(dev)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(st)
    pipelined(step, [(c1h, c2h)] * e2e_steps, [outs[i % 2] for i in range(e2e_steps)],
              device=dev)
    b.record(st)
    torch.cuda.synchronize(dev)
    e2e_ms = max_over_ranks(a.elapsed_time(b), dev)
    names = ["pack", "legendre_synth", "fft_c2r", "fft_r2c", "legendre_anal", "unpack"]
    wl = dict(w, kind="glq", lmax=L + L2)
    dom = max((1, 4), key=lambda i: ms[i])
    per_launch_ms = ms[dom] / max(1, cnt[dom])
    fl = legendre_flops(wl, F * (2 if dom == 1 else 1))
    achieved = fl / (per_launch_ms * 1e-3) / 1e12
    return {
        "metric": METRIC, "value": value, "unit": "transforms/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic seeded power-law coefficients, S(l)=(l+1)^-%g" % w["beta"],
        "config": {"workload": args.workload, "kind": "SHMultiply (GLQ)",
                   "lmax_in": [L, L2], "lmax_out": L + L2, "pairs_per_gpu": F,
                   "precision": "fp64",
                   "step": "SHMultiply of every pair: 2 syntheses + 1 analysis "
                           "(counted as 3 transforms)",
                   "l2": "flushed between steps (256 MiB write, outside step events)",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "products_per_s": F * args.steps * world / (total_ms * 1e-3),
        "roofline": {"kernel": names[dom], "bound": "fp64", "achieved": achieved,
                     "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak else None,
                     "peak_source": "measured FP64 FMA probe, this run",
                     "flops_per_launch": fl, "traffic": None},
        "stages": {names[i]: {"ms_per_launch": (ms[i] / cnt[i]) if cnt[i] else None,
                              "launches": cnt[i]} for i in range(6)},
        "multiply_by_one_max_rel_err": ident_err,
        "e2e": {"value": 3.0 * F * e2e_steps * world / (e2e_ms * 1e-3),
                "unit": "transforms/s", "steps": e2e_steps,
                "h2d_bytes_per_step": (c1h.numel() + c2h.numel()) * 8,
                "d2h_bytes_per_step": outs[0][0].numel() * 8,
                "path": "public torch API on pinned host buffers, pipelined on 3 streams"},
        # the pack stage holds 2 launches (one per input field set)
        "gpu_launches": int(sum(cnt)) + int(cnt[0]),
        "clocks": clk.summary(),
    }


def compare_mixed(dev, wname, steps=3):
    """The mixed-precision half of the metric, added to the default line:
    synthesis + analysis of the workload in FP64, with the int8x7 synthesis
    from the recursion (FP64 analysis), and with both directions on the INT8
    tensor cores from the plan's P_lm digit table (int8x7-table); transforms/s
    of each, per-launch Legendre times, the table stream's HBM rate and the
    per-degree error against FP64: of the mixed round trip against the FP64
    round trip, and of the mixed analysis of the FP64 grid against the FP64
    analysis."""
    import ctypes
    import numpy as np
    import torch
    import shtools_b200 as sht
    from shtools_b200 import _lib
    lib = _lib.load()
    w = WORKLOADS[wname]
    L, F, smp = w["lmax"], w["nfield"], w["sampling"]
    c = torch.from_numpy(np.stack([power_law(L, w["seed"] + i, w["beta"])
                                   for i in range(F)])).to(dev)
    st = torch.cuda.current_stream(dev)
    if w["kind"] == "glq":
        zero_t, w_t = sht.PreGLQ(-1.0, 1.0, L + 1, device=dev)
        zero, wts = zero_t.cpu().numpy(), w_t.cpu().numpy()

        def plans(prec):
            ps = sht.get_plan(sht.GRID_GLQ, L, L, 1, 1, 1, 0, zero=zero, device=dev,
                              precision=prec)
            pa = sht.get_plan(sht.GRID_GLQ, L, L, 1, 1, 1, 0, zero=zero, w=wts, device=dev,
                              precision=prec if prec.endswith("-table") else "fp64")
            return ps, pa
    else:
        def plans(prec):
            ps = sht.get_plan(sht.GRID_DH, L, L, 1, 1, smp, 0, device=dev, precision=prec)
            pa = ps if prec.endswith("-table") else \
                sht.get_plan(sht.GRID_DH, L, L, 1, 1, smp, 0, device=dev)
            return ps, pa

    def perdeg(b, r):
        d = (b - r).pow(2).sum(dim=(1, 3)).sqrt()
        n = r.pow(2).sum(dim=(1, 3)).sqrt()
        return float(torch.where(n > 0, d / n, d).max())

    res, ref, g64 = {}, None, None
    for prec in ("fp64", "int8x7", "int8x7-table"):
        t_plan = time.perf_counter()
        ps, pa = plans(prec)
        torch.cuda.synchronize(dev)
        t_plan = time.perf_counter() - t_plan
        g = ps.synthesis(c)
        b = pa.analysis(g)
        torch.cuda.synchronize(dev)
        ms = (ctypes.c_double * 6)()
        cnt = (ctypes.c_int * 6)()
        lib.shtc_timing_enable(1)
        lib.shtc_timing_collect(ms, cnt, 6)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(steps)]
        for i in range(steps):
            evs[i][0].record(st)
            ps.synthesis(c, out=g)
            pa.analysis(g, out=b)
            evs[i][1].record(st)
        torch.cuda.synchronize(dev)
        lib.shtc_timing_enable(0)
        lib.shtc_timing_collect(ms, cnt, 6)
        t = sum(a.elapsed_time(e) for a, e in evs)
        entry = {"transforms_per_s": 2.0 * F * steps / (t * 1e-3),
                 "ms_per_step": t / steps,
                 "legendre_synth_ms": ms[1] / max(1, cnt[1]),
                 "legendre_anal_ms": ms[4] / max(1, cnt[4]),
                 "fft_c2r_ms": ms[2] / max(1, cnt[2]), "fft_r2c_ms": ms[3] / max(1, cnt[3])}
        if prec == "fp64":
            ref = b.clone()
            g64 = g.clone()
        else:
            entry["max_perdeg_rel_err_vs_fp64"] = perdeg(b, ref)
            entry["status"] = sht.mixed_status(dev)
        if prec == "int8x7":
            grid_rec = g.clone()
            entry["directions"] = "synthesis int8x7 (recursion), analysis FP64"
        if prec == "int8x7-table":
            entry["directions"] = "synthesis and analysis int8x7 from the P_lm digit table"
            entry["table_bytes"] = ps.table_bytes
            entry["plan_build_s"] = t_plan
            # the table holds the one-step FP64 recursion's P_lm, the
            # recursion kernel runs a two-step form: close, not identical
            entry["synthesis_max_abs_diff_vs_int8x7_rel"] = float(
                (g - grid_rec).abs().max() / grid_rec.abs().max())
            grid_rec = None
            # the analysis alone: the FP64 grid through the tensor-core analysis
            entry["analysis_only_max_perdeg_rel_err_vs_fp64"] = perdeg(pa.analysis(g64), ref)
            entry["status"] = sht.mixed_status(dev)
            # the table streams once per Legendre launch: HBM rate of that read
            peak = measured_peaks().get("hbm_gbs", 6650.0)
            entry["table_stream"] = {}
            for k in ("synth", "anal"):
                tms = entry["legendre_%s_ms" % k]
                gbs = ps.table_bytes / (tms * 1e-3) / 1e9
                entry["table_stream"][k] = {"achieved_gbs": gbs, "peak_gbs": peak,
                                            "frac": gbs / peak}
        res[prec] = entry
        del g, b
        if prec == "int8x7-table":
            ps.legendre_table(False)          # frees the table's device memory
            if pa is not ps:
                pa.legendre_table(False)
    del g64, ref
    res["workload"] = "%s: %d field(s), lmax %d, %s, S(l)=(l+1)^-%g" % (
        wname, F, L, "GLQ" if w["kind"] == "glq" else "DH sampling %d" % smp, w["beta"])
    res["step"] = "synthesis + analysis, L2 not flushed, %d steps" % steps
    f64, tab = res["fp64"], res["int8x7-table"]
    res["speedup_int8x7_table_vs_fp64"] = {
        "step": f64["ms_per_step"] / tab["ms_per_step"],
        "legendre_synth": f64["legendre_synth_ms"] / tab["legendre_synth_ms"],
        "legendre_anal": f64["legendre_anal_ms"] / tab["legendre_anal_ms"],
        "legendre_both": (f64["legendre_synth_ms"] + f64["legendre_anal_ms"]) /
                         (tab["legendre_synth_ms"] + tab["legendre_anal_ms"])}
    return res


def run_cuda(args, w, rank, world, local_rank):
    import numpy as np
    import torch
    import shtools_b200 as sht
    from shtools_b200 import _lib

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    lib = _lib.load()
    L, F = w["lmax"], w["nfield"]
    cplx = w["kind"] == "dhc"
    cil = np.stack([power_law(L, w["seed"] + i, w["beta"], cplx) for i in range(F)])
    c_host = torch.from_numpy(cil).pin_memory()
    c = c_host.to(dev)
    esize = 16 if cplx else 8
    if cplx:
        s = w["sampling"]
        synth = lambda x: sht.MakeGridDHC(x, sampling=s)
        anal = lambda g: sht.SHExpandDHC(g, sampling=s)
    elif w["kind"] == "glq":
        zero_t, w_t = sht.PreGLQ(-1.0, 1.0, L + 1, device=dev)
        zero, wts = zero_t.cpu().numpy(), w_t.cpu().numpy()
        synth = lambda x: sht.MakeGridGLQ(x, zero=zero, precision=args.precision)
        anal = lambda g: sht.SHExpandGLQ(g, w=wts, zero=zero, precision=args.precision)
    else:
        s = w["sampling"]
        synth = lambda x: sht.MakeGridDH(x, sampling=s, precision=args.precision)
        anal = lambda g: sht.SHExpandDH(g, sampling=s, precision=args.precision)

    def step(x):
        g = synth(x)
        return g, anal(g)

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    st = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        g, back = step(c)
    torch.cuda.synchronize(dev)
    # accuracy of the round trip (size-independent property, per degree)
    bb = back.cpu().numpy()
    num = np.sqrt((np.abs(bb - cil) ** 2).sum(axis=(1, 3)))
    den = np.sqrt((np.abs(cil) ** 2).sum(axis=(1, 3)))
    rt_err = float((num / np.where(den > 0, den, 1)).max())

    peak = fp64_peak(torch, dev)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # ---- device-resident timed region --------------------------------------
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize(dev)
    lib.shtc_timing_enable(1)
    with ClockSampler(local_rank) as clk:
        for i in range(args.steps):
            flush.fill_(float(i))             # L2 flush outside the step events
            evs[i][0].record(st)
            g, back = step(c)
            evs[i][1].record(st)
        torch.cuda.synchronize(dev)
    barrier()
    lib.shtc_timing_enable(0)
    import ctypes
    ms = (ctypes.c_double * 6)()
    cnt = (ctypes.c_int * 6)()
    lib.shtc_timing_collect(ms, cnt, 6)
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = max_over_ranks(sum(step_ms), dev)
    transforms = 2.0 * F * args.steps * world
    value = transforms / (total_ms * 1e-3)

    # ---- end to end through the pyshtools backend call ----------------------
    # the call a pyshtools user makes after select_preferred_backend('cuda'):
    # numpy coefficients in, numpy grid out, numpy grid in, numpy
    # coefficients out, one field per call (shtools_b200.backend); the host
    # copies (numpy buffers staged through pinned memory by
    # shtools_b200.hostio) are inside the timed region
    from shtools_b200 import backend as B
    if cplx:
        s = w["sampling"]
        b_synth = lambda x: B.MakeGridDHC(x, sampling=s)
        b_anal = lambda x: B.SHExpandDHC(x, sampling=s)
    elif w["kind"] == "glq":
        b_synth = lambda x: B.MakeGridGLQ(x, zero=zero)
        b_anal = lambda x: B.SHExpandGLQ(x, w=wts, zero=zero)
    else:
        s = w["sampling"]
        b_synth = lambda x: B.MakeGridDH(x, sampling=s)
        b_anal = lambda x: B.SHExpandDH(x, sampling=s)
    plug_steps = max(2, min(args.steps, 4 if F > 1 else args.steps))
    if not cplx:
        B.set_precision(args.precision)

    def plug_step():
        out = []
        for f in range(F):
            gf = b_synth(cil[f])
            out.append(b_anal(gf))
        return gf, out

    # warm-up: three steps that keep their results as the timed loop does
    # (the previous step's arrays are alive while the next one runs), so the
    # pinned result buffers of both exist before the timed region
    for _ in range(3):
        g_last, b_plug = plug_step()
    barrier()
    torch.cuda.synchronize(dev)
    pa = torch.cuda.Event(enable_timing=True)
    pb = torch.cuda.Event(enable_timing=True)
    pa.record(st)
    for _ in range(plug_steps):
        g_last, b_plug = plug_step()
    pb.record(st)
    torch.cuda.synchronize(dev)
    plug_ms = max_over_ranks(pa.elapsed_time(pb), dev)
    plug_value = 2.0 * F * plug_steps * world / (plug_ms * 1e-3)
    B.set_precision("fp64")
    plug_ok = bool(np.array_equal(b_plug[-1], bb[-1]))
    plug_h2d = F * (cil[0].nbytes + g_last.nbytes)
    plug_d2h = F * (cil[0].nbytes + g_last.nbytes)

    # ---- end-to-end through the public API with host buffers ---------------
    # every step uploads its inputs (cilm and a grid) from pinned host memory,
    # runs synthesis and analysis, and downloads both results; the steps are
    # pipelined over three streams (shtools_b200.pipeline), the synthesis and
    # the analysis of a step as two pipeline steps, so that the synthesis
    # starts once the cilm is on the device and the grid's download overlaps
    # the analysis (measured on one B200 against one pipeline step per step:
    # glq2047 608 against 590, dh719x8 2075 against 2004 transforms/s)
    from shtools_b200.pipeline import pipelined
    g_in = g.cpu().pin_memory()
    outs = [(torch.empty(tuple(g.shape), dtype=g.dtype).pin_memory(),
             torch.empty(tuple(back.shape), dtype=back.dtype).pin_memory())
            for _ in range(2)]
    e2e_steps = max(2, args.steps)
    def e2e_run(n):
        # per step its own function: the synthesis of a cilm, then the
        # analysis of a grid
        ins, outs_n, fns = [], [], []
        for i in range(n):
            ins += [(c_host,), (g_in,)]
            outs_n += [(outs[i % 2][0],), (outs[i % 2][1],)]
            fns += [synth, anal]
        pipelined(fns, ins, outs_n, device=dev)

    e2e_run(2)     # warm-up
    barrier()
    torch.cuda.synchronize(dev)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(st)
    e2e_run(e2e_steps)
    b.record(st)
    torch.cuda.synchronize(dev)
    e2e_ms = max_over_ranks(a.elapsed_time(b), dev)
    e2e_value = 2.0 * F * e2e_steps * world / (e2e_ms * 1e-3)
    e2e_ok = bool(torch.equal(outs[(e2e_steps - 1) % 2][1], back.cpu()) and
                  torch.equal(outs[(e2e_steps - 1) % 2][0], g.cpu()))
    h2d = c_host.numel() * esize + g_in.numel() * esize
    d2h = outs[0][0].numel() * esize + outs[0][1].numel() * esize

    # ---- roofline of the dominant kernel ------------------------------------
    names = ["pack", "legendre_synth", "fft_c2r", "fft_r2c", "legendre_anal",
             "unpack"]
    dom = max((1, 4), key=lambda i: ms[i])
    per_launch_ms = ms[dom] / max(1, cnt[dom])
    # complex fields: two coefficient sets (orders +m, -m) per field
    fl = legendre_flops(w, F * (2 if cplx else 1))
    achieved = fl / (per_launch_ms * 1e-3) / 1e12
    traffic = load_traffic("%s_%s" % (names[dom], args.workload) +
                           ("" if args.precision == "fp64" else "_" + args.precision))
    roof = {"kernel": names[dom], "bound": "fp64", "achieved": achieved,
            "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak if peak else None,
            "peak_source": "measured FP64 FMA probe, this run "
                           "(MEASURED_PEAKS.json has no FP64 entry)",
            "flops_per_launch": fl, "traffic": traffic}
    if args.precision.endswith("-table") and not cplx:
        # the table-driven tensor-core kernels stream the plan's P_lm digit
        # table once per launch: HBM-bound on that read
        sht_plans = [p for k, p in sht.transforms._plans.items()
                     if k[-1] == args.precision and k[1] == L]
        tb = max(p.table_bytes for p in sht_plans) if sht_plans else 0
        gbs = tb / (per_launch_ms * 1e-3) / 1e9
        hbm = measured_peaks().get("hbm_gbs", 6650.0)
        roof = {"kernel": names[dom], "bound": "hbm", "achieved": gbs, "peak": hbm,
                "unit": "GB/s", "frac": gbs / hbm,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs",
                "bytes_per_launch": tb, "traffic": traffic,
                "bytes_note": "the P_lm digit table, read once per launch"}
    stage = {names[i]: {"ms_per_launch": (ms[i] / cnt[i]) if cnt[i] else None,
                        "launches": cnt[i],
                        "share": ms[i] / max(1e-9, sum(ms))} for i in range(6)}
    res = {
        "metric": METRIC,
        "value": value,
        "unit": "transforms/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c128" if cplx else "f64",
        "data": "synthetic seeded power-law coefficients, S(l)=(l+1)^-%g" % w["beta"],
        "config": bench_config(args, w, world),
        "l2": "flushed between steps (256 MiB write, outside step events)",
        "roofline": roof,
        "stages": stage,
        "roundtrip_max_perdeg_err": rt_err,
        "e2e": {"value": plug_value, "unit": "transforms/s",
                "h2d_bytes_per_step": plug_h2d, "d2h_bytes_per_step": plug_d2h,
                "steps": plug_steps, "result_matches_device_run": plug_ok,
                "path": "pyshtools backend call (shtools_b200.backend, numpy in and "
                        "out, one field per call): per field H2D cilm, synthesis, D2H "
                        "grid, H2D grid, analysis, D2H cilm; numpy buffers staged "
                        "through pinned chunks (shtools_b200.hostio)"},
        "e2e_pipelined": {"value": e2e_value, "unit": "transforms/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": e2e_steps, "result_matches_device_run": e2e_ok,
                "path": "public torch API on pinned host buffers: per step H2D cilm "
                        "+ H2D grid, synthesis + analysis, D2H grid + D2H cilm; "
                        "steps pipelined on 3 streams (shtools_b200.pipeline), the "
                        "synthesis and the analysis of a step as two pipeline steps"},
        "gpu_launches": int(sum(cnt)),
        "clocks": clk.summary(),
    }
    if args.workload == "glq2047" and world == 1 and not args.no_2799:
        res["mixed_glq2047"] = compare_mixed(dev, "glq2047", steps=5)
        res["lmax2799"] = compare_mixed(dev, "dh2799x16")
    return res


def main():
    args = parse()
    w = WORKLOADS[args.workload]
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        # the reference arm runs on rank 0's host cores only
        if rank != 0:
            return 0
        one_step, sample, threads = cpu_sample(w, args.cpu_seconds / 3)
        for _ in range(args.warmup):
            one_step()
        vals, dts = [], []
        for _ in range(args.steps):
            v, dt = one_step()
            vals.append(v)
            dts.append(dt)
        value = args.steps / sum(1.0 / v for v in vals)   # harmonic mean
        res = {"metric": METRIC, "impl": "reference", "value": value,
               "unit": "transforms/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": 1e3 * sum(dts) / len(dts),
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
               "dtype": "f64", "data": "synthetic seeded power-law coefficients",
               "config": bench_config(args, w, world),
               "cpu_baseline": {"value": value, "unit": "transforms/s",
                                "cores": threads, "kind": "port",
                                "sample": sample},
               "e2e": {"value": value, "unit": "transforms/s",
                       "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(res))
        return 0
    if not args.no_autotune:
        # tile shapes from the project autotuner, tuned when a plan is created
        # (before the warm-up, outside the timed region)
        os.environ.setdefault("SHTC_AUTOTUNE", "1")
    if world > 1:
        import torch
        import datetime
        torch.distributed.init_process_group(
            "nccl", timeout=datetime.timedelta(seconds=120))
    if w["kind"] == "glq_batch":
        res = run_cuda_batch(args, w, rank, world, local_rank)
    elif w["kind"] == "dh_grad":
        res = run_cuda_grad(args, w, rank, world, local_rank)
    elif w["kind"] in ("gradient", "gravity"):
        res = run_cuda_gradient(args, w, rank, world, local_rank)
    elif w["kind"] == "multiply":
        res = run_cuda_multiply(args, w, rank, world, local_rank)
    else:
        res = run_cuda(args, w, rank, world, local_rank)
    if rank == 0 and world == 1 and not args.no_cpu_baseline and \
            w["kind"] not in ("dhc", "gradient", "gravity", "multiply"):
        one_step, sample, threads = cpu_sample(w, args.cpu_seconds / 2)
        v, dt = one_step()
        res["cpu_baseline"] = {"value": v, "unit": "transforms/s",
                               "cores": threads, "kind": "port",
                               "sample": sample + " (%.1f s)" % dt}
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        if w["kind"] == "glq_batch":
            res["tile_shapes"] = "fixed batched-kernel shapes"
        else:
            res["tile_shapes"] = (
                "default" if args.no_autotune else "autotuned per plan (shtools_b200.autotune)")
        print(json.dumps(res))
    return 0


if __name__ == "__main__":
    sys.exit(main())
