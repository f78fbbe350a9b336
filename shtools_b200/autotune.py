"""Autotuner of the Legendre-kernel tile shapes.

For a plan, times the single-field synthesis kernel for each choice of ring
pairs per thread (1, 2, 4, 8) and the analysis kernel with its unpack for
each (pairs per thread, warps per CTA) pair, on random inputs of the plan's
real size, with the library's per-stage CUDA-event timing, and keeps the
fastest.  Results
are cached in a JSON file keyed by GPU model and plan geometry:
``$SHTC_TUNE_CACHE`` or ``~/.cache/shtools_b200/tune.json``.

    from shtools_b200 import autotune, get_plan, GRID_GLQ
    plan = get_plan(GRID_GLQ, 2047, 2047, 1, 1)
    autotune.tune_plan(plan)           # applies and returns the shapes

``get_plan(..., tune=True)`` or ``SHTC_AUTOTUNE=1`` tunes new plans
automatically.
"""
import ctypes
import json
import os
import threading

import torch

from . import _lib

STAGE_SYNTH = 1
STAGE_ANAL = 4
STAGE_UNPACK = 5
_lock = threading.Lock()


def cache_path():
    return os.environ.get("SHTC_TUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "shtools_b200", "tune.json")


def _load_cache():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except Exception:
        return {}


def _save_cache(d):
    p = cache_path()
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        tmp = p + ".tmp"
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, p)
    except OSError:
        pass


def plan_key(plan):
    i = plan.info
    name = torch.cuda.get_device_name(plan.device)
    return "%s|kind%d|L%d|lc%d|s%d%s" % (name, i["kind"], i["lmax"], i["lmax_comp"],
                                         i["sampling"],
                                         "|complex" if getattr(plan, "cplx", False) else "")


def _time_stage(plan, fn, stage, reps):
    """Mean time per call (ms) of one library stage, or of the sum of several
    (a tuple of stage ids)."""
    lib = plan.lib
    fn()
    torch.cuda.synchronize(plan.device)
    lib.shtc_timing_enable(1)
    for _ in range(reps):
        fn()
    torch.cuda.synchronize(plan.device)
    lib.shtc_timing_enable(0)
    ms = (ctypes.c_double * 6)()
    cnt = (ctypes.c_int * 6)()
    _lib.check(lib.shtc_timing_collect(ms, cnt, 6))
    stages = stage if isinstance(stage, tuple) else (stage,)
    return sum(ms[s] / max(1, cnt[s]) for s in stages)


def candidates(npair):
    synth = [t for t in (1, 2, 4, 8) if t * 128 <= max(256, 2 * npair)]
    # one-warp CTAs skip the cross-warp reduction but make more ring-pair
    # tiles, whose partial sums the unpack adds (timed with the analysis)
    anal = [(t, w) for t in (1, 2, 4, 8) for w in (1, 2, 4, 8)
            if t * w * 32 <= max(128, 2 * npair)]
    return synth, anal


def set_shape(plan, synth_T=0, anal_T=0, anal_W=0):
    _lib.check(plan.lib.shtc_plan_set_tuning(plan.handle, int(synth_T),
                                             int(anal_T), int(anal_W)),
               "shtc_plan_set_tuning")
    plan.shape = (int(synth_T), int(anal_T), int(anal_W))


def tune_plan(plan, reps=3, use_cache=True, verbose=False):
    """Pick and apply the fastest tile shapes for ``plan``; returns
    {"synth_T": .., "anal_T": .., "anal_W": .., "times_ms": {...}}."""
    key = plan_key(plan)
    with _lock:
        if use_cache:
            hit = _load_cache().get(key)
            if hit:
                set_shape(plan, hit["synth_T"], hit["anal_T"], hit["anal_W"])
                return hit
        i = plan.info
        lc = i["lmax_comp"]
        g = torch.Generator(device=plan.device).manual_seed(0)
        # complex plans are timed on complex fields (two coefficient sets each)
        dt = torch.complex128 if getattr(plan, "cplx", False) else torch.float64
        c = torch.randn((1, 2, lc + 1, lc + 1), generator=g, dtype=dt,
                        device=plan.device)
        grid = torch.randn((1, i["nlat"], i["nlon"]), generator=g, dtype=dt,
                           device=plan.device)
        synth = plan.synthesis_c if dt == torch.complex128 else plan.synthesis
        anal = plan.analysis_c if dt == torch.complex128 else plan.analysis
        s_c, a_c = candidates(i["npair"])
        times = {}
        best_s, best_st = None, float("inf")
        for t in s_c:
            set_shape(plan, t, 0, 0)
            ms = _time_stage(plan, lambda: synth(c), STAGE_SYNTH, reps)
            times["synth_T%d" % t] = ms
            if ms < best_st:
                best_s, best_st = t, ms
        best_a, best_at = None, float("inf")
        for t, w in a_c:
            set_shape(plan, 0, t, w)
            ms = _time_stage(plan, lambda: anal(grid), (STAGE_ANAL, STAGE_UNPACK), reps)
            times["anal_T%d_W%d" % (t, w)] = ms
            if ms < best_at:
                best_a, best_at = (t, w), ms
        res = {"synth_T": best_s, "anal_T": best_a[0], "anal_W": best_a[1],
               "times_ms": times}
        set_shape(plan, res["synth_T"], res["anal_T"], res["anal_W"])
        if verbose:
            print(key, res)
        if use_cache:
            d = _load_cache()
            d[key] = res
            _save_cache(d)
        return res
