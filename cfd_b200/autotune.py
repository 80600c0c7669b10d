"""Autotuner for the device plan's launch shapes and smoother schedule.

The knobs are those of `Tuning` (include/cfdb.h, cfdb_tuning):

* target_tiles - level-0 Krylov tiles (0: 256 rows each; else about this many CTAs),
* wide_row     - average row length above which a level switches from SELL-32 rows to
                 CSR lane groups,
* lanes_div    - lanes per CSR row = average row length / lanes_div,
* fuse_first   - first two Jacobi sweeps of the pre-smoothing fused into one kernel,
* sell_rows    - rows per CTA of SELL operators (one row per thread per pass),
* krylov_pair  - level-0 Krylov SpMV kernels take two rows per thread per pass, or one,
* krylov_stage - the level-0 Krylov SpMV streams the operator through shared memory by bulk
                 copies in this many buffers (0: the threads load it, as krylov_pair says),
* tail_rows    - coarse levels of at most this many rows run in one persistent kernel,
* vcycle_pair  - V-cycle kernels of SELL operators take two rows per thread per pass, or one,
* tail_cluster - that kernel as one thread-block cluster of this many CTAs (0: a cooperative
                 grid), searched jointly with tail_rows (the candidates keep the grid form),
* mixed_sweeps, mixed_weight - the smoother schedule of the mixed-precision V-cycle (Jacobi
                 sweeps per level before and after the coarse correction, and the weight); the
                 FP64 path keeps the hierarchy's (the reference's 2 sweeps, weight 0.7).

The launch knobs are searched by coordinate descent from the defaults: each knob (or a tuple
of knobs searched jointly) in turn is swept over its candidate values with the others fixed, the best value kept, and the pass
repeated until no knob changes (at most `passes` passes). Their objective is the device time of
a fixed number of CG iterations (tolerance 0, so every system runs exactly `iterations`
iterations) through the captured graphs of the real solve path, median of `reps` runs. The
smoother schedule changes the iteration count, so its objective is the device time of whole
solves to the caller's tolerance (`tune_smoother`); the knobs that interact with it are then
searched once more under the chosen schedule (`retune_knobs`). Results of `tune` are cached in a
JSON file keyed by a workload signature.
"""
from __future__ import annotations

import dataclasses
import json
import os
import statistics
from typing import Callable

from . import Tuning

CANDIDATES = {
    "target_tiles": [0, 148 * 8, 148 * 16],
    "wide_row": [24, 32, 48, 64],
    "lanes_div": [8, 12, 16, 32],
    "fuse_first": [0, 1],
    "sell_rows": [256, 512, 1024],
    "krylov_pair": [0, 1],
    "krylov_stage": [0, 2, 3, 4],
    "vcycle_pair": [0, 1],
    # the single-cluster tail (tail_cluster > 0) is not a candidate: on tet 95^3 x 6 it took
    # 299 us (16 CTAs) to 1,103 us (4 CTAs) per V-cycle where the separate kernels take ~50 us
    ("tail_rows", "tail_cluster"): [(0, 0), (1024, 0), (8192, 0), (65536, 0), (131072, 0)],
}

# knobs whose best value depends on the smoother schedule: with one sweep per level the first
# sweeps are never fused, so the persistent tail (which needs the unfused schedule) and the
# shapes of the kernels it replaces are searched again once the schedule is chosen
SCHEDULE_KNOBS = (("tail_rows", "tail_cluster"), "sell_rows", "target_tiles", "vcycle_pair")


def _key(t: Tuning) -> tuple:
    return tuple(dataclasses.astuple(t))


def coordinate_search(evaluate: Callable[[Tuning], float], start: Tuning | None = None,
                      candidates: dict | None = None, passes: int = 2):
    """Minimises evaluate(tuning) (milliseconds) by coordinate descent. Returns
    (best tuning, best value, trace of (tuning dict, value))."""
    cand = candidates or CANDIDATES
    best = dataclasses.replace(start) if start is not None else Tuning()
    seen = {}
    trace = []

    def ev(t):
        k = _key(t)
        if k not in seen:
            seen[k] = float(evaluate(t))
            trace.append((dataclasses.asdict(t), seen[k]))
        return seen[k]

    best_v = ev(best)
    for _ in range(max(passes, 1)):
        changed = False
        for knob, values in cand.items():
            names = knob if isinstance(knob, tuple) else (knob,)
            for v in values:
                vals = v if isinstance(knob, tuple) else (v,)
                if tuple(getattr(best, k) for k in names) == tuple(vals):
                    continue
                t = dataclasses.replace(best, **dict(zip(names, vals)))
                val = ev(t)
                if val < best_v:
                    best, best_v, changed = t, val, True
        if not changed:
            break
    return best, best_v, trace


def solve_timer(target, run_iterations: Callable[[int], None], stream_handle: int,
                iterations: int = 6, reps: int = 3):
    """An objective for coordinate_search: installs the tuning on `target` (a DeviceSolver or
    Batch), then times run_iterations(iterations) with CUDA events on the target's stream."""
    import torch

    def evaluate(t: Tuning) -> float:
        target.set_tuning(t)
        stream = torch.cuda.ExternalStream(stream_handle)
        run_iterations(iterations)  # warm: graph capture for the new plan
        times = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            run_iterations(iterations)
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        return statistics.median(times)

    return evaluate


def tune(target, run_iterations, stream_handle, signature: str, cache_path: str | None = None,
         iterations: int = 6, reps: int = 3, passes: int = 2):
    """Tunes `target` for the workload named by `signature`, reusing a cached result when the
    cache file holds one. Installs and returns the best tuning with its record."""
    cache = {}
    if cache_path and os.path.exists(cache_path):
        try:
            with open(cache_path) as f:
                cache = json.load(f)
        except (OSError, ValueError):
            cache = {}
    if signature in cache:
        rec = cache[signature]
        best = Tuning(**rec["tuning"])
        target.set_tuning(best)
        return best, dict(rec, cached=True)
    evaluate = solve_timer(target, run_iterations, stream_handle, iterations, reps)
    default_ms = evaluate(Tuning())
    best, best_ms, trace = coordinate_search(evaluate, Tuning(), passes=passes)
    target.set_tuning(best)
    rec = {"tuning": dataclasses.asdict(best), "ms": best_ms, "default_ms": default_ms,
           "iterations": iterations, "evaluations": len(trace), "trace": trace}
    if cache_path:
        cache[signature] = rec
        with open(cache_path, "w") as f:
            json.dump(cache, f, indent=1)
    return best, dict(rec, cached=False)


# (sweeps, weight) candidates of the mixed-precision smoother schedule; (2, 0.7) is the
# reference's AmgView default
SMOOTHER_CANDIDATES = [(2, 0.7), (2, 0.85), (1, 0.85), (1, 0.7), (3, 0.85)]


def tune_smoother(target, solve: Callable[[], int], stream_handle: int, base: Tuning | None = None,
                  candidates=None, reps: int = 3):
    """Picks the mixed-precision smoother schedule with the shortest device time of a whole
    solve to the caller's tolerance. solve() runs one solve on the target's stream and returns
    its iteration count. Installs the best schedule on top of `base` and returns
    (tuning, record)."""
    import torch
    base = base or Tuning()
    trace = []
    best, best_ms = None, float("inf")
    for sweeps, weight in candidates or SMOOTHER_CANDIDATES:
        t = dataclasses.replace(base, mixed_sweeps=sweeps, mixed_weight=weight)
        target.set_tuning(t)
        stream = torch.cuda.ExternalStream(stream_handle)
        solve()  # warm: graph capture for the new plan
        times, iters = [], 0
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            iters = solve()
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        ms = statistics.median(times)
        trace.append({"sweeps": sweeps, "weight": weight, "ms": ms, "iterations": iters})
        if ms < best_ms:
            best, best_ms = t, ms
    target.set_tuning(best)
    return best, {"ms": best_ms, "trace": trace}


def retune_knobs(evaluate: Callable[[Tuning], float], base: Tuning, knobs=SCHEDULE_KNOBS):
    """One coordinate-descent pass over `knobs` from `base` (a tuning that already carries the
    chosen smoother schedule); evaluate is an objective such as solve_timer's, which also
    installs the tuning it times. Returns (tuning, record); the caller installs the tuning."""
    cand = {k: CANDIDATES[k] for k in knobs}
    best, best_ms, trace = coordinate_search(evaluate, base, candidates=cand, passes=1)
    return best, {"ms": best_ms, "start_ms": trace[0][1] if trace else None,
                  "evaluations": len(trace), "trace": trace}
