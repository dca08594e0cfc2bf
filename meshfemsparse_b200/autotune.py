"""Autotuner for the factorization's free parameters on one sparsity pattern.

Two choices have no single best value: the small/large front cutoff (fronts up
to it are factored whole in one CTA's shared memory, larger ones by 128-column
panels and tensor-core tiles) and, for an FP32 factor under FP64 refinement,
the tensor-core mode (5, single FP16 operands: a faster factor, more refinement
iterations; 6, split hi/lo FP16 operands: a slower, FP32-accurate factor, fewer
iterations, which wins as the right-hand sides per solve grow). `tune` times every
candidate on the caller's own matrix and
right-hand sides (device times of the library's CUDA events: factorization plus
refined solve), keeps the fastest, and caches the choice on disk keyed by the
pattern, the pins, the precision and the GPU name, so a pattern that is
factored many times (a Newton sequence, a batch of meshes) is tuned once.
Each candidate repeats the symbolic analysis, so tuning costs a few analyses.
"""
from __future__ import annotations

import hashlib
import json
import os
from pathlib import Path
from typing import Callable

import numpy as np

from .factorizer import B200Factorizer

CUTOFFS_FP32 = (96, 128, 160, 192, 224)
CUTOFFS_FP64 = (64, 96, 128, 160)


def default_cache() -> Path:
    env = os.environ.get("MFS_AUTOTUNE_CACHE")
    if env:
        return Path(env)
    return Path.home() / ".cache" / "meshfemsparse_b200" / "autotune.json"


def pattern_key(H, pins, single: bool, refine: bool, device_name: str) -> str:
    h = hashlib.sha1()
    for a in (np.asarray(H.Ap, dtype=np.int64), np.asarray(H.Ai, dtype=np.int64),
              np.sort(np.asarray(pins, dtype=np.int64))):
        h.update(a.tobytes())
    h.update(f"{H.bs}|{int(single)}|{int(refine)}|{device_name}".encode())
    return h.hexdigest()


def _device_name(device: int) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:
        return f"device{device}"


def measure_step(H, pins, tets, Ke, rhs, single: bool, refine: bool, device: int, small_front_max: int,
                 tensor_cores: int, repeats: int, factor_group: int = 0, solve_subtrees: int = 0) -> float:
    """Best device time (ms) of assemble -> factorize -> solve with these options."""
    f = B200Factorizer(single, refine=refine, device=device, small_front_max=small_front_max,
                       tensor_cores=tensor_cores, factor_group=factor_group, solve_subtrees=solve_subtrees)
    f.factorizeSymbolic(H, pins)
    f.setElements(tets)
    best = float("inf")
    for _ in range(repeats + 1):                  # the first run also pays one-time set-up
        f.assemble(Ke, return_values=False)
        f.factorizeAssembled()
        f.solveMultiRHS(rhs)
        st = f.stats()
        best = min(best, st["factor_ms"] + st["solve_ms"])
    return best


def tune(H, pins, tets, Ke, rhs, single: bool = True, refine: bool = True, device: int = 0,
         cutoffs=None, tensor_modes=None, repeats: int = 2, cache: Path | str | None = None,
         measure: Callable | None = None, factor_groups=(0,), solve_subtrees=(0,)) -> dict:
    """Pick small_front_max (and tensor_cores for FP32 + refinement) for this pattern, and,
    when more than one value is given, the schedule shapes: factor_group (128-column blocks
    per group of the blocked large-front factorization; 0 = its default) and solve_subtrees
    (the subtree count the solve cut aims for; 0 = its default).

    Returns {"small_front_max", "tensor_cores", "factor_group", "solve_subtrees", "ms",
    "candidates", "cached"}; pass the first four to B200Factorizer.
    `measure(small_front_max, tensor_cores) -> ms` (or, when groups or subtree counts are
    tuned, `measure(small_front_max, tensor_cores, factor_group, solve_subtrees)`)
    replaces the GPU timing (tests)."""
    cache = Path(cache) if cache is not None else default_cache()
    shapes = len(factor_groups) > 1 or len(solve_subtrees) > 1
    key = pattern_key(H, pins, single, refine, _device_name(device))
    if shapes:          # a choice among schedule shapes is another entry
        key += f"|groups={tuple(int(g) for g in factor_groups)}|subtrees={tuple(int(s) for s in solve_subtrees)}"
    store = {}
    if cache.exists():
        try:
            store = json.loads(cache.read_text())
        except (OSError, ValueError):
            store = {}
    if key in store:
        return {"factor_group": 0, "solve_subtrees": 0, **store[key], "cached": True}
    if cutoffs is None:
        cutoffs = CUTOFFS_FP32 if single else CUTOFFS_FP64
    if tensor_modes is None:
        tensor_modes = (5, 6) if (single and refine) else (0,)
    if measure is None:
        def measure(cut, tc, group=0, subtrees=0):
            return measure_step(H, pins, tets, Ke, rhs, single, refine, device, cut, tc, repeats, group, subtrees)
    cands = []
    for cut in cutoffs:
        for tc in tensor_modes:
            for group in factor_groups:
                for sub in solve_subtrees:
                    ms = measure(cut, tc, group, sub) if shapes else measure(cut, tc)
                    cands.append({"small_front_max": int(cut), "tensor_cores": int(tc), "factor_group": int(group),
                                  "solve_subtrees": int(sub), "ms": float(ms)})
    best = min(cands, key=lambda c: (c["ms"], c["small_front_max"], c["tensor_cores"], c["factor_group"],
                                     c["solve_subtrees"]))
    choice = {"small_front_max": best["small_front_max"], "tensor_cores": best["tensor_cores"],
              "factor_group": best["factor_group"], "solve_subtrees": best["solve_subtrees"], "ms": best["ms"],
              "candidates": cands}
    store[key] = choice
    cache.parent.mkdir(parents=True, exist_ok=True)
    tmp = cache.with_suffix(".tmp")
    tmp.write_text(json.dumps(store, indent=1))
    os.replace(tmp, cache)
    return {**choice, "cached": False}


def choose_form(H, pins, tets, Ke, rhs, device: int = 0, cache: Path | str | None = None,
                measure: Callable | None = None, **kw) -> dict:
    """Tune both forms and keep the faster one: FP32 factor + FP64 refinement wins
    on large fronts (tensor-core Schur updates), plain FP64 can win on batches of
    small fronts, where the factor is cheap and the refinement's solves dominate.
    Returns the B200Factorizer arguments (singlePrecision, refine, small_front_max,
    tensor_cores) and the measured ms. `measure(single, cut, tc) -> ms` replaces the
    GPU timing (tests)."""
    res = {}
    for single in (True, False):
        m = None if measure is None else (lambda cut, tc, s=single: measure(s, cut, tc))
        res[single] = tune(H, pins, tets, Ke, rhs, single=single, refine=single, device=device, cache=cache,
                           measure=m, **kw)
    single = res[True]["ms"] <= res[False]["ms"]
    r = res[single]
    return {"singlePrecision": single, "refine": single, "small_front_max": r["small_front_max"],
            "tensor_cores": r["tensor_cores"], "ms": r["ms"],
            "fp32_refine_ms": res[True]["ms"], "fp64_ms": res[False]["ms"]}
