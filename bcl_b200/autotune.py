"""Autotuner for the SpGEMM and SpMM launches.

SpGEMM: the light-row bound of the row classification (a context knob, so
each candidate runs the whole product), then the numeric pass's plan
parameters (work items a warp takes from the device queue at a time, blocks
per SM, the B-segment length from which a segment is walked lane-parallel),
grid-searched on one plan.  SpMM: rows per warp item, the long-row
threshold, the long-row kernel's block count, the schedule of the
long-row and short-row kernels and the order of column panels, by coordinate descent (one knob at a time, the
others at their best so far).  The learned product: the outputs aimed at per
heavy item.

Every candidate is timed with CUDA events on the actual product, best of a
few runs.  Results are cached in a JSON file keyed by a signature of the
product (value type, tile shapes, grids, nonzeros rounded to powers of two),
so a later product of the same kind reuses the choice without tuning.  No
knob changes a result: every choice gives the same bits.
"""
from __future__ import annotations

import itertools
import json
import math
import os
from typing import Dict, Optional

import torch

SPGEMM_LIGHT_UB = (128, 256, 512)
CANDIDATES = {
    "grab": (1, 2, 4, 8),
    "blocks_per_sm": (3, 4),
    "long_seg": (32, 48, 64, 1 << 30),
}
DEFAULT = (1, 4, 32)
SPMM_CANDIDATES = {
    "spmm_rows": (0, 1, 2, 4),
    "spmm_long_row": (0, 512, 1024, 2048),
    "spmm_long_blocks": (0, 37, 74, 111),
    "spmm_schedule": (0, 1),
    "spmm_panel_major": (0, 1),
}
LEARN_TARGETS = (256, 320, 384)


def cache_path() -> str:
    d = os.environ.get("BCLX_CACHE", os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                                  ".cache"))
    os.makedirs(d, exist_ok=True)
    return os.path.join(d, "autotune.json")


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(tab):
    tmp = cache_path() + ".tmp"
    with open(tmp, "w") as f:
        json.dump(tab, f, indent=1, sort_keys=True)
    os.replace(tmp, cache_path())


def _p2(x):
    return 0 if x <= 0 else int(round(math.log2(x)))


def signature(a, b, kind: str = "spgemm") -> str:
    """Product signature from what is known before any launch."""
    if kind == "spmm":
        return (f"spmm|{b.torch_dtype}|t{a.tm}x{a.tn}x{b.tn}|g{a.gm}x{a.gn}x{b.gn}|m{_p2(a.m)}|n{_p2(b.n)}"
                f"|nnz{_p2(a.nnz())}")
    return (f"{kind}|{a.dtype.str}|t{a.tm}x{a.tn}x{b.tn}|g{a.gm}x{a.gn}x{b.gn}|a{_p2(a.nnz())}"
            f"|b{_p2(b.nnz())}")


def lookup(a, b, kind: str = "spgemm") -> Optional[Dict[str, int]]:
    hit = _load().get(signature(a, b, kind))
    return dict(hit["params"]) if hit else None


def _time(fn, reps):
    stream = torch.cuda.current_stream()
    fn()  # warm
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def tune(a, b, reps: int = 2, candidates=None, light_ubs=SPGEMM_LIGHT_UB, verbose: bool = False):
    """Tune C = A*B; store and return (params dict, ms, [(ms, params), ...])."""
    from .containers import context, spgemm, spgemm_numeric, spgemm_symbolic
    ctx = context(a.device)
    cands = candidates or CANDIDATES
    results = []
    # 1. the light-row bound (classification changes: whole products)
    best_lu, best_lu_ms = None, float("inf")
    for lu in light_ubs:
        with ctx.tuned(light_ub=lu):
            ms = _time(lambda: spgemm(a, b), reps)
        if verbose:
            print(f"  light_ub {lu}: {ms:.3f} ms")
        if ms < best_lu_ms:
            best_lu, best_lu_ms = lu, ms
    # 2. the numeric plan parameters on one plan
    with ctx.tuned(light_ub=best_lu):
        plan, out, trp, toff, nnz = spgemm_symbolic(a, b)
    ci = torch.empty(max(nnz, 1), dtype=torch.int32, device="cuda")
    v = torch.empty(max(nnz, 1), dtype=a.vals.dtype, device="cuda")
    out.col_ind, out.vals = ci.data_ptr(), v.data_ptr()
    for params in itertools.product(cands["grab"], cands["blocks_per_sm"], cands["long_seg"]):
        plan.tune(*params)
        ms = _time(lambda: spgemm_numeric(plan, a, b, out), reps)
        results.append((ms, dict(light_ub=best_lu, grab=params[0], blocks_per_sm=params[1], long_seg=params[2])))
        if verbose:
            print(f"  {params}: {ms:.3f} ms")
    plan.close()
    results.sort(key=lambda r: r[0])
    best_ms, best = results[0]
    tab = _load()
    tab[signature(a, b)] = {"params": best, "numeric_ms": best_ms, "light_ub_product_ms": best_lu_ms}
    _store(tab)
    return best, best_ms, results


def tune_spmm(a, b, c, reps: int = 3, candidates=None, verbose: bool = False):
    """Tune C += A*B (SpMM knobs, coordinate descent); store and return
    (params dict, ms).  C is overwritten by the timing runs."""
    from .containers import context, spmm
    ctx = context(a.device)
    cands = candidates or SPMM_CANDIDATES
    best = {k: ctx.get_tuning(k) for k in cands}
    with ctx.tuned(**best):
        best_ms = _time(lambda: spmm(a, b, c), reps)
    for k, values in cands.items():
        for val in values:
            if val == best[k]:
                continue
            trial = dict(best, **{k: val})
            try:
                with ctx.tuned(**trial):
                    ms = _time(lambda: spmm(a, b, c), reps)
            except Exception:  # a value out of range for this device
                continue
            if verbose:
                print(f"  {trial}: {ms:.3f} ms")
            if ms < best_ms:
                best, best_ms = trial, ms
    tab = _load()
    tab[signature(a, b, "spmm")] = {"params": best, "ms": best_ms}
    _store(tab)
    return best, best_ms


def tune_learned(a, b, reps: int = 2, targets=LEARN_TARGETS, predictor="default", verbose: bool = False):
    """Tune the learned product's outputs per heavy item; store and return
    (params dict, ms)."""
    from .containers import context, spgemm_learned
    ctx = context(a.device)
    best, best_ms = None, float("inf")
    for t in targets:
        with ctx.tuned(learn_target=t):
            ms = _time(lambda: spgemm_learned(a, b, predictor=predictor), reps)
        if verbose:
            print(f"  learn_target {t}: {ms:.3f} ms")
        if ms < best_ms:
            best, best_ms = {"learn_target": t}, ms
    tab = _load()
    tab[signature(a, b, "learned")] = {"params": best, "ms": best_ms}
    _store(tab)
    return best, best_ms
