"""Autotuner for the SpGEMM numeric pass.

Grid search over the numeric parameters of a plan (work items a warp takes
from the device queue at a time, blocks per SM, and the B-segment length from
which a segment is walked lane-parallel), timed with CUDA events on the
actual product, best of a few runs each.  Results are cached in a JSON file
keyed by a signature of the product (value type, tile shape, grid, and the
plan's row statistics rounded to powers of two), so a later product of the
same kind reuses the choice without tuning.
"""
from __future__ import annotations

import itertools
import json
import math
import os
from typing import Optional, Tuple

import torch

CANDIDATES = {
    "grab": (1, 2, 4, 8),
    "blocks_per_sm": (3, 4),
    "long_seg": (32, 48, 64, 1 << 30),
}
DEFAULT = (1, 4, 32)


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


def signature(a, b, plan) -> str:
    st = plan.stats()
    def p2(x):
        return 0 if x <= 0 else int(round(math.log2(x)))
    return (f"{a.dtype.str}|t{a.tm}x{a.tn}x{b.tn}|g{a.gm}x{a.gn}x{b.gn}|p{p2(st['products'])}"
            f"|l{p2(st['light_rows'])}|h{p2(st['heavy_rows'])}|i{p2(st['heavy_items'])}")


def lookup(a, b, plan) -> Optional[Tuple[int, int, int]]:
    hit = _load().get(signature(a, b, plan))
    return tuple(hit["params"]) if hit else None


def tune(a, b, reps: int = 2, candidates=None, verbose: bool = False):
    """Time every candidate on C = A*B; store and return (params, ms, table)."""
    from .containers import spgemm_numeric, spgemm_symbolic
    cands = candidates or CANDIDATES
    plan, out, trp, toff, nnz = spgemm_symbolic(a, b)
    ci = torch.empty(max(nnz, 1), dtype=torch.int32, device="cuda")
    v = torch.empty(max(nnz, 1), dtype=a.vals.dtype, device="cuda")
    out.col_ind, out.vals = ci.data_ptr(), v.data_ptr()
    stream = torch.cuda.current_stream()
    results = []
    for params in itertools.product(cands["grab"], cands["blocks_per_sm"], cands["long_seg"]):
        plan.tune(*params)
        spgemm_numeric(plan, a, b, out)  # warm
        best = float("inf")
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            spgemm_numeric(plan, a, b, out)
            e1.record(stream)
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        results.append((best, params))
        if verbose:
            print(f"  {params}: {best:.3f} ms")
    results.sort()
    best_ms, best_params = results[0]
    tab = _load()
    tab[signature(a, b, plan)] = {"params": list(best_params), "ms": best_ms,
                                  "default_ms": next((t for t, p in results if p == DEFAULT), None)}
    _store(tab)
    plan.close()
    return best_params, best_ms, results
