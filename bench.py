#!/usr/bin/env python
"""Benchmark of the BCL sparse tile multiply on B200.

One JSON line on rank 0.  The headline workload is the plain SpGEMM
configuration C = A*A for an R-MAT scale-16 matrix (65536^2, edge factor 16,
a=0.57, b=c=0.19, d=0.05, duplicates merged, self-loops kept, FP32 values
U(-1,1)) on an 8x8 tile grid, run as BCL::gemm(SPMatrix, SPMatrix,
SPMatrix&) does: every C tile sums its G stage products in rotated order.
A "step" is one whole product (symbolic + numeric + output allocation) over
the resident tiles.  Metric: GFLOP/s = 2 x intermediate products / time,
with the HBM GB/s of the algorithmic bytes beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl reference]

Multi-GPU (torchrun): each rank multiplies its own independent matrix of the
same configuration (seed + rank); no data-path collective; the time is the
max over ranks and ``value`` is the job total ("weak" scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SpGEMM/SpMM GFLOP/s + HBM GB/s on 1 B200: batched+learned vs plain, vs CPU"
L2_FLUSH_BYTES = 256 << 20

WORKLOADS = {
    "spgemm_rmat16": dict(kind="spgemm", scale=16, grid=8, value_type="f32",
                          desc="R-MAT scale 16 (65536^2, edge factor 16, a=.57 b=c=.19 d=.05), C = A*A, 8x8 tile grid, FP32"),
    "spgemm_rmat16_i32": dict(kind="spgemm", scale=16, grid=8, value_type="i32",
                              desc="R-MAT scale 16, C = A*A, 8x8 tile grid, int32 values in [-8, 8]"),
    "spgemm_rmat18": dict(kind="spgemm", scale=18, grid=16, value_type="f32",
                          desc="R-MAT scale 18 (262144^2), C = A*A, 16x16 tile grid, FP32"),
    "spgemm_rmat20": dict(kind="spgemm", scale=20, grid=64, value_type="f32",
                          desc="R-MAT scale 20 (1048576^2), C = A*A, 64x64 tile grid (16384-wide tiles), FP32"),
    "spgemm_stencil128": dict(kind="spgemm", matrix="stencil", g=128, grid=128, value_type="f32",
                              desc="27-point stencil Laplacian on a 128^3 grid (2097152^2), C = L*L, "
                                   "128x128 tile grid, FP32"),
    "spmm_er16k": dict(kind="spmm", matrix="er", n=16384, N=128, grid=4, dtype="f32", bdist="uniform",
                       desc="Erdos-Renyi 16384^2 (16 nnz/row) x dense 16384x128 U(-1,1), 4x4 tile grid, FP32"),
    "spmm_rmat21": dict(kind="spmm", matrix="rmat", scale=21, N=256, grid=8, dtype="f32", bdist="normal",
                        desc="R-MAT scale 21 (2097152^2) x dense 2097152x256 N(0,1), 8x8 tile grid, FP32 B/C"),
    "spmm_rmat21_bf16": dict(kind="spmm", matrix="rmat", scale=21, N=256, grid=8, dtype="bf16", bdist="normal",
                             desc="R-MAT scale 21 (2097152^2) x dense 2097152x256 N(0,1), 8x8 tile grid, "
                                  "BF16 B/C storage, FP32 accumulation"),
}


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--workload", default="spgemm_rmat16", choices=sorted(WORKLOADS))
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--no-extras", action="store_true", help="skip the secondary measurements")
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--no-cpu-baseline", action="store_true", help="skip the reference CPU timing")
    p.add_argument("--no-precision", action="store_true", help="skip the R-MAT scale-21 BF16/FP32 SpMM extra")
    p.add_argument("--no-large", action="store_true",
                   help="skip the R-MAT scale-20 and stencil-128^3 SpGEMM extras")
    p.add_argument("--path", default="fused", choices=["fused", "per_stage", "batched_graph", "learned"],
                   help="SpGEMM form timed as the step (default: all stages fused)")
    p.add_argument("--scale", type=int, default=None, help="override the R-MAT scale (profiling runs)")
    p.add_argument("--tune", action="store_true",
                   help="run the autotuner on the workload before timing and use its choice "
                        "(default: the library's defaults)")
    p.add_argument("--shard", action="store_true",
                   help="N>1: the ranks share ONE product, each computing its block-cyclic C tiles "
                        "(strong scaling; default: each rank runs its own product)")
    return p.parse_args()


# ---- distributed plumbing ---------------------------------------------------------


class Dist:
    """One process per GPU (torchrun env).  Each rank multiplies its own
    independent matrix of the workload (seed + rank): no data-path
    collective; the process group carries only the barrier around the timed
    region and the max of the ranks' times.  NCCL on GPUs; gloo where there
    is no GPU (the host-side logic is tested that way)."""

    def __init__(self, backend=None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.backend = None
        if self.world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            self.backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
            dist.init_process_group(self.backend, timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def barrier(self):
        if self.pg:
            import torch
            if self.backend == "nccl":
                self.pg.barrier(device_ids=[torch.cuda.current_device()])
            else:
                self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device="cuda" if self.backend == "nccl" else "cpu")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---- clocks ------------------------------------------------------------------------


class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
            time.sleep(0.5)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if not self.proc:
            return out
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        if not rows:
            return out
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, name in enumerate(names):
                if r[5 + k].strip().lower() == "active":
                    reasons.add(name)
        out.update(sm_mhz=statistics.median(sm) if sm else None, sm_max_mhz=max(mx) if mx else None,
                   reasons=sorted(reasons), samples=len(rows))
        return out


# ---- helpers ------------------------------------------------------------------------


def job_rate(world, work_per_rank_step, steps, max_seconds):
    """Whole-job throughput: every rank did the same work per step (weak
    scaling); the job took the slowest rank's time."""
    return world * work_per_rank_step * steps / max_seconds


def tile_nnz_grid(csr, tm, tn):
    from bcl_b200.containers import split_tiles
    _, toff, _, _ = split_tiles(csr, tm, tn)
    gm, gn = -(-csr.m // tm), -(-csr.n // tn)
    return np.diff(toff).reshape(gm, gn)


def spgemm_alg_bytes(a_nnz, b_nnz, m, k, tm, tk, nnz_c, c_tiles, vsize=4):
    """Algorithmic bytes of the stationary-C product: every tile product
    A_ik * B_kj reads its two tiles (indices + values + row pointers, the
    per-tile model of the reference's GPU driver,
    cuda/algorithms/spmm.hpp:383-394), and C is written once (col_ind, vals,
    row pointers)."""
    gm, gk = a_nnz.shape
    gn = b_nnz.shape[1]
    rows_a = np.minimum(tm, m - np.arange(gm) * tm)
    rows_b = np.minimum(tk, k - np.arange(gk) * tk)
    # only the tile products with both tiles nonempty are run (the stage maps
    # skip the others on fine grids)
    live = (a_nnz[:, None, :] > 0) & (b_nnz.T[None, :, :] > 0)          # [i, j, k]
    a_bytes = (4 + vsize) * a_nnz.astype(np.int64) + 4 * (rows_a[:, None].astype(np.int64) + 1)   # [i, k]
    b_bytes = (4 + vsize) * b_nnz.astype(np.int64) + 4 * (rows_b[:, None].astype(np.int64) + 1)   # [k, j]
    tot = int((live * (a_bytes[:, None, :] + b_bytes.T[None, :, :])).sum())
    tot += (4 + vsize) * nnz_c + 4 * c_tiles * (tm + 1)
    return tot


# The ncu summary (profiles/<name>.md) whose measured DRAM bytes belong to a
# workload's timed kernel; workloads without one report traffic as null.
PROFILE_FOR = {("spgemm_rmat16", "fused"): "spgemm_numeric_rmat16",
               ("spmm_rmat21", None): "spmm_rmat21",
               ("spmm_er16k", None): "spmm_er16k"}


def workload_traffic(workload, path=None):
    name = PROFILE_FOR.get((workload, path))
    return read_profile_traffic(name) if name else None


def read_profile_traffic(name):
    """dram bytes per launch recorded in profiles/<name>.md ("traffic_bytes_per_launch: N")."""
    path = os.path.join(ROOT, "profiles", name + ".md")
    if not os.path.exists(path):
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(path).read())
    return float(m.group(1)) if m else None


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---- our arm: SpGEMM ------------------------------------------------------------------


def spgemm_matrix(wl, seed):
    from bcl_b200 import gen
    if wl.get("matrix") == "stencil":
        return gen.stencil27(wl["g"], value_type=wl["value_type"])
    return gen.rmat(wl["scale"], seed=seed, value_type=wl["value_type"])


def plain_sampled_time(A, n_tiles, seed):
    """The per-tile-product loop (spgemm_plain) on a seeded sample of C tiles:
    each sampled tile runs its G two-phase partial products and their
    accumulation; returns the time scaled to all grid_m*grid_n tiles."""
    import torch
    from bcl_b200.containers import _tile_view, spgemm, tile_accumulate
    G = A.gn
    rng = np.random.default_rng(seed)
    picks = rng.choice(A.gm * A.gn, size=min(n_tiles, A.gm * A.gn), replace=False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for t in picks:
        i, j = divmod(int(t), A.gn)
        parts = [spgemm(_tile_view(A, (i, (k_ + i + j) % G)), _tile_view(A, ((k_ + i + j) % G, j))) for k_ in range(G)]
        tile_accumulate(parts)
    torch.cuda.synchronize()
    return (time.perf_counter() - t0) * (A.gm * A.gn) / len(picks)


def bench_spgemm(args, wl, dist, device):
    import torch
    from bcl_b200 import _lib, gen
    from bcl_b200.containers import BlockCustom, SPMatrix, spgemm, spgemm_numeric, spgemm_symbolic

    shard = bool(getattr(args, "shard", False)) and args.path == "fused"
    a = spgemm_matrix(wl, args.seed if shard else args.seed + dist.rank)
    n = a.m
    G = wl["grid"]
    ts = -(-n // G)
    products = gen.intermediate_products(a, a)
    flops = 2.0 * products
    A = SPMatrix.from_csr(a, BlockCustom((ts, ts)), device=device)
    a_nnz = tile_nnz_grid(a, ts, ts)
    stream = torch.cuda.current_stream()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    host_t = {"symbolic": 0.0, "alloc": 0.0, "numeric": 0.0, "close": 0.0}
    outbuf = {}

    pred = None
    if args.path == "learned":
        from bcl_b200 import learned as _learned
        pred = _learned.get_default(train_if_missing=False)
    learned_st = {}

    from bcl_b200 import autotune
    from bcl_b200.containers import context as _context
    ctx = _context(device)
    plan_params = None
    tuning_src = "library defaults"
    if getattr(args, "tune", False) and args.path == "fused" and not shard:
        best, _, _ = autotune.tune(A, A, reps=1)
        ctx.set_tuning(light_ub=best["light_ub"])
        plan_params = (best["grab"], best["blocks_per_sm"], best["long_seg"])
        tuning_src = "autotuned on this product before timing (bcl_b200.autotune.tune)"

    def step(record=None):
        if shard:
            # this rank's C tiles of the one product (the reference's block-cyclic owner)
            from bcl_b200.containers import spgemm_distributed
            if record:
                record[0].record(stream)
            C, _, _ = spgemm_distributed(A, A, dist.rank, dist.world)
            if record:
                record[1].record(stream)
            return (C.nnz() if C is not None else 0), None
        if args.path == "learned":
            # the learned product: prediction in place of the symbolic pass
            from bcl_b200.containers import learned_stats, spgemm_learned
            if record:
                record[0].record(stream)
            C, pl = spgemm_learned(A, A, predictor=pred, keep_plan=True)
            if record:
                record[1].record(stream)
            learned_st.update(learned_stats(pl))
            pl.close()
            return C.nnz(), None
        t0 = time.perf_counter()
        plan, out, trp, toff, nnz = spgemm_symbolic(A, A)
        if plan_params:
            plan.tune(*plan_params)
        t1 = time.perf_counter()
        # the output arrays are the caller's; reuse them while they are large enough
        if outbuf.get("cap", -1) < nnz:
            outbuf["ci"] = torch.empty(max(nnz, 1), dtype=torch.int32, device="cuda")
            outbuf["v"] = torch.empty(max(nnz, 1), dtype=torch.float32 if wl["value_type"] == "f32" else torch.int32,
                                      device="cuda")
            outbuf["cap"] = nnz
        ci, v = outbuf["ci"], outbuf["v"]
        out.col_ind, out.vals = ci.data_ptr(), v.data_ptr()
        t2 = time.perf_counter()
        if record:
            record[0].record(stream)
        spgemm_numeric(plan, A, A, out, "fused" if args.path == "fused" else args.path)
        if record:
            record[1].record(stream)
        t3 = time.perf_counter()
        plan.close()
        t4 = time.perf_counter()
        if record:
            host_t["symbolic"] += t1 - t0
            host_t["alloc"] += t2 - t1
            host_t["numeric"] += t3 - t2
            host_t["close"] += t4 - t3
        return nnz, (trp, toff, ci, v)

    for _ in range(args.warmup):
        nnz_c = step()[0]
    torch.cuda.synchronize()
    clocks = ClockSampler(device)
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches0 = _lib.load().bclx_launch_count()
    dist.barrier()
    torch.cuda.synchronize()
    for s in range(args.steps):
        flush.zero_()
        ev[s][0].record(stream)
        nnz_c = step(record=(ev[s][2], ev[s][3]))[0]
        ev[s][1].record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    launches = _lib.load().bclx_launch_count() - launches0
    clk = clocks.stop()
    step_ms = [e[0].elapsed_time(e[1]) for e in ev]
    num_ms = [e[2].elapsed_time(e[3]) for e in ev]
    total_s = dist.max(sum(step_ms) / 1e3)
    ms_per_step = total_s * 1e3 / args.steps
    if shard:  # one product per step, shared by all ranks
        value = flops * args.steps / total_s / 1e9
    else:
        value = job_rate(dist.world, flops, args.steps, total_s) / 1e9

    c_tiles = G * G
    if shard:
        from bcl_b200.containers import owned_tiles, process_grid
        rows_o, cols_o = owned_tiles(G, G, dist.rank, *process_grid(dist.world))
        c_tiles = len(rows_o) * len(cols_o)
        alg = spgemm_alg_bytes(a_nnz[rows_o, :], a_nnz[:, cols_o], n, n, ts, ts, nnz_c, c_tiles) if c_tiles else 0
    else:
        alg = spgemm_alg_bytes(a_nnz, a_nnz, n, n, ts, ts, nnz_c, c_tiles)
    hbm_peak, peak_kind = peaks()
    num_avg_s = statistics.mean(num_ms) / 1e3
    traffic = workload_traffic(args.workload, args.path)
    roofline = {"bound": "hbm", "achieved": alg / num_avg_s / 1e9, "peak": hbm_peak, "unit": "GB/s",
                "frac": alg / num_avg_s / 1e9 / hbm_peak, "traffic": traffic,
                "kernel": ("k_numeric (all SUMMA stages, one launch)" if args.path == "fused" else
                           "whole learned product" if args.path == "learned" else f"numeric pass ({args.path})"),
                "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": alg, "kernel_ms": num_avg_s * 1e3}

    # the timed loop's output buffers and the pool's cached scratch go back
    # before the end-to-end and secondary runs allocate their own
    outbuf.clear()
    from bcl_b200.containers import context
    context(device).release_cached()
    torch.cuda.empty_cache()
    # end to end: host CSR tiles in pinned memory -> device -> product -> host
    try:
        e2e = bench_spgemm_e2e(args, A, stream, flops, dist, shard)
    except Exception as e:  # e.g. pinned host memory for a very large C
        e2e = {"value": None, "unit": "GFLOP/s", "error": repr(e)[:300]}

    extras = {}
    if not args.no_extras and dist.world == 1:
        extras = spgemm_extras(args, A, a, ts, products, stream)
    cfg = {"workload": wl["desc"], "tile_grid": f"{G}x{G}", "tile": ts, "nnz_A": a.nnz, "nnz_C": nnz_c,
           "intermediate_products": products, "path": "fused SUMMA: one symbolic + one numeric launch per product",
           "l2": "flushed between steps (256 MiB write outside the timed events)",
           "parallelism": (f"one product shared by {dist.world} GPUs (block-cyclic C tiles, A replicated)"
                           if shard else f"independent products per GPU x{dist.world}")}
    cfg["tuning"] = dict({k: ctx.get_tuning(k) for k in ("light_ub", "item_outputs", "wide_light",
                                                          "btable_max_bytes")},
                         source=tuning_src,
                         plan=dict(zip(("grab", "blocks_per_sm", "long_seg"), plan_params or autotune.DEFAULT)))
    if shard:
        cfg["nnz_C"] = f"{nnz_c} on rank 0"
    line = {"metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "strong" if shard else "weak",
            "vs_baseline": None, "dtype": wl["value_type"], "data": "synthetic (seeded R-MAT)", "config": cfg,
            "hbm_gbs": alg / (total_s / args.steps) / 1e9 * dist.world,
            "roofline": roofline, "clocks": clk, "e2e": e2e, "gpu_launches": int(launches),
            "host_ms_per_step": {k: v * 1e3 / args.steps for k, v in host_t.items()},
            "step_ms": step_ms}
    if extras:
        line["extras"] = extras
    if learned_st:
        line["learned"] = dict(learned_st, misprediction_rate=learned_st["rows_redone"] / max(learned_st["heavy_rows"], 1))
    return line


def bench_spgemm_e2e(args, A, stream, flops, dist, shard=False):
    import torch
    from bcl_b200.containers import SPMatrix, spgemm, spgemm_distributed

    host = {k: getattr(A, k).cpu().pin_memory() for k in ("tile_row_ptr", "tile_offset", "col_ind", "vals")}
    dev = {k: torch.empty_like(v, device="cuda") for k, v in host.items()}
    h2d = sum(v.numel() * v.element_size() for v in host.values())
    out_host = {}

    def one():
        for k in host:
            dev[k].copy_(host[k], non_blocking=True)
        Ad = SPMatrix(A.m, A.n, A.tm, A.tn, A.dtype, A.device, dev["tile_row_ptr"], dev["tile_offset"],
                      dev["col_ind"], dev["vals"])
        C = spgemm_distributed(Ad, Ad, dist.rank, dist.world)[0] if shard else spgemm(Ad, Ad)
        if C is None:
            return 0
        nnz = C.nnz()
        d2h = 0
        for k in ("tile_row_ptr", "tile_offset", "col_ind", "vals"):
            t = getattr(C, k)
            cnt = nnz if k in ("col_ind", "vals") else t.numel()
            if k not in out_host or out_host[k].numel() < cnt:
                out_host[k] = torch.empty(max(cnt, 1), dtype=t.dtype).pin_memory()
            out_host[k][:cnt].copy_(t.reshape(-1)[:cnt], non_blocking=True)
            d2h += cnt * t.element_size()
        return d2h

    for _ in range(max(1, args.warmup)):
        one()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist.barrier()
    e0.record(stream)
    for _ in range(args.steps):
        d2h = one()
    e1.record(stream)
    torch.cuda.synchronize()
    t = dist.max(e0.elapsed_time(e1) / 1e3)
    rate = flops * args.steps / t if shard else job_rate(dist.world, flops, args.steps, t)
    forms = []
    out_host.clear()  # the pinned output buffers go back before the other forms allocate their own
    if not shard and dist.world == 1 and d2h < (4 << 30):
        forms.append(bench_spgemm_e2e_streamed(args, A, host, dev, stream, flops))
    if not shard and dist.world == 1 and d2h < (16 << 30):
        forms.append(bench_spgemm_e2e_pipelined(args, A, host, dev, stream, flops))
    one_call = {"value": rate / 1e9, "unit": "GFLOP/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": t * 1e3 / args.steps, "api": "containers.spgemm, then the output arrays copied back"}
    forms = [one_call] + [f for f in forms if f and f.get("value")]
    forms.sort(key=lambda f: -f["value"])
    best = dict(forms[0])
    if len(forms) > 1:
        best["other"] = forms[1:] if len(forms) > 2 else forms[1]
    return best


def bench_spgemm_e2e_streamed(args, A, host, dev, stream, flops):
    """The end-to-end step as a stream of products: every step copies A's
    tiles in from pinned host memory, runs containers.spgemm and copies C's
    arrays out to pinned host memory, with each step's copy out on a second
    stream while the next step's product runs (two pinned output sets, used
    in turn).  Every step's copies are inside the timed region, which ends
    when the last copy out has landed."""
    import torch
    from bcl_b200.containers import SPMatrix, spgemm
    h2d = sum(v.numel() * v.element_size() for v in host.values())
    copy = torch.cuda.Stream()
    hbuf = [{}, {}]
    state = {"d2h": 0}
    copied = [torch.cuda.Event(), torch.cuda.Event()]
    used = [False, False]

    def one(s):
        if used[s % 2]:
            # at most two steps' C in flight: step s - 2's copy out has landed
            # (so its C's memory goes back to the pool before this product)
            stream.wait_event(copied[s % 2])
        for k in host:
            dev[k].copy_(host[k], non_blocking=True)
        Ad = SPMatrix(A.m, A.n, A.tm, A.tn, A.dtype, A.device, dev["tile_row_ptr"], dev["tile_offset"],
                      dev["col_ind"], dev["vals"])
        C = spgemm(Ad, Ad)
        # nnz from the output array's length: C.nnz() would read tile_offset
        # back, a copy queued behind the previous step's copy out
        nnz = C.col_ind.numel() if C.vals.numel() > 1 else C.nnz()
        done = torch.cuda.Event()
        done.record(stream)
        copy.wait_event(done)
        hb = hbuf[s % 2]
        d2h = 0
        with torch.cuda.stream(copy):
            for k in ("tile_row_ptr", "tile_offset", "col_ind", "vals"):
                t = getattr(C, k)
                cnt = nnz if k in ("col_ind", "vals") else t.numel()
                if k not in hb or hb[k].numel() < cnt:
                    hb[k] = torch.empty(max(cnt, 1), dtype=t.dtype).pin_memory()
                hb[k][:cnt].copy_(t.reshape(-1)[:cnt], non_blocking=True)
                t.record_stream(copy)  # C's memory is not reused before its copy out
                d2h += cnt * t.element_size()
        copied[s % 2].record(copy)
        used[s % 2] = True
        state["d2h"] = d2h

    try:
        for s in range(max(1, args.warmup)):
            one(s)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for s in range(args.steps):
            one(s)
        last = torch.cuda.Event()
        last.record(copy)
        stream.wait_event(last)
        e1.record(stream)
        torch.cuda.synchronize()
    except Exception as e:  # e.g. pinned host memory
        return {"value": None, "error": repr(e)[:200]}
    t = e0.elapsed_time(e1) / 1e3
    return {"value": flops * args.steps / t / 1e9, "unit": "GFLOP/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": state["d2h"], "ms_per_step": t * 1e3 / args.steps,
            "api": "containers.spgemm per step, each step's C copied out on a second stream while the next "
                   "step's product runs"}


def bench_spgemm_e2e_pipelined(args, A, host, dev, stream, flops, block_rows=2):
    """The same end-to-end step through containers.spgemm_to_host: C is
    produced block by block (two tile rows at a time) and each block's
    arrays are copied to pinned host memory while the next block is
    computed."""
    import torch
    from bcl_b200.containers import SPMatrix, spgemm_to_host
    h2d = sum(v.numel() * v.element_size() for v in host.values())
    hbuf = {}

    def one():
        for k in host:
            dev[k].copy_(host[k], non_blocking=True)
        Ad = SPMatrix(A.m, A.n, A.tm, A.tn, A.dtype, A.device, dev["tile_row_ptr"], dev["tile_offset"],
                      dev["col_ind"], dev["vals"])
        _, blocks = spgemm_to_host(Ad, Ad, block_rows=block_rows, host=hbuf)
        return sum(sum(v.numel() * v.element_size() for v in blk[2:]) for blk in blocks)

    try:
        for _ in range(max(1, args.warmup)):
            one()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            d2h = one()
        e1.record(stream)
        torch.cuda.synchronize()
    except Exception as e:  # e.g. pinned host memory
        return {"value": None, "error": repr(e)[:200]}
    t = e0.elapsed_time(e1) / 1e3
    return {"value": flops * args.steps / t / 1e9, "unit": "GFLOP/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": t * 1e3 / args.steps,
            "api": f"containers.spgemm_to_host(block_rows={block_rows}): D2H overlapped with the next block"}


def time_region(fn, reps, stream):
    import torch
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / reps


def spgemm_extras(args, A, a, ts, products, stream):
    """Secondary numbers: the per-stage (batched SUMMA stage) form, the plain
    per-tile-product form, the int32 run, the SpMM configuration, and the
    reference CPU baseline on a row sample."""
    from bcl_b200.containers import spgemm, spgemm_plain
    flops = 2.0 * products
    ex = {}
    t = time_region(lambda: spgemm(A, A, stages="per_stage"), 3, stream)
    ex["spgemm_per_stage_gflops"] = flops / t / 1e9
    if A.gn <= 16:
        t = time_region(lambda: spgemm_plain(A, A), 1, stream)
        ex["spgemm_plain_gflops"] = flops / t / 1e9
        ex["spgemm_plain_ms"] = t * 1e3
    else:  # G^3 tile products: time a seeded sample of C tiles and scale
        t = plain_sampled_time(A, 16, args.seed)
        ex["spgemm_plain_gflops"] = flops / t / 1e9
        ex["spgemm_plain_ms"] = t * 1e3
        ex["spgemm_plain_note"] = "16 seeded C tiles (each: G partial products + accumulation), scaled to all tiles"
    try:
        t_ours = time_region(lambda: spgemm(A, A), 3, stream)
        ex["cusparse_spgemm"] = cusparse_spgemm_summary(a, products, t_ours, stream)
    except Exception as e:
        ex["cusparse_spgemm"] = {"error": repr(e)[:300]}
    try:
        ex["learned"] = learned_summary(A, products, stream)
    except Exception as e:  # keep the headline line even if an extra fails
        ex["learned"] = {"error": repr(e)}
    try:
        ex["tiling"] = tiling_summary(a, ts, stream)
    except Exception as e:
        ex["tiling"] = {"error": repr(e)}
    if A.gn <= 16:
        try:
            ex["spmm_er16k"] = spmm_summary(args, stream)
        except Exception as e:
            ex["spmm_er16k"] = {"error": repr(e)}
    if not args.no_precision and A.gn <= 16:
        try:
            ex["spmm_precision_rmat21"] = spmm_precision_summary(args, stream)
        except Exception as e:
            ex["spmm_precision_rmat21"] = {"error": repr(e)}
    if not args.no_large and A.gn <= 16:
        for name, wl_name in (("rmat20", "spgemm_rmat20"), ("stencil128", "spgemm_stencil128")):
            try:
                ex[f"spgemm_{name}"] = spgemm_large_summary(args, WORKLOADS[wl_name], stream)
            except Exception as e:
                ex[f"spgemm_{name}"] = {"error": repr(e)[:300]}
    return ex


def spgemm_large_summary(args, wl, stream, block_rows=8):
    """The large SpGEMM configurations (R-MAT s20 on 64x64 tiles, the
    27-point stencil on 128^3 with 128x128 tiles): the fused product whole;
    the fused and the learned products one block of `block_rows` C tile
    rows at a time (the learned form's temporary slots do not fit beside the
    whole C at s20), each block's C released before the next; the plain
    per-tile-product loop on 16 sampled C tiles, scaled.  GFLOP/s over the
    whole product for each, and the learned form's misprediction rate and
    wasted temporary bytes summed over the blocks."""
    import torch
    from bcl_b200 import gen, learned
    from bcl_b200.containers import BlockCustom, SPMatrix, context, learned_stats, spgemm, spgemm_sub
    a = spgemm_matrix(wl, args.seed)
    G = wl["grid"]
    ts = -(-a.m // G)
    A = SPMatrix.from_csr(a, BlockCustom((ts, ts)))
    flops = 2.0 * gen.intermediate_products(a, a)
    out = {"workload": wl["desc"], "intermediate_products": flops / 2, "block_rows": block_rows}

    def release():
        torch.cuda.synchronize()
        context().release_cached()
        torch.cuda.empty_cache()

    t = time_region(lambda: spgemm(A, A), 2, stream)
    out["fused_gflops"], out["fused_ms"] = flops / t / 1e9, t * 1e3
    release()
    pred = learned.get_default(train_if_missing=False)
    blocks = [list(range(i0, min(i0 + block_rows, A.gm))) for i0 in range(0, A.gm, block_rows)]
    for form in ("fused", "learned"):
        tot, st_sum = 0.0, {}
        for rows in blocks:
            fn = (lambda: spgemm_sub(A, A, rows, range(A.gn), form=form, predictor=pred))
            fn()  # warm (and the learned form's statistics)
            if form == "learned":
                _, pl = spgemm_sub(A, A, rows, range(A.gn), form=form, predictor=pred, keep_plan=True)
                for k, v in learned_stats(pl).items():
                    st_sum[k] = st_sum.get(k, 0) + v
                pl.close()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1) / 1e3
            release()
        out[f"{form}_blocked_gflops"], out[f"{form}_blocked_ms"] = flops / tot / 1e9, tot * 1e3
        if form == "learned":
            out["learned"] = dict(st_sum, misprediction_rate=st_sum.get("rows_redone", 0) /
                                  max(st_sum.get("heavy_rows", 1), 1),
                                  wasted_bytes=max(st_sum.get("temp_entries", 0) - st_sum.get("nnz", 0), 0) * 8)
    tp = plain_sampled_time(A, 16, args.seed)
    out["plain_gflops"], out["plain_ms"] = flops / tp / 1e9, tp * 1e3
    out["plain_note"] = "per-tile-product loop on 16 seeded C tiles, scaled to all tiles"
    out["learned_over_plain"] = out["learned_blocked_gflops"] / out["plain_gflops"]
    out["learned_over_fused_blocked"] = out["learned_blocked_gflops"] / out["fused_blocked_gflops"]
    out["batched_over_plain"] = out["fused_gflops"] / out["plain_gflops"]
    del A
    release()
    return out


def torch_csr(a, dtype=None):
    """The matrix as a torch CUDA CSR tensor (int32 indices; values cast to
    `dtype` when given): the input of the cuSPARSE comparator legs."""
    import torch
    v = torch.from_numpy(np.ascontiguousarray(a.vals)).cuda()
    return torch.sparse_csr_tensor(torch.from_numpy(a.row_ptr.astype(np.int32)).cuda(),
                                   torch.from_numpy(a.col_ind.astype(np.int32)).cuda(),
                                   v if dtype is None else v.to(dtype), size=(a.m, a.n))


def cusparse_spgemm_summary(a, products, ours_s, stream, reps=3):
    """Comparator only (never on the product path): the reference's GPU
    SpGEMM is cuSPARSE csrgemm per tile product plus csrgeam accumulation
    (cusparse_util.cuh:269-514, 86-265); here cuSPARSE multiplies the whole
    matrix in one call (torch's CUDA CSR x CSR product, cusparseSpGEMM), its
    own summation order, on the same input."""
    import torch
    M = torch_csr(a)
    out = {}
    try:
        C = M @ M
        torch.cuda.synchronize()
        out["nnz"] = int(C.values().numel())
        del C
        t = time_region(lambda: M @ M, reps, stream)
        out.update({"ms": t * 1e3, "gflops": 2.0 * products / t / 1e9, "ours_over_cusparse": t / ours_s})
    except Exception as e:
        out["error"] = repr(e)[:300]
    out["what"] = "torch CUDA CSR @ CSR (cusparseSpGEMM), whole matrix, one call"
    return out


def cusparse_spmm_leg(a, b_dev, ours_s, c_ours, stream, reps=5):
    """Comparator only: cusparseSpMM (the reference's GPU SpMM,
    cusparse_util.cuh:675-775, CSR_ALG2) via torch's CUDA CSR @ dense on the
    same A and B; reports its time, our time ratio, and the relative
    Frobenius difference between its C and ours."""
    out = {}
    import torch  # noqa: F401  (the CSR tensor and the product)
    try:
        M = torch_csr(a, b_dev.dtype)
        C = M @ b_dev
        torch.cuda.synchronize()
        if c_ours is not None:
            d = (C.float() - c_ours.float()).norm() / c_ours.float().norm().clamp_min(1e-30)
            out["rel_fro_diff_vs_ours"] = float(d)
        del C
        t = time_region(lambda: M @ b_dev, reps, stream)
        out.update({"ms": t * 1e3, "gflops": 2.0 * a.nnz * b_dev.shape[1] / t / 1e9,
                    "ours_over_cusparse": t / ours_s})
    except Exception as e:
        out["error"] = repr(e)[:300]
    return out


def learned_summary(A, products, stream):
    """The learned product on the same matrix: a trained row-nnz predictor
    sizes the work in place of the symbolic pass, mispredicted rows are
    redone exactly (bit-identical output).  Reports its speed, the
    misprediction rate and the temporary bytes written beyond the output."""
    from bcl_b200.containers import learned_stats, spgemm_learned
    from bcl_b200 import learned
    flops = 2.0 * products
    pred = learned.get_default(train_if_missing=False)
    c, plan = spgemm_learned(A, A, predictor=pred, keep_plan=True)
    st = learned_stats(plan)
    plan.close()
    del c
    t = time_region(lambda: spgemm_learned(A, A, predictor=pred), 3, stream)
    t0 = time_region(lambda: spgemm_learned(A, A, predictor=None), 3, stream)
    es = 4 + 4  # column index + value per temporary entry
    return {"gflops": flops / t / 1e9, "ms": t * 1e3,
            "no_predictor_gflops": flops / t0 / 1e9,
            "heavy_rows": st["heavy_rows"], "rows_redone": st["rows_redone"],
            "misprediction_rate": st["rows_redone"] / max(st["heavy_rows"], 1),
            "temp_entries": st["temp_entries"], "nnz": st["nnz"],
            "wasted_bytes": max(st["temp_entries"] - st["nnz"], 0) * es}


def spmm_precision_summary(args, stream):
    """BF16-storage vs FP32 SpMM: A = R-MAT scale 21 (FP32 U(-1,1)), B =
    2097152 x 256 N(0,1), 8x8 tile grid, FP32 accumulation in both.  Error
    against FP64 accumulation on 4096 seeded sampled rows (computed on the
    host in float64)."""
    import scipy.sparse as sp
    import torch
    from bcl_b200 import gen
    from bcl_b200.containers import BlockCustom, DMatrix, SPMatrix, spmm
    a = gen.rmat(21, seed=args.seed)
    N, G = 256, 8
    ts = a.m // G
    b = gen.dense(a.n, N, seed=args.seed + 7, dist="normal")
    A = SPMatrix.from_csr(a, BlockCustom((ts, ts)))
    rng = np.random.default_rng(args.seed + 11)
    rows = np.sort(rng.choice(a.m, size=4096, replace=False))
    # FP64 reference rows
    csr = sp.csr_matrix((a.vals.astype(np.float64), a.col_ind, a.row_ptr), shape=(a.m, a.n))
    ref = np.zeros((rows.size, N))
    for c0 in range(0, rows.size, 256):
        sub = csr[rows[c0:c0 + 256]]
        cols = np.unique(sub.indices)
        sub = sp.csr_matrix((sub.data, np.searchsorted(cols, sub.indices), sub.indptr), shape=(sub.shape[0], cols.size))
        ref[c0:c0 + 256] = sub @ b[cols].astype(np.float64)
    flops = 2.0 * a.nnz * N
    out = {"workload": "R-MAT scale 21 (2097152^2, nnz %d) x dense 2097152x256 N(0,1), 8x8 tile grid" % a.nnz,
           "sampled_rows": int(rows.size)}
    hbm, _ = peaks()
    times = {}
    for name, dt in (("fp32", torch.float32), ("bf16", torch.bfloat16)):
        B = DMatrix.from_array(torch.from_numpy(b), BlockCustom((ts, N)), dtype=dt)
        C = DMatrix.zeros((a.m, N), BlockCustom((ts, N)), dtype=dt)
        spmm(A, B, C)
        got = C.tiles.view(-1, N)[torch.from_numpy(rows).cuda()].float().cpu().numpy().astype(np.float64)
        t = time_region(lambda: spmm(A, B, C), 3, stream)  # C += A*B again each time: same work
        C0 = DMatrix.zeros((a.m, N), BlockCustom((ts, N)), dtype=dt)
        spmm(A, B, C0)
        cus = cusparse_spmm_leg(a, B.get_matrix(), t, C0.get_matrix(), stream)
        del C0
        es = 4 if name == "fp32" else 2
        alg = 8 * a.nnz + 4 * (a.m + 1) * G + es * a.n * N + 2 * es * a.m * N
        err = np.abs(got - ref)
        nz = ref != 0  # entries of rows with products (many R-MAT rows are empty)
        rel = err[nz] / np.abs(ref[nz])
        times[name] = t
        out[name] = {"ms": t * 1e3, "gflops": flops / t / 1e9, "alg_gbs": alg / t / 1e9,
                     "frac_hbm": alg / t / 1e9 / hbm,
                     "rel_fro_err_vs_fp64": float(np.linalg.norm(err) / np.linalg.norm(ref)),
                     "max_abs_err_over_max_abs": float(err.max() / np.abs(ref).max()),
                     "median_rel_entry_err": float(np.median(rel)) if rel.size else 0.0,
                     "p99_rel_entry_err": float(np.quantile(rel, 0.99)) if rel.size else 0.0,
                     "entries_checked": int(nz.sum()), "cusparse": cus}
        del B, C
        torch.cuda.empty_cache()
    out["bf16_speedup"] = times["fp32"] / times["bf16"]
    out["alg_bytes_model"] = "A once (8 B/entry + row pointers per tile), B once, C read and written once"
    return out


def tiling_summary(a, ts, stream):
    """The input path on the device: slicing A (already a device CSR) into
    its tile grid (bclx_csr_to_tiles) and gathering it back
    (bclx_tiles_to_csr), against the host slicing of the same matrix."""
    import torch
    from bcl_b200.containers import SPMatrix, split_tiles
    rp = torch.from_numpy(a.row_ptr.astype(np.int32)).cuda()
    ci = torch.from_numpy(a.col_ind).cuda()
    v = torch.from_numpy(a.vals).cuda()
    holder = {}

    def tile():
        holder["S"] = SPMatrix.from_device_csr(a.m, a.n, rp, ci, v, (ts, ts))
    t_tile = time_region(tile, 5, stream)
    S = holder["S"]
    t_gather = time_region(lambda: S.get_device(), 5, stream)
    t0 = time.perf_counter()
    split_tiles(a, ts, ts)
    t_host = time.perf_counter() - t0
    ntiles = S.gm * S.gn
    # bytes read and written once: CSR in (row_ptr, col, val), tiles out (row ptrs, offsets, col, val)
    moved = 4 * (a.m + 1) + 8 * a.nnz + 4 * ntiles * (ts + 1) + 8 * (ntiles + 1) + 8 * a.nnz
    return {"nnz": a.nnz, "tile_ms": t_tile * 1e3, "tile_gbs": moved / t_tile / 1e9,
            "gather_ms": t_gather * 1e3, "gather_gbs": moved / t_gather / 1e9,
            "host_slicing_ms": t_host * 1e3, "note": "device slicing includes one host read (validation)"}


def spmm_summary(args, stream):
    import torch
    from bcl_b200 import gen
    from bcl_b200.containers import BlockCustom, DMatrix, SPMatrix, spmm, spmm_plain
    wl = WORKLOADS["spmm_er16k"]
    n, N, G = wl["n"], wl["N"], wl["grid"]
    ts = n // G
    a = gen.erdos_renyi(n, 16, seed=args.seed)
    b = gen.dense(n, N, seed=args.seed + 1)
    A = SPMatrix.from_csr(a, BlockCustom((ts, ts)))
    B = DMatrix.from_array(torch.from_numpy(b), BlockCustom((ts, N)))
    C = DMatrix.zeros((n, N), BlockCustom((ts, N)))
    flops = 2.0 * a.nnz * N
    # compulsory bytes: A (indices, values, row pointers) and B read once, C read and written once
    alg = 8 * a.nnz + 4 * (ts + 1) * G * G + 4 * n * N + 8 * n * N
    # reference model per tile product: indices + values of A_ik, B_kj, C_ij read and written once
    tile_nnz = tile_nnz_grid(a, ts, ts)
    ref_model = 0
    for i in range(G):
        for k in range(G):
            ref_model += 8 * int(tile_nnz[i, k]) + 4 * (ts + 1) + 4 * ts * N + 8 * ts * N
    t = time_region(lambda: spmm(A, B, C), 20, stream)
    tp = time_region(lambda: spmm_plain(A, B, C), 5, stream)
    B16 = DMatrix.from_array(torch.from_numpy(b), BlockCustom((ts, N)), dtype=torch.bfloat16)
    C16 = DMatrix.zeros((n, N), BlockCustom((ts, N)), dtype=torch.bfloat16)
    t16 = time_region(lambda: spmm(A, B16, C16), 20, stream)
    C0 = DMatrix.zeros((n, N), BlockCustom((ts, N)))
    spmm(A, B, C0)
    cus = cusparse_spmm_leg(a, B.get_matrix(), t, C0.get_matrix(), stream, reps=20)
    hbm, _ = peaks()
    return {"workload": wl["desc"], "gflops": flops / t / 1e9, "alg_gbs": alg / t / 1e9, "frac_hbm": alg / t / 1e9 / hbm,
            "bytes_model": "compulsory", "reference_model_gbs": ref_model / t / 1e9, "ms": t * 1e3, "plain_gflops": flops / tp / 1e9, "bf16_gflops": flops / t16 / 1e9,
            "bf16_speedup": t / t16, "cusparse": cus}


def spmm_inputs(wl, seed):
    from bcl_b200 import gen
    if wl["matrix"] == "er":
        a = gen.erdos_renyi(wl["n"], 16, seed=seed)
    else:
        a = gen.rmat(wl["scale"], seed=seed)
    b = gen.dense(a.n, wl["N"], seed=seed + 1, dist=wl["bdist"])
    return a, b


def spmm_model_bytes(a, ts, G, N, es):
    """The reference's per-tile-product bytes (cuda/algorithms/spmm.hpp:383-394):
    A_ik indices + values + row pointers, B_kj and C_ij once per product."""
    tile_nnz = tile_nnz_grid(a, ts, ts)
    total = 0
    for i in range(G):
        rows = min(ts, a.m - i * ts)
        for k in range(G):
            cols = min(ts, a.n - k * ts)
            total += 8 * int(tile_nnz[i, k]) + 4 * (rows + 1) + es * cols * N + es * rows * N
    return total


def bench_spmm(args, wl, dist, device):
    """C += A*B over the tile grids (BCL::gemm(SPMatrix, DMatrix, DMatrix&)),
    one product per step (k_spmm, and k_spmm_long beside it on products with
    at least 65536 A rows)."""
    import torch
    from bcl_b200 import _lib
    from bcl_b200.containers import BlockCustom, DMatrix, SPMatrix, spmm
    a, b = spmm_inputs(wl, args.seed + dist.rank)
    N, G = wl["N"], wl["grid"]
    ts = -(-a.m // G)
    tdt = torch.float32 if wl["dtype"] == "f32" else torch.bfloat16
    es = 4 if wl["dtype"] == "f32" else 2
    A = SPMatrix.from_csr(a, BlockCustom((ts, ts)), device=device)
    B = DMatrix.from_array(torch.from_numpy(b), BlockCustom((ts, N)), dtype=tdt)
    C = DMatrix.zeros((a.m, N), BlockCustom((ts, N)), dtype=tdt)
    flops = 2.0 * a.nnz * N
    stream = torch.cuda.current_stream()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    from bcl_b200 import autotune
    from bcl_b200.containers import context as _context
    ctx = _context(device)
    tuning_src = "library defaults"
    if getattr(args, "tune", False):
        best, _ = autotune.tune_spmm(A, B, C)
        ctx.set_tuning(**best)
        tuning_src = "autotuned on this product before timing (bcl_b200.autotune.tune_spmm)"
    for _ in range(args.warmup):
        spmm(A, B, C)
    torch.cuda.synchronize()
    clocks = ClockSampler(device)
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches0 = _lib.load().bclx_launch_count()
    dist.barrier()
    torch.cuda.synchronize()
    for s_ in range(args.steps):
        flush.zero_()
        ev[s_][0].record(stream)
        spmm(A, B, C)
        ev[s_][1].record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    launches = _lib.load().bclx_launch_count() - launches0
    clk = clocks.stop()
    step_ms = [e[0].elapsed_time(e[1]) for e in ev]
    total_s = dist.max(sum(step_ms) / 1e3)
    ms_per_step = total_s * 1e3 / args.steps
    value = job_rate(dist.world, flops, args.steps, total_s) / 1e9
    hbm_peak, peak_kind = peaks()
    kern_s = statistics.mean(step_ms) / 1e3  # the step is the product's kernels
    model = spmm_model_bytes(a, ts, G, N, es)
    compulsory = 8 * a.nnz + 4 * (ts + 1) * G * G + es * a.n * N + 2 * es * a.m * N
    # the roofline counts compulsory bytes (A, B once; C read and written
    # once); the reference's per-tile-product model counts each B tile once per
    # C tile that uses it, bytes a kernel need not move, and is kept beside it
    roofline = {"bound": "hbm", "achieved": compulsory / kern_s / 1e9, "peak": hbm_peak, "unit": "GB/s",
                "frac": compulsory / kern_s / 1e9 / hbm_peak, "traffic": workload_traffic(args.workload),
                "kernel": "k_spmm + k_spmm_long (one product, all SUMMA stages)", "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": compulsory,
                "bytes_model": "compulsory: A and B read once, C read and written once",
                "reference_model_bytes_per_launch": model,
                "reference_model": "per-tile-product model (spmm.hpp:383-394): A_ik, B_kj, C_ij once per product",
                "reference_model_gbs": model / kern_s / 1e9, "kernel_ms": kern_s * 1e3}
    e2e = bench_spmm_e2e(args, A, B, C, stream, flops, dist)
    cfg = {"workload": wl["desc"], "tile_grid": f"{G}x{G}", "tile": ts, "nnz_A": a.nnz, "N": N,
           "path": "k_spmm (short rows, grouped per warp) + k_spmm_long (rows of >= 1024 entries, side "
                   "stream): every C row sums its stages in rotated order, C += A*B in place",
           "l2": "flushed between steps (256 MiB write outside the timed events)" if wl["matrix"] == "er"
                 else "inputs larger than L2 (B %d MB)" % (a.n * N * es >> 20),
           "parallelism": f"independent products per GPU x{dist.world}",
           "tuning": dict({k: ctx.get_tuning(k) for k in ("spmm_rows", "spmm_long_row", "spmm_long_blocks",
                                                          "spmm_schedule", "spmm_panel_major")},
                          source=tuning_src)}
    line = {"metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if wl["dtype"] == "f32" else "bf16 storage, f32 accumulate",
            "data": "synthetic (seeded)", "config": cfg,
            "hbm_gbs": model / (total_s / args.steps) / 1e9 * dist.world,
            "roofline": roofline, "clocks": clk, "e2e": e2e, "gpu_launches": int(launches), "step_ms": step_ms}
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline_spmm(a, b, wl)
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "error": repr(e)}
    return line


def bench_spmm_e2e(args, A, B, C, stream, flops, dist):
    """Every step: A's tiles and B from pinned host memory, C zeroed, the
    product, C back to pinned host memory."""
    import torch
    from bcl_b200.containers import SPMatrix, spmm
    host = {k: getattr(A, k).cpu().pin_memory() for k in ("tile_row_ptr", "tile_offset", "col_ind", "vals")}
    dev = {k: torch.empty_like(v, device="cuda") for k, v in host.items()}
    hb = B.tiles.cpu().pin_memory()
    hc = torch.empty(C.tiles.shape, dtype=C.tiles.dtype).pin_memory()
    h2d = sum(v.numel() * v.element_size() for v in host.values()) + hb.numel() * hb.element_size()
    d2h = hc.numel() * hc.element_size()

    def one():
        for k in host:
            dev[k].copy_(host[k], non_blocking=True)
        B.tiles.copy_(hb, non_blocking=True)
        C.tiles.zero_()
        Ad = SPMatrix(A.m, A.n, A.tm, A.tn, A.dtype, A.device, dev["tile_row_ptr"], dev["tile_offset"],
                      dev["col_ind"], dev["vals"])
        spmm(Ad, B, C)
        hc.copy_(C.tiles, non_blocking=True)

    for _ in range(max(1, args.warmup)):
        one()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist.barrier()
    e0.record(stream)
    for _ in range(args.steps):
        one()
    e1.record(stream)
    torch.cuda.synchronize()
    t = dist.max(e0.elapsed_time(e1) / 1e3)
    one_call = {"value": job_rate(dist.world, flops, args.steps, t) / 1e9, "unit": "GFLOP/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": t * 1e3 / args.steps,
                "api": "containers.spmm with every copy on the product's stream"}
    streamed = bench_spmm_e2e_streamed(args, A, B, C, host, hb, hc, stream, flops, dist)
    forms = sorted([f for f in (one_call, streamed) if f and f.get("value")], key=lambda f: -f["value"])
    best = dict(forms[0])
    if len(forms) > 1:
        best["other"] = forms[1]
    return best


def bench_spmm_e2e_streamed(args, A, B, C, host, hb, hc, stream, flops, dist):
    """The end-to-end SpMM as a stream of products over two sets of device
    buffers used in turn: each step copies A's tiles and B in from pinned
    host memory on one stream, zeroes C and runs containers.spmm on the
    product's stream, and copies C out on a third, so that one step's copy
    in, another's product and a third's copy out overlap (PCIe carries both
    directions at once).  Every step's copies are inside the timed region,
    which ends when the last copy out has landed."""
    import torch
    from bcl_b200.containers import DMatrix, SPMatrix, spmm
    ok, err, t_local = True, "", 0.0
    try:
        sets = []
        for i in range(2):
            dev = {k: torch.empty_like(v, device="cuda") for k, v in host.items()}
            Bi = B if i == 0 else DMatrix(B.m, B.n, B.tm, B.tn, torch.empty_like(B.tiles))
            Ci = C if i == 0 else DMatrix(C.m, C.n, C.tm, C.tn, torch.empty_like(C.tiles))
            sets.append((dev, Bi, Ci))
        cin, cout = torch.cuda.Stream(), torch.cuda.Stream()
        loaded = [torch.cuda.Event(), torch.cuda.Event()]
        computed = [torch.cuda.Event(), torch.cuda.Event()]
        copied = [torch.cuda.Event(), torch.cuda.Event()]
        used = [False, False]

        def one(s):
            i = s % 2
            dev, Bi, Ci = sets[i]
            if used[i]:
                cin.wait_event(computed[i])  # set i's inputs are no longer read
            with torch.cuda.stream(cin):
                for k in host:
                    dev[k].copy_(host[k], non_blocking=True)
                Bi.tiles.copy_(hb, non_blocking=True)
            loaded[i].record(cin)
            stream.wait_event(loaded[i])
            if used[i]:
                stream.wait_event(copied[i])  # set i's C has been copied out
            Ci.tiles.zero_()
            Ad = SPMatrix(A.m, A.n, A.tm, A.tn, A.dtype, A.device, dev["tile_row_ptr"], dev["tile_offset"],
                          dev["col_ind"], dev["vals"])
            spmm(Ad, Bi, Ci)
            computed[i].record(stream)
            cout.wait_event(computed[i])
            with torch.cuda.stream(cout):
                hc.copy_(Ci.tiles, non_blocking=True)
            copied[i].record(cout)
            used[i] = True

        for s in range(max(1, args.warmup)):
            one(s)
        torch.cuda.synchronize()
    except Exception as e:  # e.g. device memory for the second set
        ok, err = False, repr(e)[:200]
    # every rank takes the same collective steps, failed or not
    dist.barrier()
    if ok:
        try:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for s in range(args.steps):
                one(s)
            last = torch.cuda.Event()
            last.record(cout)
            stream.wait_event(last)
            e1.record(stream)
            torch.cuda.synchronize()
            t_local = e0.elapsed_time(e1) / 1e3
        except Exception as e:
            ok, err = False, repr(e)[:200]
    t = dist.max(t_local)
    if dist.max(0.0 if ok else 1.0) > 0.0:
        return {"value": None, "error": err or "failed on another rank"}
    h2d = sum(v.numel() * v.element_size() for v in host.values()) + hb.numel() * hb.element_size()
    return {"value": job_rate(dist.world, flops, args.steps, t) / 1e9, "unit": "GFLOP/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": hc.numel() * hc.element_size(), "ms_per_step": t * 1e3 / args.steps,
            "api": "containers.spmm per step over two buffer sets; copies in, products and copies out of "
                   "different steps overlap on three streams"}


# ---- CPU baselines (the reference's own code) -------------------------------------------


def row_sample(a, stride):
    from bcl_b200 import gen
    rows = np.arange(0, a.m, stride)
    rp = a.row_ptr.astype(np.int64)
    counts = rp[rows + 1] - rp[rows]
    idx = np.concatenate([np.arange(rp[r], rp[r + 1]) for r in rows]) if rows.size else np.zeros(0, np.int64)
    nrp = np.zeros(rows.size + 1, np.int64)
    np.cumsum(counts, out=nrp[1:])
    return gen.CSR(rows.size, a.n, nrp.astype(np.int32), a.col_ind[idx], a.vals[idx])


def reference_ranks():
    """Reference processes run at once: one per host core."""
    return max(1, os.cpu_count() or 1)


def run_reference_ranks(jobs, timeout=3000, threads=1):
    """Run the reference binary once per argument list, all at the same time
    (with one list per host core: the reference's one rank per core, each
    owning its own C rows), `threads` OpenMP threads each; returns the
    processes' JSON lines."""
    from oracle import oracle as O
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    procs = [subprocess.Popen([O.REF_BIN] + [str(x) for x in j], stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                              text=True, env=env) for j in jobs]
    out = []
    try:
        for p in procs:
            so, se = p.communicate(timeout=timeout)
            if p.returncode != 0:
                raise RuntimeError(f"bcl_ref exited {p.returncode}: {se[-300:]}")
            lines = [ln for ln in so.splitlines() if ln.strip().startswith("{")]
            if not lines:
                raise RuntimeError(f"bcl_ref printed no result: {so[-300:]!r}")
            out.append(json.loads(lines[-1]))
    finally:  # none of these processes outlives a failure of another
        for p in procs:
            if p.poll() is None:
                p.kill()
                p.wait()
    return out


def split_rows(s, parts):
    """Rows p, p + parts, p + 2 parts, ... of CSR `s`, for p < parts."""
    from bcl_b200 import gen
    out = []
    rp = s.row_ptr.astype(np.int64)
    for p in range(parts):
        rows = np.arange(p, s.m, parts)
        if rows.size == 0:
            continue
        counts = rp[rows + 1] - rp[rows]
        idx = np.concatenate([np.arange(rp[r], rp[r + 1]) for r in rows])
        nrp = np.zeros(rows.size + 1, np.int64)
        np.cumsum(counts, out=nrp[1:])
        out.append(gen.CSR(rows.size, s.n, nrp.astype(np.int32), s.col_ind[idx], s.vals[idx]))
    return out


def best_layout(run, rows, run_ranks=None):
    """Time `run(parts, threads)` as one process with every host thread and
    as one single-threaded process per core (rows dealt round-robin), and
    `run_ranks(pm, pn)`, the reference's own distributed BCL::gemm with one
    rank per core on a pm x pn process grid (when its binary is built);
    return (seconds per rep, layout) of the fastest, the layout being
    ("threads", n), ("rows", processes) or ("ranks", pm, pn)."""
    from oracle import oracle as O
    cores = reference_ranks()
    best = (run(1, cores), ("threads", cores))
    procs = min(cores, rows)
    if procs > 1:
        t = run(procs, 1)
        if t < best[0]:
            best = (t, ("rows", procs))
    if run_ranks is not None and cores > 1 and O.ref_mp_available():
        pm = int(cores ** 0.5)
        while cores % pm:
            pm -= 1
        try:
            t = run_ranks(pm, cores // pm)
        except (RuntimeError, OSError, subprocess.SubprocessError) as e:  # an extra layout: the others stand
            print(f"reference on {cores} ranks skipped: {e}", file=sys.stderr)
            t = None
        if t is not None and t < best[0]:
            best = (t, ("ranks", pm, cores // pm))
    return best


def reference_spgemm_sample(a, G, stride, warmup, reps):
    """Run the reference's BCL::gemm on every `stride`-th row of A times A
    (same tile columns; tile height scaled so the grid stays G x G), as one
    process with every host thread and as one process per host core with the
    sample's rows dealt round-robin.  Returns (products, seconds per rep of
    the slowest process in the faster layout, rows, processes)."""
    from bcl_b200 import gen
    s = row_sample(a, stride)
    ts = -(-a.m // G)
    products = gen.intermediate_products(s, a)
    mode = "f32" if a.vals.dtype == np.float32 else "i32"

    def run(nparts, threads):
        parts = split_rows(s, nparts)
        with tempfile.TemporaryDirectory() as d:
            fb = os.path.join(d, "a.binary")
            gen.write_binary(fb, a)
            jobs = []
            for i, q in enumerate(parts):
                fa = os.path.join(d, f"s{i}.binary")
                gen.write_binary(fa, q)
                jobs.append(["spgemm", fa, fb, -(-q.m // G), ts, ts, mode, "-", warmup, reps])
            res = run_reference_ranks(jobs, threads=threads)
        return max(statistics.mean(r["times_s"]) for r in res)

    def run_ranks(pm, pn):
        from oracle import oracle as O
        with tempfile.TemporaryDirectory() as d:
            fa, fb = os.path.join(d, "s.binary"), os.path.join(d, "a.binary")
            gen.write_binary(fa, s)
            gen.write_binary(fb, a)
            res = O.run_ref_mp(["spgemm", fa, fb, -(-s.m // G), ts, ts, pm, pn, mode, "-", warmup, reps], pm * pn)
        return statistics.mean(res["times_s"])

    t, layout = best_layout(run, s.m, run_ranks)
    return products, t, s.m, layout


def layout_note(layout):
    if layout[0] == "threads":
        return f"one process, {layout[1]} OpenMP threads (only the accumulate is threaded)"
    if layout[0] == "rows":
        return (f"the rows dealt to {layout[1]} processes run at once (one per core, 1 thread each), time of the "
                f"slowest")
    pm, pn = layout[1], layout[2]
    return (f"the reference's distributed BCL::gemm on {pm * pn} ranks ({pm}x{pn} process grid, one per core, "
            f"1 thread each), barrier to barrier")


def cpu_baseline_spgemm(a, G, stride=16):
    products, t, rows, layout = reference_spgemm_sample(a, G, stride, 0, 1)
    return {"value": 2.0 * products / t / 1e9, "unit": "GFLOP/s", "cores": reference_ranks(),
            "kind": "reference",
            "sample": f"every {stride}th row of A ({rows} rows, {products} products) times A, {G}x{G} tile grid, "
                      f"reference BCL::gemm built from its headers; the fastest of one multi-threaded process, "
                      f"one process per core and the distributed gemm on one rank per core: {layout_note(layout)}",
            "seconds": t}


def spmm_cpu_sample(a, b, wl):
    """Row stride for the reference SpMM sample: all rows for the ER
    configuration (CPU-runnable whole), every 64th row at scale 21."""
    return 1 if wl["matrix"] == "er" else 64


def reference_spmm_sample(a, b, wl, stride, warmup, reps):
    """The reference's BCL::gemm(SPMatrix, DMatrix) on every `stride`-th row
    of A times B, as one process and as one process per host core with the
    rows dealt round-robin.  Returns (flops, seconds per rep of the slowest
    process in the faster layout, rows, processes)."""
    from bcl_b200 import gen
    s = row_sample(a, stride) if stride > 1 else a
    G = wl["grid"]
    ts = -(-a.n // G)
    if wl["dtype"] != "f32":
        raise ValueError("the reference SpMM is FP32 only (spgemm.hpp:80-96)")
    def run(nparts, threads):
        parts = split_rows(s, nparts)
        with tempfile.TemporaryDirectory() as d:
            fb = os.path.join(d, "b.dense")
            gen.write_dense(fb, b)
            jobs = []
            for i, q in enumerate(parts):
                fa = os.path.join(d, f"s{i}.binary")
                gen.write_binary(fa, q)
                jobs.append(["spmm", fa, fb, -(-q.m // G), ts, wl["N"], "-", warmup, reps])
            res = run_reference_ranks(jobs, threads=threads)
        return max(statistics.mean(r["times_s"]) for r in res)

    def run_ranks(pm, pn):
        from oracle import oracle as O
        with tempfile.TemporaryDirectory() as d:
            fa, fb = os.path.join(d, "s.binary"), os.path.join(d, "b.dense")
            gen.write_binary(fa, s)
            gen.write_dense(fb, b)
            res = O.run_ref_mp(["spmm", fa, fb, -(-s.m // G), ts, wl["N"], pm, pn, "-", warmup, reps], pm * pn)
        return statistics.mean(res["times_s"])

    t, layout = best_layout(run, s.m, run_ranks)
    return 2.0 * s.nnz * wl["N"], t, s.m, layout


def cpu_baseline_spmm(a, b, wl):
    stride = spmm_cpu_sample(a, b, wl)
    flops, t, rows, layout = reference_spmm_sample(a, b, wl, stride, 0, 1 if stride > 1 else 3)
    return {"value": flops / t / 1e9, "unit": "GFLOP/s", "cores": reference_ranks(), "kind": "reference",
            "sample": (f"every {stride}th row of A ({rows} rows)" if stride > 1 else "the whole product") +
                      f" times B ({a.n}x{wl['N']}), reference BCL::gemm(SPMatrix, DMatrix) built from its "
                      f"headers; the fastest of one process, one process per core and the distributed gemm on "
                      f"one rank per core (its SpMM loop is serial): {layout_note(layout)}", "seconds": t}


def run_reference(args, dist):
    """The reference arm: the reference's own CPU BCL::gemm on this config,
    all host threads, each step a bounded row sample of the same product."""
    if dist.rank != 0:
        return None
    from bcl_b200 import gen
    from oracle import oracle as O
    wl = WORKLOADS[args.workload]
    if not O.ref_available():
        return {"impl": "reference", "unavailable": "reference CPU binary oracle/_ref/bcl_ref was not built"}
    if wl["kind"] == "spmm":
        if wl["dtype"] != "f32":
            return {"impl": "reference", "unavailable": "the reference SpMM has no BF16 storage (FP32 only)"}
        a, b = spmm_inputs(wl, args.seed)
        stride = spmm_cpu_sample(a, b, wl)
        flops, t, rows, layout = reference_spmm_sample(a, b, wl, stride, args.warmup, args.steps)
        value = flops / t / 1e9
        sample = ((f"every {stride}th row of A ({rows} rows)" if stride > 1 else "the whole product") +
                  f" times B; {layout_note(layout)}")
        return {"metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
                "config": {"workload": wl["desc"], "tile_grid": f"{wl['grid']}x{wl['grid']}", "sample": sample},
                "impl": "reference",
                "cpu_baseline": {"value": value, "unit": "GFLOP/s", "cores": reference_ranks(), "kind": "reference",
                                 "sample": sample + f", {args.steps} reps"},
                "e2e": {"value": value, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "gpu_launches": 0}
    a = spgemm_matrix(wl, args.seed)
    G = wl["grid"]
    stride = 128 if a.m <= 65536 else 2048
    products, t, rows, layout = reference_spgemm_sample(a, G, stride, args.warmup, args.steps)
    value = 2.0 * products / t / 1e9
    return {"metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": wl["value_type"], "data": "synthetic (seeded R-MAT)",
            "config": {"workload": wl["desc"], "tile_grid": f"{G}x{G}",
                       "sample": f"every {stride}th row of A ({rows} rows, {products} products) times A; "
                                 f"{layout_note(layout)}"},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "GFLOP/s", "cores": reference_ranks(), "kind": "reference",
                             "sample": f"every {stride}th row of A times A, {G}x{G} tiles; {layout_note(layout)}, "
                                       f"{args.steps} reps"},
            "e2e": {"value": value, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "gpu_launches": 0}


def main():
    args = parse_args()
    dist = Dist()
    if args.impl == "reference":
        line = run_reference(args, dist)
        if line is not None:
            print(json.dumps(line), flush=True)
        dist.close()
        return
    import torch
    device = dist.local_rank
    torch.cuda.set_device(device)
    wl = dict(WORKLOADS[args.workload])
    if args.scale is not None:
        wl["scale"] = args.scale
        wl["desc"] = wl["desc"].replace("scale 16", f"scale {args.scale}") + " (scale overridden)"
    if wl["kind"] == "spgemm":
        line = bench_spgemm(args, wl, dist, device)
        if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
            a = spgemm_matrix(wl, args.seed)
            try:
                line["cpu_baseline"] = cpu_baseline_spgemm(a, wl["grid"], stride=64 if a.m <= 65536 else 1024)
            except Exception as e:
                line["cpu_baseline"] = {"value": None, "error": repr(e)}
    else:
        line = bench_spmm(args, wl, dist, device)
    if dist.rank == 0:
        print(json.dumps(line), flush=True)
    dist.close()


if __name__ == "__main__":
    main()
