"""ctypes front end of the C restatement in oracle.c, and runners for the
reference's own CPU binaries (_ref/bcl_ref: one rank; _ref/bcl_ref_mp: the
reference's distributed BCL::gemm on several ranks over the shared-memory
MPI subset in ref_stubs_mp/).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by bench.py's CPU-baseline and reference legs, always as the checker or
the baseline, never as the product path.  See oracle.c for the reference
files and lines each function follows and how the restatement is pinned.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "bcl_ref")
REF_MP_BIN = os.path.join(HERE, "_ref", "bcl_ref_mp")

_lib = None


def build() -> None:
    """Compile liboracle.so (and the reference binary when its tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.oracle_spgemm_count.restype = ctypes.c_int64
        _lib.oracle_accumulate_count.restype = ctypes.c_int64
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _i64(*xs):
    return [ctypes.c_int64(int(x)) for x in xs]


def _rows_arg(rows):
    if rows is None:
        return None, 0
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    return rows, rows.size


def spgemm_count(a, b, rows=None):
    """Per-row nnz of C = A*B (all rows, or the listed ones)."""
    rows, nr = _rows_arg(rows)
    nout = a.m if rows is None else nr
    counts = np.zeros(nout, dtype=np.int64)
    lib().oracle_spgemm_count(*_i64(a.m, b.n), _p(a.row_ptr), _p(a.col_ind), _p(b.row_ptr),
                              _p(b.col_ind), _p(rows), ctypes.c_int64(nr), _p(counts))
    return counts


def gemm_tiled(a, b, tm, tk, tn, rows=None, mode="f32", use_fma=True):
    """Stationary-C tiled product C = A*B with the reference's per-entry
    summation order.  ``mode``: "f32" (float inputs, FP32 result), "i32",
    "f64" (float inputs accumulated in double).  Returns (row_ptr int64,
    col_ind int32, vals) over all rows or the listed rows."""
    rows_a, nr = _rows_arg(rows)
    counts = spgemm_count(a, b, rows_a)
    offsets = np.zeros(counts.size + 1, dtype=np.int64)
    np.cumsum(counts, out=offsets[1:])
    nnz = int(offsets[-1])
    cci = np.empty(nnz, dtype=np.int32)
    if mode == "f32":
        cv, fn, vt = np.empty(nnz, np.float32), lib().oracle_gemm_tiled_f32, np.float32
    elif mode == "i32":
        cv, fn, vt = np.empty(nnz, np.int32), lib().oracle_gemm_tiled_i32, np.int32
    elif mode == "f64":
        cv, fn, vt = np.empty(nnz, np.float64), lib().oracle_gemm_tiled_f64, np.float32
    else:
        raise ValueError(mode)
    av = np.ascontiguousarray(a.vals, dtype=vt)
    bv = np.ascontiguousarray(b.vals, dtype=vt)
    fn(*_i64(a.m, a.n, b.n), _p(a.row_ptr), _p(a.col_ind), _p(av), _p(b.row_ptr), _p(b.col_ind),
       _p(bv), *_i64(tm, tk, tn), _p(rows_a), ctypes.c_int64(nr), _p(offsets), _p(cci), _p(cv),
       ctypes.c_int(1 if use_fma else 0))
    return offsets, cci, cv


def spgemm_local(a, b, mode="f32", use_fma=True):
    """Untiled local product (CSRMatrix::dot): one tile covering everything."""
    big = max(a.m, a.n, b.n, 1)
    return gemm_tiled(a, b, big, big, big, mode=mode, use_fma=use_fma)


def accumulate(parts, mode="f32"):
    """Sum of partial CSRs (same shape) in list order, union structure."""
    m, n = parts[0].m, parts[0].n
    P = len(parts)
    rps = (ctypes.c_void_p * P)(*[p.row_ptr.ctypes.data for p in parts])
    cis = (ctypes.c_void_p * P)(*[p.col_ind.ctypes.data for p in parts])
    vt = np.float32 if mode == "f32" else np.int32
    vals = [np.ascontiguousarray(p.vals, dtype=vt) for p in parts]
    vs = (ctypes.c_void_p * P)(*[v.ctypes.data for v in vals])
    counts = np.zeros(m, dtype=np.int64)
    lib().oracle_accumulate_count(*_i64(m, n, P), rps, cis, _p(counts))
    offsets = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(counts, out=offsets[1:])
    nnz = int(offsets[-1])
    cci = np.empty(nnz, np.int32)
    cv = np.empty(nnz, vt)
    fn = lib().oracle_accumulate_f32 if mode == "f32" else lib().oracle_accumulate_i32
    fn(*_i64(m, n, P), rps, cis, vs, _p(offsets), _p(cci), _p(cv))
    return offsets, cci, cv


def spmm_tiled(a, b, c0, tm, tk, tn, rows=None, use_fma=True):
    """C = C0 + A*B (FP32, in place on a copy) with the reference's order.
    With ``rows``, c0 is the (len(rows) x N) block of those rows."""
    rows_a, nr = _rows_arg(rows)
    c = np.array(c0, dtype=np.float32, copy=True, order="C")
    b = np.ascontiguousarray(b, dtype=np.float32)
    av = np.ascontiguousarray(a.vals, dtype=np.float32)
    lib().oracle_spmm_tiled_f32(*_i64(a.m, a.n, b.shape[1]), _p(a.row_ptr), _p(a.col_ind), _p(av),
                                _p(b), ctypes.c_int64(b.shape[1]), _p(c), ctypes.c_int64(c.shape[1]),
                                *_i64(tm, tk, tn), _p(rows_a), ctypes.c_int64(nr),
                                ctypes.c_int(1 if use_fma else 0))
    return c


def spmm_rowwise(a, b, c0, tm, tk, tn, rows=None):
    """C = C0 + A*B with the stages in ascending k (rowwise_gemm and its
    cached / batched variants, experimental_gemm.hpp:83-214)."""
    rows_a, nr = _rows_arg(rows)
    c = np.array(c0, dtype=np.float32, copy=True, order="C")
    b = np.ascontiguousarray(b, dtype=np.float32)
    av = np.ascontiguousarray(a.vals, dtype=np.float32)
    lib().oracle_spmm_rowwise_f32(*_i64(a.m, a.n, b.shape[1]), _p(a.row_ptr), _p(a.col_ind), _p(av),
                                  _p(b), ctypes.c_int64(b.shape[1]), _p(c), ctypes.c_int64(c.shape[1]),
                                  *_i64(tm, tk, tn), _p(rows_a), ctypes.c_int64(nr))
    return c


def dmatrix_sum(x, tm, tn):
    """DMatrix::sum in the reference's order (FP32 sequential), plus the
    FP64 sum and the sum of magnitudes: (f32_sum, f64_sum, abs_sum)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.zeros(3, np.float64)
    lib().oracle_dsum_f32(*_i64(x.shape[0], x.shape[1], tm, tn), _p(x), _p(out))
    return np.float32(out[0]), float(out[1]), float(out[2])


def binary_op(a, b_dense, op):
    """SPMatrix::binary_op_inplace (SPMatrix.hpp:571-616): every stored
    entry a(i, j) becomes fn(a(i, j), b(i, j)); one IEEE rounding per
    operation for FP32, wrapping for int32.  Returns the new values."""
    rows = np.repeat(np.arange(a.m), np.diff(a.row_ptr.astype(np.int64)))
    bv = np.asarray(b_dense)[rows, a.col_ind]
    av = np.asarray(a.vals)
    with np.errstate(all="ignore"):
        if op == "plus":
            return av + bv
        if op == "minus":
            return av - bv
        if op == "multiplies":
            return av * bv
        if op == "divides":
            if av.dtype == np.int32:  # C truncation; division by zero gives 0 here
                q = np.zeros_like(av)
                nz = bv != 0
                q[nz] = np.trunc(av[nz].astype(np.float64) / bv[nz]).astype(np.int64).astype(np.int32)
                return q
            return av / bv
        if op == "min":
            return np.where(bv < av, bv, av)
        if op == "max":
            return np.where(av < bv, bv, av)
        if op == "second":
            return bv.copy()
    raise ValueError(op)


def gather_value(v):
    """What SPMatrix::get (SPMatrix.hpp:516-546) makes of a stored value: it
    goes through SparseHashAccumulator, which adds it to a zero-initialised
    slot (SparseHashAccumulator.hpp:50-53), so -0.0 becomes +0.0 and a NaN
    comes back quiet; everything else is unchanged."""
    v = np.asarray(v)
    if v.dtype != np.float32:
        return v.copy()
    return np.float32(0) + v


def spmm_f64(a, b, rows=None):
    """A*B accumulated in double (all rows or the listed ones)."""
    rows_a, nr = _rows_arg(rows)
    nout = a.m if rows_a is None else nr
    c = np.zeros((nout, b.shape[1]), dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float32)
    av = np.ascontiguousarray(a.vals, dtype=np.float32)
    lib().oracle_spmm_tiled_f64(*_i64(a.m, a.n, b.shape[1]), _p(a.row_ptr), _p(a.col_ind), _p(av),
                                _p(b), ctypes.c_int64(b.shape[1]), _p(c), ctypes.c_int64(c.shape[1]),
                                _p(rows_a), ctypes.c_int64(nr))
    return c


def spmm_tiled_bf16(a, b_bf16, c0_bf16, tm, tk, tn, rows=None):
    """BF16-storage SpMM (uint16 bit patterns in and out), FP32 chain,
    one rounding per C row at the end."""
    rows_a, nr = _rows_arg(rows)
    c = np.array(c0_bf16, dtype=np.uint16, copy=True, order="C")
    b = np.ascontiguousarray(b_bf16, dtype=np.uint16)
    av = np.ascontiguousarray(a.vals, dtype=np.float32)
    lib().oracle_spmm_tiled_bf16(*_i64(a.m, a.n, b.shape[1]), _p(a.row_ptr), _p(a.col_ind), _p(av),
                                 _p(b), ctypes.c_int64(b.shape[1]), _p(c), ctypes.c_int64(c.shape[1]),
                                 *_i64(tm, tk, tn), _p(rows_a), ctypes.c_int64(nr))
    return c


def to_bf16(x):
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.empty(x.shape, dtype=np.uint16)
    lib().oracle_f32_to_bf16(_p(x), _p(y), ctypes.c_int64(x.size))
    return y


def bf16_to_f32(h):
    return (np.asarray(h, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


def num_threads() -> int:
    lib().oracle_num_threads.restype = ctypes.c_int
    return int(lib().oracle_num_threads())


# ---- the reference's own CPU binary --------------------------------------

def ref_available() -> bool:
    return os.path.exists(REF_BIN)


def run_ref(args, env=None, timeout=3600):
    """Run _ref/bcl_ref with ``args`` and return its JSON line."""
    e = dict(os.environ)
    if env:
        e.update(env)
    out = subprocess.run([REF_BIN] + [str(x) for x in args], check=True, capture_output=True,
                         text=True, env=e, timeout=timeout)
    for line in out.stdout.splitlines()[::-1]:
        line = line.strip()
        if line.startswith("{"):
            return json.loads(line)
    raise RuntimeError(f"bcl_ref printed no result: {out.stdout!r} {out.stderr!r}")


def ref_spgemm(a, b, tm, tk, tn, mode="f32", warmup=0, reps=1, want_output=True, workdir=None):
    """Reference BCL::gemm(SPMatrix, SPMatrix, SPMatrix&) on A, B; returns
    (result CSR or None, timing dict)."""
    from bcl_b200 import gen

    with tempfile.TemporaryDirectory(dir=workdir) as d:
        fa, fb, fc = (os.path.join(d, x + ".binary") for x in "abc")
        gen.write_binary(fa, a)
        gen.write_binary(fb, b)
        res = run_ref(["spgemm", fa, fb, tm, tk, tn, mode, fc if want_output else "-", warmup, reps])
        c = gen.read_binary(fc, np.float32 if mode == "f32" else np.int32) if want_output else None
    return c, res


def ref_spmm(a, b, tm, tk, tn, warmup=0, reps=1, want_output=True, workdir=None):
    """Reference BCL::gemm(SPMatrix, DMatrix, DMatrix&) with C = 0 first."""
    from bcl_b200 import gen

    with tempfile.TemporaryDirectory(dir=workdir) as d:
        fa, fb, fc = os.path.join(d, "a.binary"), os.path.join(d, "b.dense"), os.path.join(d, "c.dense")
        gen.write_binary(fa, a)
        gen.write_dense(fb, b)
        res = run_ref(["spmm", fa, fb, tm, tk, tn, fc if want_output else "-", warmup, reps])
        c = gen.read_dense(fc) if want_output else None
    return c, res


def ref_mp_available() -> bool:
    return os.path.exists(REF_MP_BIN)


def _shared_dir():
    """A tmpfs directory for the ranks' shared windows when there is one."""
    return "/dev/shm" if os.path.isdir("/dev/shm") and os.access("/dev/shm", os.W_OK) else None


def run_ref_mp(args, nranks, timeout=3600, threads=1, binary=None):
    """Run _ref/bcl_ref_mp (or another program built over ref_stubs_mp/) as
    `nranks` ranks (one process each, `threads` OpenMP threads each) on
    ``args`` and return rank 0's JSON line.  The ranks share a fresh
    directory for their windows; when one rank fails or the time runs out,
    the others are stopped."""
    with tempfile.TemporaryDirectory(dir=_shared_dir(), prefix="bclx_ranks_") as d:
        procs, logs = [], []
        try:
            for r in range(nranks):
                env = dict(os.environ, BCLX_STUB_RANK=str(r), BCLX_STUB_SIZE=str(nranks), BCLX_STUB_DIR=d,
                           BCLX_STUB_TIMEOUT=str(int(min(timeout, 900))), OMP_NUM_THREADS=str(threads))
                out = open(os.path.join(d, f"out{r}"), "w+")
                err = open(os.path.join(d, f"err{r}"), "w+")
                logs.append((out, err))
                procs.append(subprocess.Popen([binary or REF_MP_BIN] + [str(x) for x in args], stdout=out,
                                              stderr=err, env=env))
            deadline = time.time() + timeout
            while True:
                states = [p.poll() for p in procs]
                if all(s == 0 for s in states) or any(s not in (None, 0) for s in states):
                    break
                if time.time() > deadline:
                    raise RuntimeError(f"bcl_ref_mp: {nranks} ranks did not finish in {timeout} s")
                time.sleep(0.005)
            for r, (p, (out, err)) in enumerate(zip(procs, logs)):
                if p.returncode not in (None, 0):
                    err.seek(0)
                    raise RuntimeError(f"bcl_ref_mp rank {r} exited {p.returncode}: {err.read()[-400:]}")
            out = logs[0][0]
            out.seek(0)
            for line in out.read().splitlines()[::-1]:
                if line.strip().startswith("{"):
                    return json.loads(line)
            raise RuntimeError("bcl_ref_mp printed no result")
        finally:  # no rank outlives the call
            for p in procs:
                if p.poll() is None:
                    p.kill()
                    p.wait()
            for out, err in logs:
                out.close()
                err.close()


def ref_spgemm_mp(a, b, tm, tk, tn, pgrid, mode="f32", warmup=0, reps=1, want_output=True, workdir=None,
                  threads=1):
    """The reference's distributed BCL::gemm(SPMatrix, SPMatrix, SPMatrix&)
    with A, B and C on a pm x pn process grid (pm * pn ranks); returns
    (result CSR gathered by rank 0, or None; rank 0's timing line)."""
    from bcl_b200 import gen

    pm, pn = pgrid
    with tempfile.TemporaryDirectory(dir=workdir) as d:
        fa, fb, fc = (os.path.join(d, x + ".binary") for x in "abc")
        gen.write_binary(fa, a)
        gen.write_binary(fb, b)
        res = run_ref_mp(["spgemm", fa, fb, tm, tk, tn, pm, pn, mode, fc if want_output else "-", warmup, reps],
                         pm * pn, threads=threads)
        c = gen.read_binary(fc, np.float32 if mode == "f32" else np.int32) if want_output else None
    return c, res


def ref_spmm_mp(a, b, tm, tk, tn, pgrid, warmup=0, reps=1, want_output=True, workdir=None, threads=1):
    """The reference's distributed BCL::gemm(SPMatrix, DMatrix, DMatrix&),
    C = 0 first, on a pm x pn process grid."""
    from bcl_b200 import gen

    pm, pn = pgrid
    with tempfile.TemporaryDirectory(dir=workdir) as d:
        fa, fb, fc = os.path.join(d, "a.binary"), os.path.join(d, "b.dense"), os.path.join(d, "c.dense")
        gen.write_binary(fa, a)
        gen.write_dense(fb, b)
        res = run_ref_mp(["spmm", fa, fb, tm, tk, tn, pm, pn, fc if want_output else "-", warmup, reps], pm * pn,
                         threads=threads)
        c = gen.read_dense(fc) if want_output else None
    return c, res


def ref_dot(a, b, mode="f32", workdir=None):
    """Reference CSRMatrix::dot (the local tile kernel) on whole matrices."""
    from bcl_b200 import gen

    with tempfile.TemporaryDirectory(dir=workdir) as d:
        fa, fb, fc = (os.path.join(d, x + ".binary") for x in "abc")
        gen.write_binary(fa, a)
        gen.write_binary(fb, b)
        res = run_ref(["dot", fa, fb, mode, fc])
        c = gen.read_binary(fc, np.float32 if mode == "f32" else np.int32)
    return c, res


def ref_accumulate(parts, mode="f32", workdir=None):
    """Reference SparseHashAccumulator: push ``parts`` in order, get_matrix."""
    from bcl_b200 import gen

    with tempfile.TemporaryDirectory(dir=workdir) as d:
        files = []
        for i, p in enumerate(parts):
            f = os.path.join(d, f"p{i}.binary")
            gen.write_binary(f, p)
            files.append(f)
        fc = os.path.join(d, "c.binary")
        res = run_ref(["accumulate", mode, fc] + files)
        c = gen.read_binary(fc, np.float32 if mode == "f32" else np.int32)
    return c, res
