"""Generate the golden fixtures for the sparse tile multiply by running the
reference's own CPU implementation (oracle/_ref/bcl_ref, compiled from the
unmodified reference headers with oracle/Makefile).

Each fixture is an .npz holding the inputs and the reference's outputs:

* ``spgemm_*``: BCL::gemm(SPMatrix, SPMatrix, SPMatrix&) on a tile grid
  (bcl/containers/algorithms/spgemm.hpp:182-242), result gathered with
  SPMatrix::get().
* ``dot_*``: CSRMatrix::dot, the local tile kernel (spgemm.hpp:41-76).
* ``accumulate_*``: SparseHashAccumulator::get_matrix over partials pushed in
  order (SparseHashAccumulator.hpp:101-182).
* ``spmm_*``: BCL::gemm(SPMatrix, DMatrix, DMatrix&) with C = 0 first
  (spgemm.hpp:153-179).
* ``mm_*.mtx`` / ``mm_*.npz``: MatrixMarket files written here (duplicates,
  comments, empty rows, symmetric, pattern, integer) and the CSR matrix the
  reference's reader makes of each (CSRMatrix(fname), matrix_io.hpp:218-356).
* ``tiles_*``: every tile of SPMatrix(fname, BlockCustom) (the reference's
  slicing, SPMatrix.hpp:194-271), row-major over the grid.
* ``rowwise_*``: rowwise_gemm / cached_rowwise_gemm / batched_rowwise_gemm
  (experimental_gemm.hpp:83-214), C = 0 first.
* ``dsum_*``: DMatrix::sum (DMatrix.hpp:537-554), the FP32 bits it returns.
* ``binop_*``: SPMatrix::binary_op_inplace (SPMatrix.hpp:571-616) with the
  standard functors, on one tile (the reference's loops bound i and j by
  grid_shape()[i] and grid_shape()[j], in range only for a 1x1 grid).

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from bcl_b200 import gen  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def csr_dict(prefix, m):
    return {f"{prefix}_shape": np.array([m.m, m.n], np.int64), f"{prefix}_row_ptr": m.row_ptr,
            f"{prefix}_col_ind": m.col_ind, f"{prefix}_vals": m.vals}


def sparse_with_empty(m, n, seed, value_type="f32"):
    """Random sparse matrix where about half the rows and columns are empty."""
    rng = np.random.default_rng(seed)
    live_rows = rng.choice(m, m // 2, replace=False)
    live_cols = rng.choice(n, n // 2, replace=False)
    r = rng.choice(live_rows, 6 * m)
    c = rng.choice(live_cols, 6 * m)
    keys = np.unique(r.astype(np.int64) * n + c)
    vals = (rng.uniform(-1, 1, keys.size).astype(np.float32) if value_type == "f32"
            else rng.integers(-8, 9, keys.size).astype(np.int32))
    return gen._csr_from_sorted_keys(keys, m, n, vals)


def rect(m, k, seed, per_row):
    rng = np.random.default_rng(seed)
    keys = np.unique(np.repeat(np.arange(m, dtype=np.int64), per_row) * k
                     + rng.integers(0, k, m * per_row))
    return gen._csr_from_sorted_keys(keys, m, k, rng.uniform(-1, 1, keys.size).astype(np.float32))


def spgemm_case(name, a, b, tiles, mode):
    c, _ = O.ref_spgemm(a, b, *tiles, mode=mode)
    d = {"tiles": np.array(tiles, np.int64), "mode": np.array(mode)}
    d.update(csr_dict("a", a))
    d.update(csr_dict("b", b))
    d.update(csr_dict("c", c))
    np.savez_compressed(os.path.join(OUT, f"spgemm_{name}.npz"), **d)
    print(f"spgemm_{name}: nnz(C)={c.nnz}")


def main():
    # SpGEMM through the SUMMA tile loop.
    a = gen.rmat(10, seed=11)
    spgemm_case("rmat10_f32_t256", a, a, (256, 256, 256), "f32")
    ai = gen.rmat(10, seed=12, value_type="i32")
    spgemm_case("rmat10_i32_t256", ai, ai, (256, 256, 256), "i32")
    a9 = gen.rmat(9, seed=13)
    spgemm_case("rmat9_f32_ragged", a9, a9, (100, 70, 130), "f32")
    er = gen.erdos_renyi(600, 8, seed=14)
    spgemm_case("er600_f32_t128", er, er, (128, 128, 128), "f32")
    ea = sparse_with_empty(300, 200, seed=15)
    eb = sparse_with_empty(200, 350, seed=16)
    spgemm_case("empty_rect_f32", ea, eb, (64, 50, 90), "f32")
    st = gen.stencil27(8)
    spgemm_case("stencil8_f32_t128", st, st, (128, 128, 128), "f32")
    ra, rb = rect(257, 129, 17, 5), rect(129, 383, 18, 9)
    spgemm_case("rect_f32_one_tile", ra, rb, (512, 512, 512), "f32")

    # Local tile kernel (CSRMatrix::dot).
    c, _ = O.ref_dot(a9, a9, mode="f32")
    d = csr_dict("a", a9)
    d.update(csr_dict("c", c))
    np.savez_compressed(os.path.join(OUT, "dot_rmat9_f32.npz"), **d)
    print(f"dot_rmat9_f32: nnz={c.nnz}")

    # Tile accumulation of partials in push order.
    parts = [gen.rmat(9, seed=20 + s) for s in range(4)]
    c, _ = O.ref_accumulate(parts, mode="f32")
    d = {}
    for i, p in enumerate(parts):
        d.update(csr_dict(f"p{i}", p))
    d.update(csr_dict("c", c))
    np.savez_compressed(os.path.join(OUT, "accumulate_rmat9x4_f32.npz"), **d)
    parts_i = [gen.rmat(8, seed=30 + s, value_type="i32") for s in range(3)]
    c, _ = O.ref_accumulate(parts_i, mode="i32")
    d = {}
    for i, p in enumerate(parts_i):
        d.update(csr_dict(f"p{i}", p))
    d.update(csr_dict("c", c))
    np.savez_compressed(os.path.join(OUT, "accumulate_rmat8x3_i32.npz"), **d)
    print("accumulate fixtures written")

    # SpMM through the SUMMA tile loop (C zeroed first).
    for name, am, bd, tiles in [
        ("er1024_n64_t256", gen.erdos_renyi(1024, 16, seed=40), gen.dense(1024, 64, seed=41), (256, 256, 32)),
        ("rmat10_n128_t256", gen.rmat(10, seed=42), gen.dense(1024, 128, seed=43), (256, 256, 128)),
        ("empty_rect_n40_ragged", sparse_with_empty(300, 200, seed=44), gen.dense(200, 40, seed=45, dist="normal"),
         (70, 60, 24)),
    ]:
        c, _ = O.ref_spmm(am, bd, *tiles)
        d = {"tiles": np.array(tiles, np.int64), "b": bd, "c": c}
        d.update(csr_dict("a", am))
        np.savez_compressed(os.path.join(OUT, f"spmm_{name}.npz"), **d)
        print(f"spmm_{name}: C {c.shape}")


def _mtx_lines(rng, m, n, count, field, symmetric):
    i = rng.integers(0, m, count)
    j = rng.integers(0, n, count)
    if symmetric:
        i, j = np.maximum(i, j), np.minimum(i, j)
    # about 10 % repeat an earlier index with another value
    rep_ = rng.random(count) < 0.1
    src = rng.integers(0, count, count)
    i = np.where(rep_, i[src], i)
    j = np.where(rep_, j[src], j)
    lines = []
    for a, b in zip(i, j):
        if field == "pattern":
            lines.append(f"{a + 1} {b + 1}")
        elif field == "integer":
            lines.append(f"{a + 1} {b + 1} {int(rng.integers(-9, 10))}")
        else:
            lines.append(f"{a + 1} {b + 1} {rng.uniform(-2, 2):.6g}")
    return lines


def io_fixtures():
    import subprocess
    import tempfile
    rng = np.random.default_rng(60)
    cases = [("general_real_dups", 60, 45, 300, "real", "general", "f32"),
             ("symmetric_real", 50, 50, 200, "real", "symmetric", "f32"),
             ("pattern_general", 40, 70, 150, "pattern", "general", "f32"),
             ("integer_general", 30, 30, 90, "integer", "general", "i32")]
    for name, m, n, cnt, field, sym, dt in cases:
        lines = _mtx_lines(rng, m, n, cnt, field, sym == "symmetric")
        path = os.path.join(OUT, f"mm_{name}.mtx")
        with open(path, "w") as f:
            f.write(f"%%MatrixMarket matrix coordinate {field} {sym}\n% written by make_golden.py\n%\n")
            f.write(f"{m} {n} {len(lines)}\n")
            f.write("\n".join(lines) + "\n")
        with tempfile.TemporaryDirectory() as d:
            out = os.path.join(d, "a.binary")
            subprocess.run([O.REF_BIN, "mmread", path, dt, out], check=True)
            c = gen.read_binary(out, np.float32 if dt == "f32" else np.int32)
        np.savez_compressed(os.path.join(OUT, f"mm_{name}.npz"), dtype=np.array(dt), **csr_dict("c", c))
        print(f"mm_{name}: nnz={c.nnz}")
    for name, a, tiles in [("rmat9_ragged", gen.rmat(9, seed=61), (100, 70)),
                           ("empty_rect", sparse_with_empty(300, 200, seed=62), (64, 50)),
                           ("stencil6", gen.stencil27(6), (50, 128))]:
        dt = "f32" if a.vals.dtype == np.float32 else "i32"
        vt = np.float32 if dt == "f32" else np.int32
        with tempfile.TemporaryDirectory() as d:
            fa, ft = os.path.join(d, "a.binary"), os.path.join(d, "t.bin")
            gen.write_binary(fa, a)
            subprocess.run([O.REF_BIN, "tiles", fa, str(tiles[0]), str(tiles[1]), dt, ft], check=True)
            raw = open(ft, "rb").read()
        rps, cis, vs, nnzs = [], [], [], []
        pos = 0
        while pos < len(raw):
            tm_, tn_, nz = np.frombuffer(raw, np.uint64, 3, pos).astype(np.int64)
            pos += 24
            vs.append(np.frombuffer(raw, vt, nz, pos)); pos += 4 * nz
            cis.append(np.frombuffer(raw, np.int32, nz, pos)); pos += 4 * nz
            rps.append(np.frombuffer(raw, np.int32, tm_ + 1, pos)); pos += 4 * (tm_ + 1)
            nnzs.append(nz)
        d = csr_dict("a", a)
        d.update({"tiles": np.array(tiles, np.int64), "tile_nnz": np.array(nnzs, np.int64),
                  "tile_rows": np.array([r.size - 1 for r in rps], np.int64),
                  "row_ptr": np.concatenate(rps), "col_ind": np.concatenate(cis),
                  "vals": np.concatenate(vs)})
        np.savez_compressed(os.path.join(OUT, f"tiles_{name}.npz"), **d)
        print(f"tiles_{name}: {len(nnzs)} tiles")


def container_fixtures():
    import subprocess
    import tempfile
    for name, am, bd, tiles in [
        ("rmat10_n64_t256", gen.rmat(10, seed=70), gen.dense(1024, 64, seed=71), (256, 256, 64)),
        ("empty_rect_n24_ragged", sparse_with_empty(300, 200, seed=72), gen.dense(200, 24, seed=73, dist="normal"),
         (70, 60, 24)),
    ]:
        d = {"tiles": np.array(tiles, np.int64), "b": bd}
        d.update(csr_dict("a", am))
        for variant in ("plain", "cached", "batched"):
            with tempfile.TemporaryDirectory() as td:
                fa, fb, fc = (os.path.join(td, x) for x in ("a.binary", "b.dense", "c.dense"))
                gen.write_binary(fa, am)
                gen.write_dense(fb, bd)
                subprocess.run([O.REF_BIN, "rowwise", variant, fa, fb] + [str(t) for t in tiles] + [fc],
                               check=True, capture_output=True)
                d[f"c_{variant}"] = gen.read_dense(fc)
        np.savez_compressed(os.path.join(OUT, f"rowwise_{name}.npz"), **d)
        print(f"rowwise_{name}")
    import json
    for name, x, tiles in [("u300x70_t64x32", gen.dense(300, 70, seed=74), (64, 32)),
                           ("n1000x257_t128x100", gen.dense(1000, 257, seed=75, dist="normal") * 1e3, (128, 100))]:
        with tempfile.TemporaryDirectory() as td:
            fb = os.path.join(td, "b.dense")
            gen.write_dense(fb, x.astype(np.float32))
            out = subprocess.run([O.REF_BIN, "dsum", fb, str(tiles[0]), str(tiles[1])], check=True,
                                 capture_output=True, text=True).stdout
        res = json.loads([ln for ln in out.splitlines() if ln.startswith("{")][-1])
        np.savez_compressed(os.path.join(OUT, f"dsum_{name}.npz"), x=x.astype(np.float32),
                            tiles=np.array(tiles, np.int64), bits=np.array(res["bits"], np.uint32))
        print(f"dsum_{name}: {res['sum']}")
    rng = np.random.default_rng(76)
    for dt in ("f32", "i32"):
        am = sparse_with_empty(120, 90, seed=77, value_type=dt)
        if dt == "f32":
            bd = rng.uniform(-2, 2, (120, 90)).astype(np.float32)
            bd[rng.random(bd.shape) < 0.05] = 0.0
        else:
            bd = rng.integers(-5, 6, (120, 90)).astype(np.int32)
        d = {"b": bd}
        d.update(csr_dict("a", am))
        for op in ("plus", "minus", "multiplies", "divides", "min", "max", "second"):
            with tempfile.TemporaryDirectory() as td:
                fa, fb, fc = (os.path.join(td, x) for x in ("a.binary", "b.dense", "c.binary"))
                gen.write_binary(fa, am)
                gen.write_dense(fb, bd)
                if dt == "i32" and op == "divides":
                    continue  # integer division by zero is undefined in the reference
                subprocess.run([O.REF_BIN, "binop", op, fa, fb, dt, fc], check=True, capture_output=True)
                c = gen.read_binary(fc, np.float32 if dt == "f32" else np.int32)
                cg = gen.read_binary(fc + ".get", np.float32 if dt == "f32" else np.int32)
            d[f"vals_{op}"] = c.vals
            d[f"get_{op}"] = cg.vals
        np.savez_compressed(os.path.join(OUT, f"binop_sparse120x90_{dt}.npz"), **d)
        print(f"binop_sparse120x90_{dt}")


if __name__ == "__main__":
    if sys.argv[1:] == ["io"]:
        io_fixtures()
    elif sys.argv[1:] == ["containers"]:
        container_fixtures()
    else:
        main()
        io_fixtures()
        container_fixtures()
