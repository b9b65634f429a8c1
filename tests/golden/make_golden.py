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


if __name__ == "__main__":
    main()
