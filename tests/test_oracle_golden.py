"""The C restatement (oracle/oracle.c) against the golden fixtures made by the
reference's own CPU code (tests/golden/make_golden.py), and against the
reference binary itself where it is present.  Everything here is bit-exact:
structure (row_ptr, sorted col_ind, explicit zeros kept) and values."""
import glob
import os

import numpy as np
import pytest

from bcl_b200 import gen
from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_csr(d, prefix):
    m, n = (int(x) for x in d[f"{prefix}_shape"])
    return gen.CSR(m, n, d[f"{prefix}_row_ptr"], d[f"{prefix}_col_ind"], d[f"{prefix}_vals"])


def same_bits(x, y):
    x, y = np.asarray(x), np.asarray(y)
    return x.shape == y.shape and np.array_equal(x.view(np.uint32) if x.dtype == np.float32 else x,
                                                 y.view(np.uint32) if y.dtype == np.float32 else y)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "spgemm_*.npz"))), ids=os.path.basename)
def test_oracle_spgemm_matches_reference(path):
    d = np.load(path)
    a, b, c = load_csr(d, "a"), load_csr(d, "b"), load_csr(d, "c")
    mode = str(d["mode"])
    rp, ci, cv = O.gemm_tiled(a, b, *[int(t) for t in d["tiles"]], mode=mode)
    assert np.array_equal(rp, c.row_ptr.astype(np.int64))
    assert np.array_equal(ci, c.col_ind)
    assert same_bits(cv, c.vals)


def test_oracle_spgemm_without_fma_differs():
    """The reference build contracts `c += a*b` into a fused multiply-add;
    the separately rounded form does not reproduce it."""
    d = np.load(os.path.join(GOLD, "spgemm_rmat10_f32_t256.npz"))
    a, c = load_csr(d, "a"), load_csr(d, "c")
    _, _, cv = O.gemm_tiled(a, a, 256, 256, 256, mode="f32", use_fma=False)
    assert not same_bits(cv, c.vals)
    np.testing.assert_allclose(cv, c.vals, rtol=1e-3, atol=1e-4)


def test_oracle_dot_matches_reference():
    d = np.load(os.path.join(GOLD, "dot_rmat9_f32.npz"))
    a, c = load_csr(d, "a"), load_csr(d, "c")
    rp, ci, cv = O.spgemm_local(a, a)
    assert np.array_equal(rp, c.row_ptr.astype(np.int64))
    assert np.array_equal(ci, c.col_ind)
    assert same_bits(cv, c.vals)


@pytest.mark.parametrize("name,mode", [("accumulate_rmat9x4_f32", "f32"), ("accumulate_rmat8x3_i32", "i32")])
def test_oracle_accumulate_matches_reference(name, mode):
    d = np.load(os.path.join(GOLD, name + ".npz"))
    parts = []
    i = 0
    while f"p{i}_shape" in d:
        parts.append(load_csr(d, f"p{i}"))
        i += 1
    c = load_csr(d, "c")
    rp, ci, cv = O.accumulate(parts, mode=mode)
    assert np.array_equal(rp, c.row_ptr.astype(np.int64))
    assert np.array_equal(ci, c.col_ind)
    assert same_bits(cv, c.vals)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "spmm_*.npz"))), ids=os.path.basename)
def test_oracle_spmm_matches_reference(path):
    d = np.load(path)
    a = load_csr(d, "a")
    tiles = [int(t) for t in d["tiles"]]
    c = O.spmm_tiled(a, d["b"], np.zeros_like(d["c"]), *tiles)
    assert same_bits(c, d["c"])


def test_oracle_f64_close_to_f32():
    d = np.load(os.path.join(GOLD, "spgemm_rmat9_f32_ragged.npz"))
    a, c = load_csr(d, "a"), load_csr(d, "c")
    _, _, c64 = O.gemm_tiled(a, a, 100, 70, 130, mode="f64")
    np.testing.assert_allclose(c.vals, c64, rtol=1e-4, atol=1e-5)


@pytest.mark.skipif(not O.ref_available(), reason="reference binary not built")
def test_oracle_matches_live_reference_fresh_seed():
    """A fresh input not in the fixtures: ragged tiles, FP32 and int32."""
    for mode in ("f32", "i32"):
        a = gen.rmat(9, seed=99, value_type=mode)
        c, _ = O.ref_spgemm(a, a, 96, 160, 200, mode=mode)
        rp, ci, cv = O.gemm_tiled(a, a, 96, 160, 200, mode=mode)
        assert np.array_equal(rp, c.row_ptr.astype(np.int64))
        assert np.array_equal(ci, c.col_ind)
        assert same_bits(cv, c.vals)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "rowwise_*.npz"))), ids=os.path.basename)
def test_oracle_rowwise_matches_reference(path):
    """rowwise_gemm, cached_rowwise_gemm and batched_rowwise_gemm all equal
    the ascending-stage restatement, bit for bit."""
    d = np.load(path)
    a = load_csr(d, "a")
    tiles = [int(t) for t in d["tiles"]]
    c = O.spmm_rowwise(a, d["b"], np.zeros_like(d["c_plain"]), *tiles)
    for variant in ("plain", "cached", "batched"):
        assert same_bits(c, d[f"c_{variant}"]), variant


def test_oracle_rowwise_order_differs_from_summa():
    """On a grid with more than one stage the ascending order is a different
    FP32 sum from the SUMMA loop's rotated order (so the two are told apart)."""
    d = np.load(os.path.join(GOLD, "rowwise_rmat10_n64_t256.npz"))
    a = load_csr(d, "a")
    tiles = [int(t) for t in d["tiles"]]
    c = O.spmm_tiled(a, d["b"], np.zeros_like(d["c_plain"]), *tiles)
    assert not same_bits(c, d["c_plain"])


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "dsum_*.npz"))), ids=os.path.basename)
def test_oracle_dsum_matches_reference(path):
    d = np.load(path)
    s32, s64, sabs = O.dmatrix_sum(d["x"], *[int(t) for t in d["tiles"]])
    assert np.array_equal(np.array([s32], np.float32).view(np.uint32), d["bits"].reshape(1))
    # the sequential FP32 sum is within its rounding bound of the FP64 sum
    n = d["x"].size
    assert abs(float(s32) - s64) <= (n - 1) * 2.0 ** -24 * sabs


@pytest.mark.parametrize("dt", ["f32", "i32"])
def test_oracle_binary_op_matches_reference(dt):
    d = np.load(os.path.join(GOLD, f"binop_sparse120x90_{dt}.npz"))
    a = load_csr(d, "a")
    for key in d.files:
        if key.startswith("vals_"):
            op = key[5:]
            got = O.binary_op(a, d["b"], op)
            assert same_bits(got, d[key]), op
            # SPMatrix::get adds every value to 0: -0 comes back as +0
            assert same_bits(O.gather_value(got), d["get_" + op]), op
