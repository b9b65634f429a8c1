"""The input path: the reference's MatrixMarket reader (matrix_io.hpp:218-356,
CSRMatrix.hpp:370-410) restated in bcl_b200.gen, checked against what the
reference's own reader made of the same files (tests/golden/mm_*), and the
host restatement of the tile slicing checked against the reference's
SPMatrix(fname, BlockCustom) tiles (tests/golden/tiles_*)."""
import glob
import os

import numpy as np
import pytest

from bcl_b200 import gen

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "mm_*.mtx"))), ids=os.path.basename)
def test_matrix_market_matches_reference_reader(path):
    d = np.load(path[:-4] + ".npz")
    vt = np.float32 if str(d["dtype"]) == "f32" else np.int32
    a = gen.read_matrix(path, vt)
    assert (a.m, a.n) == tuple(d["c_shape"])
    assert np.array_equal(a.row_ptr, d["c_row_ptr"])
    assert np.array_equal(a.col_ind, d["c_col_ind"])
    assert np.array_equal(a.vals, d["c_vals"])


def test_matrix_market_errors(tmp_path):
    p = tmp_path / "x.mtx"
    p.write_text("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n")
    with pytest.raises(RuntimeError):
        gen.read_matrix_market(str(p))
    p.write_text("%%MatrixMarket matrix coordinate real hermitian\n2 2 1\n1 1 1\n")
    with pytest.raises(RuntimeError):
        gen.read_matrix_market(str(p))
    p.write_text("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1\n")
    with pytest.raises(RuntimeError):
        gen.read_matrix_market(str(p))
    p.write_text("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 1\n2 2 1\n")
    with pytest.raises(RuntimeError):
        gen.read_matrix_market(str(p))
    with pytest.raises(RuntimeError):
        gen.read_matrix(str(tmp_path / "x.csv"))


def test_matrix_market_write_read(tmp_path):
    a = gen.rmat(7, seed=5)
    p = str(tmp_path / "a.mtx")
    gen.write_matrix_market(p, a)
    assert open(p).readline().startswith("%%MatrixMarket matrix coordinate integer general")
    b = gen.read_matrix_market(p)
    assert np.array_equal(a.row_ptr, b.row_ptr) and np.array_equal(a.col_ind, b.col_ind)
    assert np.allclose(a.vals, b.vals, atol=5e-7)  # values are written with %f


def tile_records(d):
    """Golden tiles as a list of (row_ptr, col_ind, vals)."""
    out, rp0, nz0 = [], 0, 0
    for rows, nnz in zip(d["tile_rows"], d["tile_nnz"]):
        out.append((d["row_ptr"][rp0:rp0 + rows + 1], d["col_ind"][nz0:nz0 + nnz], d["vals"][nz0:nz0 + nnz]))
        rp0 += rows + 1
        nz0 += nnz
    return out


def load_a(d):
    m, n = d["a_shape"]
    return gen.CSR(int(m), int(n), d["a_row_ptr"], d["a_col_ind"], d["a_vals"])


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "tiles_*.npz"))), ids=os.path.basename)
def test_host_slicing_matches_reference_tiles(path):
    from bcl_b200.containers import split_tiles
    d = np.load(path)
    a = load_a(d)
    tm, tn = (int(x) for x in d["tiles"])
    trp, toff, ci, v = split_tiles(a, tm, tn)
    for t, (rp, c, x) in enumerate(tile_records(d)):
        rows = rp.size - 1
        assert np.array_equal(trp[t, : rows + 1], rp)
        assert np.array_equal(ci[toff[t]:toff[t + 1]], c)
        assert np.array_equal(v[toff[t]:toff[t + 1]], x)
