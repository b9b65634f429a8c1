"""Host-side tiling and container bookkeeping (no GPU): cutting a CSR into a
tile grid reproduces SPMatrix's per-tile slices (SPMatrix.hpp:211-271 via
CSRMatrix::get_slice_impl_, CSRMatrix.hpp:238-276), including ragged edges
and empty tiles."""
import numpy as np
import pytest

from bcl_b200 import gen
from bcl_b200.containers import BlockCustom, split_tiles


def naive_slice(a, i0, i1, j0, j1):
    rp, ci, v = [0], [], []
    for r in range(i0, min(i1, a.m)):
        for p in range(a.row_ptr[r], a.row_ptr[r + 1]):
            if j0 <= a.col_ind[p] < j1:
                ci.append(a.col_ind[p] - j0)
                v.append(a.vals[p])
        rp.append(len(ci))
    return np.array(rp), np.array(ci, dtype=np.int64), np.array(v)


@pytest.mark.parametrize("tm,tn", [(64, 64), (100, 37), (512, 512), (7, 300)])
def test_split_tiles_matches_slices(tm, tn):
    a = gen.rmat(9, seed=3)
    trp, toff, ci, v = split_tiles(a, tm, tn)
    gm, gn = -(-a.m // tm), -(-a.n // tn)
    assert trp.shape == (gm * gn, tm + 1) and toff.shape == (gm * gn + 1,)
    assert toff[-1] == a.nnz
    for i in range(gm):
        for j in range(gn):
            t = i * gn + j
            rp, c, vv = naive_slice(a, i * tm, (i + 1) * tm, j * tn, (j + 1) * tn)
            rows = len(rp) - 1
            assert np.array_equal(trp[t, : rows + 1], rp)
            assert np.all(trp[t, rows + 1:] == rp[-1])
            assert np.array_equal(ci[toff[t]:toff[t + 1]], c)
            assert np.array_equal(v[toff[t]:toff[t + 1]], vv)


def test_blocking_seed_divides():
    assert BlockCustom((0, 0), (4, 2)).seed(100, 30) == (25, 15)
    assert BlockCustom((64, 32)).seed(100, 30) == (64, 32)
    with pytest.raises(ValueError):
        BlockCustom((-1, 5)).seed(10, 10)


def test_generators_shapes_and_sortedness():
    for a in (gen.rmat(8, seed=1), gen.erdos_renyi(300, 9, seed=2), gen.stencil27(5)):
        rp, ci = a.row_ptr.astype(np.int64), a.col_ind
        assert rp[0] == 0 and np.all(np.diff(rp) >= 0) and rp[-1] == ci.size
        for r in range(a.m):
            seg = ci[rp[r]:rp[r + 1]]
            assert np.all(np.diff(seg) > 0)
    e = gen.erdos_renyi(300, 9, seed=2)
    assert np.all(e.row_nnz() == 9)
    s = gen.stencil27(6)
    assert s.nnz == (3 * 6 - 2) ** 3
    assert s.row_nnz().max() == 27
    # closed form of the stencil square's nnz: (5g-6)^3
    from oracle import oracle as O
    assert int(O.spgemm_count(s, s).sum()) == (5 * 6 - 6) ** 3


def test_binary_roundtrip(tmp_path):
    a = gen.rmat(7, seed=5, value_type="i32")
    p = tmp_path / "a.binary"
    gen.write_binary(str(p), a)
    b = gen.read_binary(str(p), np.int32)
    assert (b.m, b.n, b.nnz) == (a.m, a.n, a.nnz)
    assert np.array_equal(b.row_ptr, a.row_ptr) and np.array_equal(b.col_ind, a.col_ind)
    assert np.array_equal(b.vals, a.vals)


@pytest.mark.parametrize("m,n,tm,tn", [(10, 7, 4, 3), (64, 128, 64, 128), (37, 5, 8, 8)])
def test_dmatrix_layout_on_host_tensors(m, n, tm, tn):
    """DMatrix bookkeeping with host tensors: padded row-major tiles
    (DMatrix.hpp:55-95), set_matrix / get_matrix round trip, edge tile
    shapes, get_tile (the padded tile), operator=(value) over the padding."""
    import torch
    from bcl_b200.containers import DMatrix
    gm, gn = -(-m // tm), -(-n // tn)
    d = DMatrix(m, n, tm, tn, torch.zeros((gm * gn, tm, tn), dtype=torch.float32))
    full = torch.arange(m * n, dtype=torch.float32).reshape(m, n)
    d.set_matrix(full)
    assert torch.equal(d.get_matrix(), full)
    assert d.grid_shape() == (gm, gn) and d.tile_size() == tm * tn and d.tile_rank((0, 0)) == 0
    for i in range(gm):
        for j in range(gn):
            th, tw = d.tile_shape((i, j))
            assert (th, tw) == (min(tm, m - i * tm), min(tn, n - j * tn))
            t = d.get_tile((i, j)).reshape(tm, tn)
            assert torch.equal(t[:th, :tw], full[i * tm:i * tm + th, j * tn:j * tn + tw])
            assert torch.all(t[th:, :] == 0) and torch.all(t[:, tw:] == 0)  # padding
    d.fill_(2.5)
    assert torch.all(d.tiles == 2.5)


@pytest.mark.parametrize("tm,tn", [(100, 37), (64, 512)])
def test_spmatrix_bookkeeping_on_host_tensors(tm, tn):
    """SPMatrix bookkeeping with host tensors (no kernels): get_tile /
    arget_tile against direct slices, tile_nnz, and a matrix rebuilt tile by
    tile with assign_tile (SPMatrix.hpp:277-308, 476-514) gathered back."""
    import torch
    from bcl_b200.containers import SPMatrix
    a = gen.rmat(9, seed=4)
    trp, toff, ci, v = split_tiles(a, tm, tn)
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x))  # noqa: E731
    A = SPMatrix(a.m, a.n, tm, tn, np.float32, 0, t(trp.astype(np.int32)), t(toff.astype(np.int64)),
                 t(ci.astype(np.int32)), t(v.astype(np.float32)))
    gm, gn = A.grid_shape()
    E = SPMatrix(a.m, a.n, tm, tn, np.float32, 0, torch.zeros((gm * gn, tm + 1), dtype=torch.int32),
                 torch.zeros(gm * gn + 1, dtype=torch.int64), torch.zeros(0, dtype=torch.int32),
                 torch.zeros(0, dtype=torch.float32))
    for i in range(gm):
        for j in range(gn):
            tile = A.get_tile((i, j))
            rp, c, vals = naive_slice(a, i * tm, (i + 1) * tm, j * tn, (j + 1) * tn)
            assert np.array_equal(tile.row_ptr, rp) and np.array_equal(tile.col_ind, c)
            assert np.array_equal(tile.vals, vals) and A.tile_nnz((i, j)) == len(c)
            fut = A.arget_tile((i, j))
            assert np.array_equal(fut.get().col_ind, tile.col_ind)
            E.assign_tile((i, j), tile)
    g = E.get_host_gather()
    assert np.array_equal(g.row_ptr, a.row_ptr) and np.array_equal(g.col_ind, a.col_ind)
    assert np.array_equal(g.vals, a.vals) and E.nnz() == a.nnz
