"""GPU parity of the device-side slicing into tiles (bclx_csr_to_tiles, the
SPMatrix(fname, blocking) constructor's job) and of the gather back to one
CSR matrix (bclx_tiles_to_csr, SPMatrix::get): bit-exact against the
reference's own tiles (tests/golden/tiles_*) and against the host slicing,
round trips, empty and ragged cases, and the rejection of rows whose columns
are not ascending."""
import glob
import os

import numpy as np
import pytest

from bcl_b200 import gen

from test_matrix_io import GOLD, load_a, tile_records

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def tiles_on_host(S):
    trp = S.tile_row_ptr.cpu().numpy()
    toff = S.tile_offset.cpu().numpy()
    nnz = int(toff[-1])
    return trp, toff, S.col_ind[:nnz].cpu().numpy(), S.vals[:nnz].cpu().numpy()


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "tiles_*.npz"))), ids=os.path.basename)
def test_device_slicing_matches_reference_tiles(path):
    from bcl_b200.containers import BlockCustom, SPMatrix
    d = np.load(path)
    a = load_a(d)
    tm, tn = (int(x) for x in d["tiles"])
    trp, toff, ci, v = tiles_on_host(SPMatrix.from_csr(a, BlockCustom((tm, tn))))
    for t, (rp, c, x) in enumerate(tile_records(d)):
        rows = rp.size - 1
        assert np.array_equal(trp[t, : rows + 1], rp)
        assert np.array_equal(ci[toff[t]:toff[t + 1]], c)
        assert np.array_equal(v[toff[t]:toff[t + 1]].view(np.uint32), x.view(np.uint32))


@pytest.mark.parametrize("value_type", ["f32", "i32"])
@pytest.mark.parametrize("tiles", [(1000, 700), (4096, 4096), (333, 16384), (1, 5000)])
def test_device_slicing_matches_host_and_round_trips(value_type, tiles):
    from bcl_b200.containers import BlockCustom, SPMatrix, split_tiles
    a = gen.rmat(13, seed=71, value_type=value_type)
    S = SPMatrix.from_csr(a, BlockCustom(tiles))
    trp, toff, ci, v = tiles_on_host(S)
    htrp, htoff, hci, hv = split_tiles(a, *tiles)
    assert np.array_equal(trp, htrp) and np.array_equal(toff, htoff)
    assert np.array_equal(ci, hci) and np.array_equal(v, hv)
    back = S.get()
    assert np.array_equal(back.row_ptr, a.row_ptr) and np.array_equal(back.col_ind, a.col_ind)
    assert np.array_equal(back.vals, a.vals)


def test_empty_rows_tiles_and_matrices():
    from bcl_b200.containers import BlockCustom, SPMatrix
    d = np.load(os.path.join(GOLD, "tiles_empty_rect.npz"))
    a = load_a(d)
    back = SPMatrix.from_csr(a, BlockCustom((7, 300))).get()
    assert np.array_equal(back.row_ptr, a.row_ptr) and np.array_equal(back.col_ind, a.col_ind)
    z = gen.CSR(50, 40, np.zeros(51, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32))
    S = SPMatrix.from_csr(z, BlockCustom((16, 16)))
    assert S.nnz() == 0
    back = S.get()
    assert back.nnz == 0 and np.array_equal(back.row_ptr, z.row_ptr)


def test_product_gathered_on_device_matches_host_gather():
    from bcl_b200.containers import BlockCustom, SPMatrix, spgemm
    a = gen.rmat(11, seed=72)
    A = SPMatrix.from_csr(a, BlockCustom((300, 500)))
    B = SPMatrix.from_csr(a, BlockCustom((500, 260)))
    C = spgemm(A, B)
    dev, host = C.get(), C.get_host_gather()
    assert np.array_equal(dev.row_ptr, host.row_ptr) and np.array_equal(dev.col_ind, host.col_ind)
    assert np.array_equal(dev.vals.view(np.uint32), host.vals.view(np.uint32))


def test_unsorted_columns_rejected():
    from bcl_b200 import _lib
    from bcl_b200.containers import BlockCustom, SPMatrix
    a = gen.rmat(8, seed=73)
    r = int(np.argmax(np.diff(a.row_ptr)))
    s, e = a.row_ptr[r], a.row_ptr[r + 1]
    ci = a.col_ind.copy()
    ci[s:e] = ci[s:e][::-1]  # a row in descending order
    bad = gen.CSR(a.m, a.n, a.row_ptr, ci, a.vals)
    with pytest.raises(_lib.BclxError):
        SPMatrix.from_csr(bad, BlockCustom((64, 64)))


def test_from_file_matrix_market_and_binary(tmp_path):
    from bcl_b200.containers import BlockCustom, SPMatrix
    path = os.path.join(GOLD, "mm_symmetric_real.mtx")
    want = gen.read_matrix_market(path)
    got = SPMatrix.from_file(path, BlockCustom((16, 20))).get()
    assert np.array_equal(got.col_ind, want.col_ind) and np.array_equal(got.vals, want.vals)
    a = gen.rmat(9, seed=74)
    p = str(tmp_path / "a.binary")
    gen.write_binary(p, a)
    got = SPMatrix.from_file(p, BlockCustom((100, 128))).get()
    assert np.array_equal(got.col_ind, a.col_ind) and np.array_equal(got.vals, a.vals)
