"""GPU parity of the container operations beside the products, through the
C ABI:

* rowwise_gemm / cached_rowwise_gemm / batched_rowwise_gemm
  (experimental_gemm.hpp:83-214): bit-exact against the reference's own
  outputs (golden fixtures) and the oracle's ascending-stage restatement;
* DMatrix::sum (DMatrix.hpp:537-554): int32 exact; FP32/BF16 accumulated in
  FP64 on the device, within the reference's own sequential-sum rounding
  bound of the reference's FP32 result (and within FP64 rounding of the exact
  sum);
* SPMatrix::binary_op_inplace (SPMatrix.hpp:571-616): bit-exact against the
  reference (tile values, and the whole matrix through SPMatrix::get, which
  turns -0.0 into +0.0) and against the oracle on ragged multi-tile grids."""
import glob
import math
import os

import numpy as np
import pytest

from bcl_b200 import gen
from oracle import oracle as O

from gpu_util import GOLD, bits, load_csr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def dense(arr, tiles, dtype=None):
    import torch
    from bcl_b200.containers import BlockCustom, DMatrix
    t = torch.from_numpy(np.ascontiguousarray(arr))
    return DMatrix.from_array(t, BlockCustom(tiles), dtype=dtype or t.dtype)


@pytest.mark.parametrize("variant", ["rowwise_gemm", "cached_rowwise_gemm", "batched_rowwise_gemm"])
@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "rowwise_*.npz"))), ids=os.path.basename)
def test_golden_rowwise(path, variant):
    from bcl_b200 import containers as K
    d = np.load(path)
    a = load_csr(d, "a")
    tm, tk, tn = (int(t) for t in d["tiles"])
    A = K.SPMatrix.from_csr(a, K.BlockCustom((tm, tk)))
    B = dense(d["b"], (tk, tn))
    C = dense(np.zeros_like(d["c_plain"]), (tm, tn))
    getattr(K, variant)(A, B, C)
    key = {"rowwise_gemm": "c_plain", "cached_rowwise_gemm": "c_cached", "batched_rowwise_gemm": "c_batched"}[variant]
    assert np.array_equal(bits(C.get_matrix().cpu().numpy()), bits(d[key]))


@pytest.mark.parametrize("tiles", [(1000, 700, 96), (4096, 4096, 128), (333, 2048, 40)])
def test_rowwise_vs_oracle(tiles):
    from bcl_b200 import containers as K
    a = gen.rmat(13, seed=31)
    n = tiles[2]
    b = gen.dense(a.n, n, seed=32)
    c0 = gen.dense(a.m, n, seed=33)
    A = K.SPMatrix.from_csr(a, K.BlockCustom(tiles[:2]))
    B = dense(b, tiles[1:])
    C = dense(c0, (tiles[0], n))
    K.rowwise_gemm(A, B, C)
    want = O.spmm_rowwise(a, b, c0, *tiles)
    assert np.array_equal(bits(C.get_matrix().cpu().numpy()), bits(want))


def test_rowwise_needs_one_tile_column():
    from bcl_b200 import containers as K
    a = gen.rmat(8, seed=34)
    A = K.SPMatrix.from_csr(a, K.BlockCustom((64, 64)))
    B = dense(gen.dense(a.n, 64, seed=35), (64, 32))
    C = dense(np.zeros((a.m, 64), np.float32), (64, 32))
    with pytest.raises(RuntimeError):
        K.rowwise_gemm(A, B, C)


def sum_bound(x):
    x = np.asarray(x, np.float64)
    return (x.size - 1) * 2.0 ** -24 * np.abs(x).sum()


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "dsum_*.npz"))), ids=os.path.basename)
def test_golden_dmatrix_sum(path):
    d = np.load(path)
    ref = float(d["bits"].view(np.float32)[()])
    got = dense(d["x"], tuple(int(t) for t in d["tiles"])).sum()
    exact = math.fsum(d["x"].astype(np.float64).ravel())
    assert abs(got - ref) <= sum_bound(d["x"]) + abs(ref) * 2.0 ** -23
    assert abs(got - exact) <= abs(exact) * 2.0 ** -24 + 1e-30 + d["x"].size * 2.0 ** -52 * np.abs(d["x"]).sum()


def test_dmatrix_sum_int32_bf16_and_ragged():
    import torch
    rng = np.random.default_rng(36)
    xi = rng.integers(-2**31, 2**31 - 1, (700, 333), dtype=np.int64).astype(np.int32)
    got = dense(xi, (128, 100)).sum()
    want = np.int32(np.uint32(int(xi.astype(np.int64).sum()) & 0xffffffff).view(np.int32))
    assert got == int(want)
    xf = gen.dense(2000, 70, seed=37, dist="normal")
    D = dense(xf, (512, 64), dtype=torch.bfloat16)
    xb = D.get_matrix().float().cpu().numpy().astype(np.float64)
    got = D.sum()
    exact = math.fsum(xb.ravel())
    assert abs(got - exact) <= abs(exact) * 2.0 ** -24 + xb.size * 2.0 ** -52 * np.abs(xb).sum()
    # the padding of edge tiles (rows 2000..2047, columns 70..127) is not summed
    D2 = dense(xf, (512, 64))
    tv = D2.tiles.view(4, 2, 512, 64)
    tv[3, :, 2000 - 3 * 512:, :] = 1e30
    tv[:, 1, :, 70 - 64:] = 1e30
    exact = math.fsum(xf.astype(np.float64).ravel())
    assert abs(D2.sum() - exact) <= abs(exact) * 2.0 ** -24 + xf.size * 2.0 ** -52 * np.abs(xf).sum()


@pytest.mark.parametrize("dt", ["f32", "i32"])
def test_golden_binary_op(dt):
    from bcl_b200 import containers as K
    d = np.load(os.path.join(GOLD, f"binop_sparse120x90_{dt}.npz"))
    a = load_csr(d, "a")
    for key in d.files:
        if not key.startswith("vals_"):
            continue
        op = key[5:]
        A = K.SPMatrix.from_csr(a, K.BlockCustom((a.m, a.n)))
        B = dense(d["b"], (a.m, a.n))
        A.binary_op_inplace(B, op)
        tile = A.get_tile((0, 0))
        assert np.array_equal(bits(tile.vals), bits(d[key])), op
        assert np.array_equal(bits(A.get().vals), bits(d["get_" + op])), op


@pytest.mark.parametrize("op", ["plus", "minus", "multiplies", "divides", "min", "max", "second"])
def test_binary_op_ragged_grids_vs_oracle(op):
    from bcl_b200 import containers as K
    a = gen.rmat(11, seed=38)
    b = gen.dense(a.m, a.n, seed=39, dist="normal")
    b[np.random.default_rng(40).random(b.shape) < 0.02] = 0.0
    A = K.SPMatrix.from_csr(a, K.BlockCustom((300, 700)))   # sparse and dense grids differ
    B = dense(b, (512, 256))
    A.binary_op_inplace(B, op)
    want = O.binary_op(a, b, op)
    got = A.get()
    assert np.array_equal(got.col_ind, a.col_ind)
    assert np.array_equal(bits(got.vals), bits(O.gather_value(want)))
