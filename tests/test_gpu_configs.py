"""GPU parity at the benchmark configurations' own sizes and tile grids.

Every timed configuration is checked against the oracle (the CPU restatement
of the reference's tile loop, pinned to the reference binary by
test_oracle_golden.py) on its full-size input:

* Erdos-Renyi 16384^2 (16 per row) x dense 16384x128, 4x4 grid: the whole
  product, FP32 bit-exact.
* R-MAT s16 A*A on 8x8 tiles: the whole product, FP32 and int32, bit-exact
  (structure and values), for the fused and the learned forms.
* R-MAT s18 A*A on 16x16 tiles and R-MAT s20 A*A on 64x64 tiles (16384-wide
  tiles: every row takes the block symbolic pass, stage maps are active and
  at s20 the B-row table exceeds its cap, so heavy items binary-search B
  rows): 4096 seeded rows bit-exact, plus every sampled row's length.
* 27-point stencil L*L on 128^3 with 128x128 tiles: the closed-form nnz
  (5*128-6)^3 and 4096 seeded rows bit-exact.
* R-MAT s21 x dense 2097152x256 N(0,1) on 8x8 tiles: 4096 seeded rows, FP32
  bit-exact; BF16 storage bit-exact against the oracle's BF16 restatement and
  within 1e-2 relative (Frobenius) of FP64 on the same rows.

Rows are compared where the oracle would take minutes for the whole product;
rows are independent in the reference's algorithm, so a row's result does
not depend on which other rows are computed."""
import gc

import numpy as np
import pytest

from bcl_b200 import gen
from oracle import oracle as O

from gpu_util import assert_csr_identical, bits

pytestmark = pytest.mark.gpu

SAMPLE_ROWS = 4096


@pytest.fixture(scope="module", autouse=True)
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.fixture(autouse=True)
def release_memory():
    """The large products' outputs and scratch go back between tests."""
    yield
    import torch
    from bcl_b200.containers import context
    gc.collect()
    torch.cuda.synchronize()
    context().release_cached()
    torch.cuda.empty_cache()


def seeded_rows(m, count, seed):
    rows = np.random.default_rng(seed).choice(m, size=min(count, m), replace=False)
    rows.sort()
    return rows


def sample_rows(C, rows):
    """Rows `rows` (global indices) of a tiled sparse result, gathered on the
    device from its packed tiles: (row_ptr int64 [R+1], global col_ind int32,
    vals), each row's tiles in column order."""
    import torch
    dev = C.col_ind.device
    r = torch.as_tensor(np.asarray(rows, np.int64), device=dev)
    ti, lr = r // C.tm, r % C.tm
    t = ti[:, None] * C.gn + torch.arange(C.gn, device=dev)[None, :]
    trp = C.tile_row_ptr.reshape(-1).to(torch.int64)
    base = C.tile_offset[t]
    s = base + trp[t * (C.tm + 1) + lr[:, None]]
    e = base + trp[t * (C.tm + 1) + lr[:, None] + 1]
    lens = (e - s).reshape(-1)
    seg = torch.repeat_interleave(torch.arange(lens.numel(), device=dev), lens)
    first = torch.cumsum(lens, 0) - lens
    pos = s.reshape(-1)[seg] + (torch.arange(seg.numel(), device=dev) - first[seg])
    cols = (C.col_ind[pos].to(torch.int64) + (seg % C.gn) * C.tn).to(torch.int32)
    vals = C.vals[pos]
    rp = torch.zeros(len(rows) + 1, dtype=torch.int64, device=dev)
    rp[1:] = torch.cumsum(lens.view(-1, C.gn).sum(1), 0)
    return rp.cpu().numpy(), cols.cpu().numpy(), vals.cpu().numpy()


def spgemm_config(a, grid, form="fused"):
    from bcl_b200.containers import BlockCustom, SPMatrix, spgemm, spgemm_learned
    ts = -(-a.m // grid)
    A = SPMatrix.from_csr(a, BlockCustom((ts, ts)))
    C = spgemm_learned(A, A) if form == "learned" else spgemm(A, A)
    return C, ts


def check_rows(C, a, ts, rows, mode="f32"):
    grp, gci, gv = sample_rows(C, rows)
    rp, ci, cv = O.gemm_tiled(a, a, ts, ts, ts, rows=rows, mode=mode)
    assert np.array_equal(np.diff(grp), np.diff(rp)), "row lengths differ"
    assert np.array_equal(gci, ci), "col_ind differs"
    assert np.array_equal(bits(gv), bits(cv)), "values differ"


@pytest.mark.parametrize("form", ["fused", "learned"])
@pytest.mark.parametrize("value_type", ["f32", "i32"])
def test_rmat16_8x8_whole_product(value_type, form):
    a = gen.rmat(16, seed=0, value_type=value_type)
    C, ts = spgemm_config(a, 8, form)
    rp, ci, cv = O.gemm_tiled(a, a, ts, ts, ts, mode=value_type)
    assert C.nnz() == int(rp[-1])
    assert_csr_identical(C.get(), rp, ci, cv)


def test_rmat18_16x16_sampled_rows():
    a = gen.rmat(18, seed=0)
    C, ts = spgemm_config(a, 16)
    check_rows(C, a, ts, seeded_rows(a.m, SAMPLE_ROWS, 18))


def test_rmat20_64x64_sampled_rows():
    a = gen.rmat(20, seed=0)
    C, ts = spgemm_config(a, 64)
    rows = seeded_rows(a.m, SAMPLE_ROWS, 20)
    # the heaviest rows of R-MAT sit at indices with few one bits: add some
    rows = np.unique(np.concatenate([rows, np.arange(64)]))
    check_rows(C, a, ts, rows)


def test_stencil128_128x128_closed_form_and_rows():
    s = gen.stencil27(128)
    C, ts = spgemm_config(s, 128)
    assert C.nnz() == (5 * 128 - 6) ** 3
    check_rows(C, s, ts, seeded_rows(s.m, SAMPLE_ROWS, 128))


def test_er16k_spmm_whole_product():
    import torch
    from bcl_b200.containers import BlockCustom, DMatrix, SPMatrix, spmm
    a = gen.erdos_renyi(16384, 16, seed=0)
    b = gen.dense(a.n, 128, seed=1)
    ts = 4096
    A = SPMatrix.from_csr(a, BlockCustom((ts, ts)))
    B = DMatrix.from_array(torch.from_numpy(b), BlockCustom((ts, 128)))
    C = DMatrix.zeros((a.m, 128), BlockCustom((ts, 128)))
    spmm(A, B, C)
    want = O.spmm_tiled(a, b, np.zeros((a.m, 128), np.float32), ts, ts, 128)
    assert np.array_equal(bits(C.get_matrix().cpu().numpy()), bits(want))


def test_rmat21_spmm_256_sampled_rows_fp32_and_bf16():
    import torch
    from bcl_b200.containers import BlockCustom, DMatrix, SPMatrix, spmm
    a = gen.rmat(21, seed=0)
    b = gen.dense(a.n, 256, seed=1, dist="normal")
    G = 8
    ts = -(-a.m // G)
    rows = seeded_rows(a.m, SAMPLE_ROWS, 21)
    rows = np.unique(np.concatenate([rows, np.arange(64)]))  # include the longest rows
    A = SPMatrix.from_csr(a, BlockCustom((ts, ts)))
    rsel = torch.as_tensor(rows, device="cuda")
    zero_rows = np.zeros((rows.size, 256), np.float32)
    # FP32 storage: bit-exact
    B = DMatrix.from_array(torch.from_numpy(b), BlockCustom((ts, 256)))
    C = DMatrix.zeros((a.m, 256), BlockCustom((ts, 256)))
    spmm(A, B, C)
    got = C.get_matrix()[rsel].cpu().numpy()
    want = O.spmm_tiled(a, b, zero_rows, ts, ts, 256, rows=rows)
    assert np.array_equal(bits(got), bits(want))
    del B, C
    torch.cuda.empty_cache()
    # BF16 storage: bit-exact against the BF16 restatement, close to FP64
    b16 = O.to_bf16(b)
    B16 = DMatrix.from_array(torch.from_numpy(b16.view(np.int16)).view(torch.bfloat16), BlockCustom((ts, 256)),
                             dtype=torch.bfloat16)
    C16 = DMatrix.zeros((a.m, 256), BlockCustom((ts, 256)), dtype=torch.bfloat16)
    spmm(A, B16, C16)
    got16 = C16.get_matrix()[rsel].cpu().view(torch.int16).numpy().view(np.uint16)
    want16 = O.spmm_tiled_bf16(a, b16, np.zeros((rows.size, 256), np.uint16), ts, ts, 256, rows=rows)
    assert np.array_equal(got16, want16)
    c64 = O.spmm_f64(a, b, rows=rows)
    err = np.linalg.norm(O.bf16_to_f32(got16) - c64) / np.linalg.norm(c64)
    err32 = np.linalg.norm(got.astype(np.float64) - c64) / np.linalg.norm(c64)
    print(f"\nR-MAT s21 x 256 on {rows.size} rows vs FP64: FP32 {err32:.3e}, BF16 storage {err:.3e}")
    assert err < 1e-2 and err32 < 1e-5
