"""GPU parity of the sparse x dense path, through the C ABI.

FP32: bit-exact against the reference's own outputs (golden fixtures) and
the oracle (same order of fused multiply-adds, C accumulated in place).
BF16 storage: bit-exact against the oracle's BF16 restatement, and within
1e-2 relative (Frobenius) of FP64 accumulation."""
import glob
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


def run(a, bd, tiles, mode="grid", dtype="f32", c0=None):
    import torch
    from bcl_b200.containers import BlockCustom, DMatrix, SPMatrix, spmm, spmm_plain
    tm, tk, tn = tiles
    tdt = torch.float32 if dtype == "f32" else torch.bfloat16
    A = SPMatrix.from_csr(a, BlockCustom((tm, tk)))
    if dtype == "f32":
        B = DMatrix.from_array(torch.from_numpy(bd), BlockCustom((tk, tn)), dtype=tdt)
    else:
        B = DMatrix.from_array(torch.from_numpy(bd.view(np.int16)).view(torch.bfloat16), BlockCustom((tk, tn)),
                               dtype=tdt)
    C = DMatrix.zeros((a.m, bd.shape[1]), BlockCustom((tm, tn)), dtype=tdt)
    if c0 is not None:
        C.set_matrix(torch.from_numpy(c0) if dtype == "f32" else torch.from_numpy(c0.view(np.int16)).view(torch.bfloat16))
    (spmm if mode == "grid" else spmm_plain)(A, B, C)
    out = C.get_matrix().cpu()
    return out.numpy() if dtype == "f32" else out.view(torch.int16).numpy().view(np.uint16)


@pytest.mark.parametrize("mode", ["grid", "plain"])
@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "spmm_*.npz"))), ids=os.path.basename)
def test_golden_spmm(path, mode):
    d = np.load(path)
    a = load_csr(d, "a")
    got = run(a, d["b"], [int(t) for t in d["tiles"]], mode)
    assert np.array_equal(bits(got), bits(d["c"]))


@pytest.mark.parametrize("n,tiles", [(128, (4096, 4096, 128)), (37, (1000, 700, 37)), (600, (2048, 4096, 600)),
                                     (256, (8192, 8192, 256))])
def test_spmm_vs_oracle(n, tiles):
    a = gen.rmat(13, seed=3)
    b = gen.dense(a.n, n, seed=4)
    c0 = gen.dense(a.m, n, seed=5)
    got = run(a, b, tiles, c0=c0)
    want = O.spmm_tiled(a, b, c0, *tiles)
    assert np.array_equal(bits(got), bits(want))


@pytest.mark.parametrize("n,tiles", [(256, (8192, 8192, 256)), (128, (4096, 4096, 128)), (40, (3000, 5000, 40))])
def test_spmm_bf16(n, tiles):
    a = gen.rmat(13, seed=8)
    b = gen.dense(a.n, n, seed=9, dist="normal")
    b16 = O.to_bf16(b)
    got = run(a, b16, tiles, dtype="bf16", c0=np.zeros((a.m, n), np.uint16))
    want = O.spmm_tiled_bf16(a, b16, np.zeros((a.m, n), np.uint16), *tiles)
    assert np.array_equal(got, want)
    c64 = O.spmm_f64(a, b)
    err = np.linalg.norm(O.bf16_to_f32(got) - c64) / np.linalg.norm(c64)
    print(f"\nBF16 storage vs FP64: relative Frobenius error {err:.3e}")
    assert err < 1e-2


def heavy_rows_matrix(n=16384, light=8, heavy=(12000, 9000, 6000, 4500, 1024, 1023), seed=11):
    """Mostly `light` entries per row, a few empty rows, and a few rows long
    enough for the long-row kernel (1024 or more entries over all stages)
    with one just below."""
    rng = np.random.default_rng(seed)
    lens = np.full(n, light, np.int64)
    lens[rng.choice(n, size=300, replace=False)] = 0
    rows = rng.choice(n, size=len(heavy), replace=False)
    lens[rows] = heavy
    cols = [np.sort(rng.choice(n, size=int(k), replace=False)) for k in lens]
    row_ptr = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=row_ptr[1:])
    col_ind = np.concatenate(cols).astype(np.int32)
    vals = rng.uniform(-1, 1, size=col_ind.size).astype(np.float32)
    return gen.CSR(n, n, row_ptr.astype(np.int32), col_ind, vals)


@pytest.mark.parametrize("dtype", ["f32", "bf16"])
@pytest.mark.parametrize("tiles", [(4096, 4096, 256), (16384, 16384, 256), (3000, 5000, 200), (1000, 1024, 128)])
def test_spmm_long_rows(monkeypatch, dtype, tiles):
    """Rows of thousands of entries run by the long-row kernel on the side
    stream (its panels and tile columns spread over warps) while the rest
    run as usual; enabled here below its size threshold."""
    monkeypatch.setenv("BCLX_SPMM_LONG_MIN_ROWS", "0")
    a = heavy_rows_matrix()
    n = tiles[2] if tiles[2] in (128, 256) else 400
    b = gen.dense(a.n, n, seed=12, dist="normal")
    c0 = gen.dense(a.m, n, seed=13)
    if dtype == "f32":
        got = run(a, b, tiles, c0=c0)
        want = O.spmm_tiled(a, b, c0, *tiles)
        assert np.array_equal(bits(got), bits(want))
    else:
        b16, c16 = O.to_bf16(b), O.to_bf16(c0)
        got = run(a, b16, tiles, dtype="bf16", c0=c16)
        want = O.spmm_tiled_bf16(a, b16, c16, *tiles)
        assert np.array_equal(got, want)


def test_spmm_ragged_last_tile_unaligned_width(monkeypatch):
    """Aligned leading dimension but a last tile column whose width is not a
    whole number of 16-byte vectors: element-wise access for that tile (and
    the long-row kernel leaves its long rows to the element-wise form)."""
    monkeypatch.setenv("BCLX_SPMM_LONG_MIN_ROWS", "0")
    a = heavy_rows_matrix(n=4096, heavy=(3000, 2000))
    b = gen.dense(a.n, 38, seed=15)
    c0 = gen.dense(a.m, 38, seed=16)
    tiles = (1000, 1500, 24)
    got = run(a, b, tiles, c0=c0)
    want = O.spmm_tiled(a, b, c0, *tiles)
    assert np.array_equal(bits(got), bits(want))


@pytest.mark.parametrize("rows", ["2", "4"])
@pytest.mark.parametrize("dtype", ["f32", "bf16"])
@pytest.mark.parametrize("tiles,n,long_rows", [((4096, 4096, 256), 256, True), ((3001, 5000, 200), 400, False),
                                               ((1000, 1024, 128), 128, True), ((999, 1500, 24), 38, False)])
def test_spmm_grouped_rows(monkeypatch, rows, dtype, tiles, n, long_rows):
    """Several rows of one C tile walked by one warp (their entries
    flattened, each row's chain started from its own C value): the same bits
    as one row per warp, with empty rows, tile row counts that are not a
    multiple of the group, long rows left to the long-row kernel, and an
    element-wise (unaligned width) tile column."""
    monkeypatch.setenv("BCLX_SPMM_ROWS", rows)
    if long_rows:
        monkeypatch.setenv("BCLX_SPMM_LONG_MIN_ROWS", "0")
    a = heavy_rows_matrix(n=8192, light=3, heavy=(5000, 1024, 700))
    b = gen.dense(a.n, n, seed=17, dist="normal")
    c0 = gen.dense(a.m, n, seed=18)
    if dtype == "f32":
        got = run(a, b, tiles, c0=c0)
        want = O.spmm_tiled(a, b, c0, *tiles)
        assert np.array_equal(bits(got), bits(want))
    else:
        b16, c16 = O.to_bf16(b), O.to_bf16(c0)
        got = run(a, b16, tiles, dtype="bf16", c0=c16)
        want = O.spmm_tiled_bf16(a, b16, c16, *tiles)
        assert np.array_equal(got, want)


@pytest.mark.parametrize("rows", ["1", "4"])
@pytest.mark.parametrize("dtype", ["f32", "bf16"])
def test_spmm_rows_without_entries_untouched(monkeypatch, dtype, rows):
    """C rows whose A rows have no entries (over all stages) keep their exact
    bits, NaN payloads included: no load or store reaches them; the other
    rows match the oracle bit for bit.  With and without the long-row path."""
    monkeypatch.setenv("BCLX_SPMM_LONG_MIN_ROWS", "0")
    monkeypatch.setenv("BCLX_SPMM_ROWS", rows)
    a = heavy_rows_matrix(n=8192, light=2, heavy=(3000, 1100))
    n = 256
    tiles = (1024, 2048, 256)
    empty = np.diff(a.row_ptr) == 0
    assert empty.sum() >= 100
    b = gen.dense(a.n, n, seed=21, dist="normal")
    c0 = gen.dense(a.m, n, seed=22)
    if dtype == "f32":
        c0.view(np.uint32)[empty] = np.uint32(0x7FC01234)
        got = run(a, b, tiles, c0=c0)
        want = O.spmm_tiled(a, b, c0, *tiles)
        assert np.all(bits(got)[empty] == np.uint32(0x7FC01234))
        assert np.array_equal(bits(got)[~empty], bits(want)[~empty])
    else:
        b16, c16 = O.to_bf16(b), O.to_bf16(c0)
        c16[empty] = np.uint16(0x7FC5)
        got = run(a, b16, tiles, dtype="bf16", c0=c16)
        want = O.spmm_tiled_bf16(a, b16, c16, *tiles)
        assert np.all(got[empty] == np.uint16(0x7FC5))
        assert np.array_equal(got[~empty], want[~empty])


def test_spmm_tile_single_call_ld():
    """bclx_spmm_tile with leading dimensions larger than n (sub-blocks)."""
    import ctypes
    import torch
    from bcl_b200 import _lib
    from bcl_b200.containers import context
    a = gen.erdos_renyi(500, 7, seed=1)
    b = gen.dense(500, 96, seed=2)
    c0 = gen.dense(500, 64, seed=3)
    B = torch.from_numpy(b).cuda()            # ldb = 96, use the first 64 columns
    C = torch.zeros((500, 80), device="cuda")  # ldc = 80
    C[:, :64] = torch.from_numpy(c0)
    rp = torch.from_numpy(a.row_ptr).cuda()
    ci = torch.from_numpy(a.col_ind).cuda()
    v = torch.from_numpy(a.vals).cuda()
    h = context().use_current_stream()
    _lib.call("bclx_spmm_tile", h, 500, 64, 500, a.nnz, ctypes.c_void_p(C.data_ptr()),
              ctypes.c_void_p(B.data_ptr()), ctypes.c_void_p(v.data_ptr()), ctypes.c_void_p(rp.data_ptr()),
              ctypes.c_void_p(ci.data_ptr()), 96, 80, _lib.F32)
    want = O.spmm_tiled(a, b[:, :64].copy(), c0, 500, 500, 64)
    assert np.array_equal(bits(C[:, :64].cpu().numpy()), bits(want))
    assert torch.count_nonzero(C[:, 64:]) == 0


@pytest.mark.parametrize("knobs", [dict(spmm_rows=1), dict(spmm_rows=4, spmm_long_row=64, spmm_long_blocks=20),
                                   dict(spmm_schedule=1), dict(spmm_schedule=1, spmm_long_row=128),
                                   dict(spmm_panel_major=1), dict(spmm_panel_major=1, spmm_rows=2)])
def test_spmm_knobs_do_not_change_results(monkeypatch, knobs):
    """Rows per item, the long-row threshold and block count, the schedule
    (the long-row path forced on by a small product-size bound) and the
    panel order leave every bit of C as it was."""
    monkeypatch.setenv("BCLX_SPMM_LONG_MIN_ROWS", "1024")
    import torch
    from bcl_b200.containers import BlockCustom, DMatrix, SPMatrix, spmm
    a = gen.rmat(13, seed=11)
    b = gen.dense(a.n, 256, seed=12)
    c0 = gen.dense(a.m, 256, seed=13)
    A = SPMatrix.from_csr(a, BlockCustom((2048, 2048)))
    B = DMatrix.from_array(torch.from_numpy(b), BlockCustom((2048, 256)))
    C = DMatrix.from_array(torch.from_numpy(c0), BlockCustom((2048, 256)))
    spmm(A, B, C, tuning=knobs)
    want = O.spmm_tiled(a, b, c0, 2048, 2048, 256)
    assert np.array_equal(bits(C.get_matrix().cpu().numpy()), bits(want))


def test_spmm_autotune_roundtrip(tmp_path, monkeypatch):
    monkeypatch.setenv("BCLX_CACHE", str(tmp_path))
    import torch
    from bcl_b200 import autotune
    from bcl_b200.containers import BlockCustom, DMatrix, SPMatrix, spmm
    a = gen.rmat(12, seed=14)
    b = gen.dense(a.n, 128, seed=15)
    A = SPMatrix.from_csr(a, BlockCustom((1024, 1024)))
    B = DMatrix.from_array(torch.from_numpy(b), BlockCustom((1024, 128)))
    C = DMatrix.zeros((a.m, 128), BlockCustom((1024, 128)))
    params, ms = autotune.tune_spmm(A, B, C, reps=1, candidates={"spmm_rows": (1, 2), "spmm_schedule": (0, 1)})
    assert ms > 0 and autotune.lookup(A, B, "spmm") == params
    C2 = DMatrix.zeros((a.m, 128), BlockCustom((1024, 128)))
    spmm(A, B, C2, tuning="auto")
    want = O.spmm_tiled(a, b, np.zeros((a.m, 128), np.float32), 1024, 1024, 128)
    assert np.array_equal(bits(C2.get_matrix().cpu().numpy()), bits(want))


@pytest.mark.parametrize("schedule,panel_major", [(0, 0), (1, 0), (0, 1)])
def test_spmm_schedules_large(schedule, panel_major):
    """R-MAT s18 x 256 FP32 (long rows on their own kernel) under both
    schedules (side stream with a launch delay, programmatic dependent
    launch) and both panel orders: sampled rows bit-exact."""
    import torch
    from bcl_b200.containers import BlockCustom, DMatrix, SPMatrix, spmm
    a = gen.rmat(18, seed=16)
    b = gen.dense(a.n, 256, seed=17, dist="normal")
    ts = a.m // 4
    A = SPMatrix.from_csr(a, BlockCustom((ts, ts)))
    B = DMatrix.from_array(torch.from_numpy(b), BlockCustom((ts, 256)))
    C = DMatrix.zeros((a.m, 256), BlockCustom((ts, 256)))
    spmm(A, B, C, tuning=dict(spmm_schedule=schedule, spmm_panel_major=panel_major))
    rows = np.unique(np.concatenate([np.random.default_rng(18).choice(a.m, 2048, replace=False), np.arange(32)]))
    got = C.get_matrix()[torch.as_tensor(rows, device="cuda")].cpu().numpy()
    want = O.spmm_tiled(a, b, np.zeros((rows.size, 256), np.float32), ts, ts, 256, rows=rows)
    assert np.array_equal(bits(got), bits(want))

