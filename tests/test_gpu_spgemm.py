"""GPU parity of the sparse x sparse path, through the C ABI.

Bar: structure (row_ptr, sorted col_ind, explicit zeros kept) bit-exact;
values bit-exact for int32 and also bit-exact for FP32, because the kernels
reproduce the reference's per-entry order of fused multiply-adds; the
north-star tolerance (1e-5 relative per entry against the reference) is
therefore met with zero error, and the FP32 result's error against an FP64
accumulation is stated in test_fp32_error_vs_fp64."""
import glob
import os

import numpy as np
import pytest

from bcl_b200 import gen
from oracle import oracle as O

from gpu_util import GOLD, assert_csr_identical, assert_rel_close, load_csr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def product(a, b, tiles, mode="fused"):
    from bcl_b200.containers import BlockCustom, SPMatrix, spgemm, spgemm_plain
    tm, tk, tn = tiles
    A = SPMatrix.from_csr(a, BlockCustom((tm, tk)))
    B = SPMatrix.from_csr(b, BlockCustom((tk, tn)))
    if mode == "plain":
        C = spgemm_plain(A, B)
    else:
        C = spgemm(A, B, stages=mode)
    return C


@pytest.mark.parametrize("mode", ["fused", "per_stage", "plain"])
@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "spgemm_*.npz"))), ids=os.path.basename)
def test_golden_spgemm(path, mode):
    d = np.load(path)
    a, b, c = load_csr(d, "a"), load_csr(d, "b"), load_csr(d, "c")
    C = product(a, b, [int(t) for t in d["tiles"]], mode)
    got = C.get()
    assert_csr_identical(got, c.row_ptr, c.col_ind, c.vals)
    assert C.nnz() == c.nnz


def test_golden_dot_one_tile():
    """The local tile kernel alone (CSRMatrix::dot) is a 1x1x1 grid."""
    d = np.load(os.path.join(GOLD, "dot_rmat9_f32.npz"))
    a, c = load_csr(d, "a"), load_csr(d, "c")
    got = product(a, a, (a.m, a.n, a.n)).get()
    assert_csr_identical(got, c.row_ptr, c.col_ind, c.vals)


@pytest.mark.parametrize("name,mode", [("accumulate_rmat9x4_f32", "f32"), ("accumulate_rmat8x3_i32", "i32")])
def test_golden_tile_accumulate(name, mode):
    from bcl_b200.containers import BlockCustom, SPMatrix, tile_accumulate
    d = np.load(os.path.join(GOLD, name + ".npz"))
    parts, i = [], 0
    while f"p{i}_shape" in d:
        p = load_csr(d, f"p{i}")
        parts.append(SPMatrix.from_csr(p, BlockCustom((p.m, p.n))))
        i += 1
    c = load_csr(d, "c")
    got = tile_accumulate(parts).get()
    assert_csr_identical(got, c.row_ptr, c.col_ind, c.vals)


def test_light_and_heavy_rows_mixed():
    """8192-wide tiles of an R-MAT s13 product: both light rows and heavy rows
    (with several items each) occur; compared bit-for-bit."""
    from bcl_b200.containers import BlockCustom, SPMatrix, spgemm
    a = gen.rmat(13, seed=17)
    A = SPMatrix.from_csr(a, BlockCustom((2048, 8192)))
    B = SPMatrix.from_csr(a, BlockCustom((8192, 8192)))
    C, plan = spgemm(A, B, keep_plan=True)
    st = plan.stats()
    plan.close()
    assert st["light_rows"] > 0 and st["heavy_rows"] > 0 and st["heavy_items"] > st["heavy_rows"]
    rp, ci, cv = O.gemm_tiled(a, a, 2048, 8192, 8192)
    assert_csr_identical(C.get(), rp, ci, cv)


@pytest.mark.parametrize("value_type", ["f32", "i32"])
@pytest.mark.parametrize("tiles", [(512, 512, 512), (300, 700, 260), (2048, 2048, 2048)])
def test_rmat11_vs_oracle(value_type, tiles):
    a = gen.rmat(11, seed=101, value_type=value_type)
    rp, ci, cv = O.gemm_tiled(a, a, *tiles, mode=value_type)
    got = product(a, a, tiles).get()
    assert_csr_identical(got, rp, ci, cv)


@pytest.mark.parametrize("mode", ["fused", "per_stage"])
def test_fine_grid_stage_map(mode):
    """Grids with more than 16 tile columns walk only the stages whose A and
    B tiles both have entries: a banded stencil (most tile products empty)
    and R-MAT, against the oracle on the same grid."""
    s = gen.stencil27(24)
    rp, ci, cv = O.gemm_tiled(s, s, 512, 512, 512)
    assert_csr_identical(product(s, s, (512, 512, 512), mode).get(), rp, ci, cv)
    a = gen.rmat(12, seed=103)
    rp, ci, cv = O.gemm_tiled(a, a, 128, 128, 128)
    assert_csr_identical(product(a, a, (128, 128, 128), mode).get(), rp, ci, cv)


@pytest.mark.parametrize("learned", [False, True])
def test_without_btable_binary_search(monkeypatch, learned):
    """With the B-row table disabled (as for grids where it would not fit),
    heavy items find their column-block ranges by binary search: same
    result."""
    from bcl_b200.containers import BlockCustom, SPMatrix, spgemm_learned
    monkeypatch.setenv("BCLX_BTABLE_MAX_BYTES", "0")
    a = gen.rmat(12, seed=104)
    tiles = (1024, 4096, 4096)
    rp, ci, cv = O.gemm_tiled(a, a, *tiles)
    if learned:
        A = SPMatrix.from_csr(a, BlockCustom(tiles[:2]))
        B = SPMatrix.from_csr(a, BlockCustom(tiles[1:]))
        got = spgemm_learned(A, B).get()
    else:
        got = product(a, a, tiles).get()
    assert_csr_identical(got, rp, ci, cv)


def test_wide_tiles_heavy_rows():
    """Tiles 16384 columns wide send every row through the block-wide
    symbolic pass and the cut into <= 512-output items (heavy path)."""
    from bcl_b200.containers import BlockCustom, SPMatrix, spgemm
    a = gen.rmat(14, seed=7)
    A = SPMatrix.from_csr(a, BlockCustom((4096, 16384)))
    B = SPMatrix.from_csr(a, BlockCustom((16384, 16384)))
    C, plan = spgemm(A, B, keep_plan=True)
    st = plan.stats()
    plan.close()
    assert st["heavy_rows"] > 0 and st["light_rows"] == 0 and st["heavy_items"] >= st["heavy_rows"]
    rows = np.random.default_rng(0).choice(a.m, 2000, replace=False)
    rows.sort()
    rp, ci, cv = O.gemm_tiled(a, a, 4096, 16384, 16384, rows=rows)
    full = C.get()
    got_rp = full.row_ptr.astype(np.int64)
    for q, r in enumerate(rows[:400]):
        seg = slice(got_rp[r], got_rp[r + 1])
        assert np.array_equal(full.col_ind[seg], ci[rp[q]:rp[q + 1]])
        assert np.array_equal(full.vals[seg].view(np.uint32), cv[rp[q]:rp[q + 1]].view(np.uint32))
    counts = np.diff(got_rp)[rows]
    assert np.array_equal(counts, np.diff(rp))


def test_empty_and_degenerate():
    from bcl_b200.containers import BlockCustom, SPMatrix, spgemm
    z = gen.CSR(300, 200, np.zeros(301, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32))
    b = gen.rmat(8, seed=1)
    b = gen.CSR(200, 256, *_crop(b, 200, 256))
    C = spgemm(SPMatrix.from_csr(z, BlockCustom((64, 50))), SPMatrix.from_csr(b, BlockCustom((50, 100))))
    assert C.nnz() == 0
    got = C.get()
    assert got.m == 300 and got.n == 256 and got.row_ptr[-1] == 0
    # a single nonzero
    one = gen.CSR(1, 1, np.array([0, 1], np.int32), np.array([0], np.int32), np.array([3.0], np.float32))
    C = spgemm(SPMatrix.from_csr(one, BlockCustom((1, 1))), SPMatrix.from_csr(one, BlockCustom((1, 1))))
    assert C.get().vals.tolist() == [9.0]


def _crop(a, m, n):
    keep_rows = np.arange(m)
    rp, ci, v = [0], [], []
    for r in keep_rows:
        s = slice(a.row_ptr[r], a.row_ptr[r + 1])
        sel = a.col_ind[s] < n
        ci.extend(a.col_ind[s][sel])
        v.extend(a.vals[s][sel])
        rp.append(len(ci))
    return np.array(rp, np.int32), np.array(ci, np.int32), np.array(v, np.float32)


def test_stencil_square_closed_form():
    s = gen.stencil27(12)
    C = product(s, s, (1024, 1024, 1024))
    assert C.nnz() == (5 * 12 - 6) ** 3
    rp, ci, cv = O.gemm_tiled(s, s, 1024, 1024, 1024)
    assert_csr_identical(C.get(), rp, ci, cv)


def test_fp32_error_vs_fp64():
    """State the FP32 result's error against FP64 accumulation (R-MAT s12)."""
    a = gen.rmat(12, seed=5)
    got = product(a, a, (1024, 1024, 1024)).get()
    _, _, c64 = O.gemm_tiled(a, a, 1024, 1024, 1024, mode="f64")
    err = np.abs(got.vals.astype(np.float64) - c64)
    scale = np.abs(c64)
    rel = err / np.maximum(scale, 1e-12)
    print(f"\nFP32 vs FP64: max abs {err.max():.3e}, median rel {np.median(rel):.3e}, "
          f"norm ratio {np.linalg.norm(err) / np.linalg.norm(c64):.3e}")
    assert np.linalg.norm(err) / np.linalg.norm(c64) < 1e-6


@pytest.mark.parametrize("mode", ["batched", "batched_graph"])
def test_batched_forms_match(mode):
    """One launch per SUMMA stage (all tile products of the stage), directly
    or through the plan's CUDA graph: bit-identical to the oracle."""
    a = gen.rmat(12, seed=61)
    tiles = (1024, 1024, 1024)
    rp, ci, cv = O.gemm_tiled(a, a, *tiles)
    assert_csr_identical(product(a, a, tiles, mode).get(), rp, ci, cv)


def test_graph_replay_with_new_values():
    """Same structure, new values: replaying the captured stage launches
    recomputes C for the new values (the plan keeps the structure)."""
    import torch
    from bcl_b200.containers import BlockCustom, SPMatrix, spgemm_numeric, spgemm_symbolic
    a = gen.rmat(12, seed=62)
    A = SPMatrix.from_csr(a, BlockCustom((1024, 1024)))
    plan, out, trp, toff, nnz = spgemm_symbolic(A, A)
    ci = torch.empty(nnz, dtype=torch.int32, device="cuda")
    v = torch.empty(nnz, dtype=torch.float32, device="cuda")
    out.col_ind, out.vals = ci.data_ptr(), v.data_ptr()
    spgemm_numeric(plan, A, A, out, "batched_graph")       # captures
    rng = np.random.default_rng(5)
    for rep in range(2):
        a2 = gen.CSR(a.m, a.n, a.row_ptr, a.col_ind, rng.uniform(-1, 1, a.nnz).astype(np.float32))
        A2 = SPMatrix.from_csr(a2, BlockCustom((1024, 1024)))
        A.vals.copy_(A2.vals)                               # new values, same structure and addresses
        spgemm_numeric(plan, A, A, out, "batched_graph")    # replays
        torch.cuda.synchronize()
        from bcl_b200.containers import SPMatrix as S
        C = S(A.m, A.n, A.tm, A.tn, A.dtype, A.device, trp, toff, ci, v)
        rp, cc, cv = O.gemm_tiled(a2, a2, 1024, 1024, 1024)
        assert_csr_identical(C.get(), rp, cc, cv)
    plan.close()


@pytest.mark.parametrize("tuning", [(1, 3, 32), (8, 4, 1 << 30), (4, 2, 16)])
def test_tuning_does_not_change_results(tuning):
    from bcl_b200.containers import BlockCustom, SPMatrix, spgemm
    a = gen.rmat(12, seed=63)
    A = SPMatrix.from_csr(a, BlockCustom((1024, 1024)))
    rp, ci, cv = O.gemm_tiled(a, a, 1024, 1024, 1024)
    assert_csr_identical(spgemm(A, A, tuning=tuning).get(), rp, ci, cv)


def test_autotune_roundtrip(tmp_path, monkeypatch):
    monkeypatch.setenv("BCLX_CACHE", str(tmp_path))
    from bcl_b200 import autotune
    from bcl_b200.containers import BlockCustom, SPMatrix, spgemm
    a = gen.rmat(11, seed=64)
    A = SPMatrix.from_csr(a, BlockCustom((1024, 1024)))
    params, ms, table = autotune.tune(A, A, reps=1, candidates={"grab": (1, 4), "blocks_per_sm": (4,),
                                                                "long_seg": (48,)}, light_ubs=(256, 512))
    assert len(table) == 2 and ms > 0 and params["light_ub"] in (256, 512)
    C, plan = spgemm(A, A, tuning="auto", keep_plan=True)
    assert autotune.lookup(A, A) == params
    plan.close()
    rp, ci, cv = O.gemm_tiled(a, a, 1024, 1024, 1024)
    assert_csr_identical(C.get(), rp, ci, cv)


@pytest.mark.parametrize("light_ub", [32, 128, 512])
def test_light_row_bound_does_not_change_results(light_ub):
    """The light/heavy classification bound moves rows between the warp and
    the cut-item paths; the result stays bit-identical."""
    from bcl_b200.containers import BlockCustom, SPMatrix, context, spgemm
    a = gen.rmat(12, seed=65)
    A = SPMatrix.from_csr(a, BlockCustom((1024, 1024)))
    with context().tuned(light_ub=light_ub):
        C = spgemm(A, A)
    rp, ci, cv = O.gemm_tiled(a, a, 1024, 1024, 1024)
    assert_csr_identical(C.get(), rp, ci, cv)


def test_tuning_knobs_reject_out_of_range():
    from bcl_b200 import _lib
    from bcl_b200.containers import context
    ctx = context()
    for key, bad in ((_lib.TUNE_LIGHT_UB, 1000), (_lib.TUNE_LEARN_TARGET, 10), (_lib.TUNE_SPMM_ROWS, 3),
                     (_lib.TUNE_SPMM_SCHEDULE, 2), (_lib.TUNE_SPMM_LONG_BLOCKS, 100000)):
        assert _lib.load().bclx_context_set_tuning(ctx.h, key, bad) == _lib.ERR_INVALID
    assert ctx.get_tuning("light_ub") == 512


@pytest.mark.parametrize("tiles", [(1024, 1024, 1024), (2048, 8192, 8192), (4096, 16384, 16384)])
def test_item_outputs_1024_does_not_change_results(tiles):
    """Heavy rows cut into items of up to 1024 outputs (larger shared-memory
    accumulators, fewer items): bit-identical."""
    from bcl_b200.containers import BlockCustom, SPMatrix, context, spgemm
    a = gen.rmat(13, seed=66)
    A = SPMatrix.from_csr(a, BlockCustom(tiles[:2]))
    B = SPMatrix.from_csr(a, BlockCustom(tiles[1:]))
    with context().tuned(item_outputs=1024):
        C = spgemm(A, B)
    rp, ci, cv = O.gemm_tiled(a, a, *tiles)
    assert_csr_identical(C.get(), rp, ci, cv)


def test_wide_tiles_with_light_rows_do_not_change_results():
    """16384-wide tiles with light rows allowed (BCLX_TUNE_WIDE_LIGHT): the
    light path with the wide bitmap template, bit-identical."""
    from bcl_b200.containers import BlockCustom, SPMatrix, context, spgemm
    a = gen.rmat(14, seed=67)
    s = gen.stencil27(26)
    for m, tiles in ((a, (4096, 16384, 16384)), (s, (16384, 16384, 16384))):
        A = SPMatrix.from_csr(m, BlockCustom(tiles[:2]))
        B = SPMatrix.from_csr(m, BlockCustom(tiles[1:]))
        with context().tuned(wide_light=1):
            C, plan = spgemm(A, B, keep_plan=True)
        assert plan.stats()["light_rows"] > 0
        plan.close()
        rows = np.sort(np.random.default_rng(1).choice(m.m, 1500, replace=False))
        rp, ci, cv = O.gemm_tiled(m, m, *tiles, rows=rows)
        full = C.get()
        got_rp = full.row_ptr.astype(np.int64)
        sel = np.concatenate([np.arange(got_rp[r], got_rp[r + 1]) for r in rows])
        assert np.array_equal(np.diff(got_rp)[rows], np.diff(rp))
        assert np.array_equal(full.col_ind[sel], ci)
        assert np.array_equal(full.vals[sel].view(np.uint32), cv.view(np.uint32))
