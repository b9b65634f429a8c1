"""The distributed product's device path on one GPU: each process of the
reference's stationary-C loop owns the C tiles (i, j) with process
(j % pn) + (i % pm) * pn (SPMatrix.hpp:230-237) and computes them with their
global stage order (spgemm.hpp:194-224).  Here every process's sub-grid is
computed in turn on the one GPU (bclx_spgemm_symbolic_sub through
containers.spgemm_distributed) and the sub-grids, assembled, must equal the
whole product bit for bit: the per-tile order of sums does not depend on
which process computes a tile."""
import numpy as np
import pytest

from bcl_b200 import gen
from oracle import oracle as O

from gpu_util import assert_csr_identical

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def sub_parts(A, world, pgrid=None):
    from bcl_b200.containers import spgemm_distributed
    parts = []
    for p in range(world):
        C, rows, cols = spgemm_distributed(A, A, p, world, pgrid)
        if C is None:
            continue
        n = C.nnz()
        parts.append((rows, cols, C.tile_row_ptr.cpu().numpy(), C.tile_offset.cpu().numpy(),
                      C.col_ind[:n].cpu().numpy(), C.vals[:n].cpu().numpy()))
    return parts


@pytest.mark.parametrize("world,pgrid", [(1, None), (2, None), (4, None), (3, (1, 3)), (6, (2, 3)), (8, (4, 2))])
@pytest.mark.parametrize("value_type", ["f32", "i32"])
def test_sub_grids_assemble_to_the_whole_product(world, pgrid, value_type):
    from bcl_b200.containers import BlockCustom, SPMatrix, assemble_tiles
    a = gen.rmat(12, seed=71, value_type=value_type)
    ts = 512
    A = SPMatrix.from_csr(a, BlockCustom((ts, ts)))
    whole = assemble_tiles(a.m, a.n, ts, ts, sub_parts(A, world, pgrid))
    rp, ci, cv = O.gemm_tiled(a, a, ts, ts, ts, mode=value_type)
    assert_csr_identical(whole, rp, ci, cv)


def test_sub_grids_ragged_and_fine_grid():
    """Ragged edge tiles (only the last tile row / column of a sub-grid can
    be one) and a grid past 16 tiles (stage maps), 4 processes."""
    from bcl_b200.containers import BlockCustom, SPMatrix, assemble_tiles
    a = gen.rmat(12, seed=72)
    for ts in (300, 200):
        A = SPMatrix.from_csr(a, BlockCustom((ts, ts)))
        whole = assemble_tiles(a.m, a.n, ts, ts, sub_parts(A, 4))
        rp, ci, cv = O.gemm_tiled(a, a, ts, ts, ts)
        assert_csr_identical(whole, rp, ci, cv)


@pytest.mark.parametrize("form", ["fused", "learned"])
def test_blocked_product_matches_whole(form):
    """A product computed one block of C tile rows at a time (fused and
    learned forms) equals the whole product bit for bit."""
    from bcl_b200.containers import BlockCustom, SPMatrix, assemble_tiles, spgemm_blocks
    a = gen.rmat(12, seed=73)
    ts = 512
    A = SPMatrix.from_csr(a, BlockCustom((ts, ts)))
    parts = []
    for rows, C in spgemm_blocks(A, A, 3, form=form):
        n = C.nnz()
        parts.append((rows, list(range(A.gn)), C.tile_row_ptr.cpu().numpy(), C.tile_offset.cpu().numpy(),
                      C.col_ind[:n].cpu().numpy(), C.vals[:n].cpu().numpy()))
    whole = assemble_tiles(a.m, a.n, ts, ts, parts)
    rp, ci, cv = O.gemm_tiled(a, a, ts, ts, ts)
    assert_csr_identical(whole, rp, ci, cv)


def test_product_to_host_blocks():
    """containers.spgemm_to_host: C block by block into pinned host memory,
    copies overlapped with the next block's product; the blocks assemble to
    the whole product bit for bit, also on a second call reusing buffers."""
    from bcl_b200.containers import BlockCustom, SPMatrix, assemble_tiles, spgemm_to_host
    a = gen.rmat(12, seed=74)
    ts = 512
    A = SPMatrix.from_csr(a, BlockCustom((ts, ts)))
    rp, ci, cv = O.gemm_tiled(a, a, ts, ts, ts)
    host = None
    for _ in range(2):
        host, blocks = spgemm_to_host(A, A, block_rows=3, host=host)
        parts = [(rows, list(range(A.gn)), trp.numpy(), toff.numpy(), c.numpy(), v.numpy())
                 for rows, nnz, trp, toff, c, v in blocks]
        assert_csr_identical(assemble_tiles(a.m, a.n, ts, ts, parts), rp, ci, cv)


@pytest.mark.parametrize("world,pgrid,tiles,value_type", [(4, (2, 2), (512, 512, 512), "f32"),
                                                          (3, (3, 1), (300, 200, 250), "f32"),
                                                          (4, (2, 2), (300, 200, 250), "i32")])
def test_owned_product_from_fetched_operands(world, pgrid, tiles, value_type):
    """Each process's C tiles from the operand tiles it holds after the row /
    column exchange (bcl_b200.distributed: A's tile rows I and B's tile
    columns J packed as compact grids, bclx_spgemm_symbolic_sub with the
    global tile indices).  The exchange's delivery is the owners' tiles bit
    for bit (checked with gloo ranks on CPU); here each process's share is
    taken from the host matrix, and the sub-grids computed on the GPU
    assemble to the whole product.  Ragged tiles in every dimension and a
    grid of 21 tiles along k (stage maps) are covered."""
    import torch
    from bcl_b200.containers import assemble_tiles
    from bcl_b200.distributed import host_tile, spgemm_owned
    a = gen.rmat(12, seed=75, value_type=value_type)
    b = gen.rmat(12, seed=76, value_type=value_type)
    tm, tk, tn = tiles
    gm, gk, gn = -(-a.m // tm), -(-a.n // tk), -(-b.n // tn)
    pm, pn = pgrid
    dtype = np.float32 if value_type == "f32" else np.int32
    parts = []
    for p in range(world):
        r, c = divmod(p, pn)
        I = [i for i in range(gm) if i % pm == r]
        J = [j for j in range(gn) if j % pn == c]
        a_rows = {(i, k): tuple(torch.from_numpy(x) for x in host_tile(a, tm, tk, i, k)) for i in I for k in range(gk)}
        b_cols = {(k, j): tuple(torch.from_numpy(x) for x in host_tile(b, tk, tn, k, j)) for k in range(gk) for j in J}
        C = spgemm_owned(a_rows, b_cols, I, J, (a.m, a.n), (b.m, b.n), tm, tk, tn, dtype=dtype, device=0)
        n = C.nnz()
        parts.append((I, J, C.tile_row_ptr.cpu().numpy(), C.tile_offset.cpu().numpy(), C.col_ind[:n].cpu().numpy(),
                      C.vals[:n].cpu().numpy()))
    whole = assemble_tiles(a.m, b.n, tm, tn, parts)
    rp, ci, cv = O.gemm_tiled(a, b, tm, tk, tn, mode=value_type)
    assert_csr_identical(whole, rp, ci, cv)


def _nccl_exchange_one_rank(port, q):
    """One NCCL rank on cuda:0: its tiles pass through exchange_operands as
    device tensors (NCCL broadcasts of the counts, index and value buffers)
    and spgemm_owned multiplies them in place."""
    import os
    from datetime import timedelta
    import torch
    import torch.distributed as tdist
    from bcl_b200.containers import assemble_tiles
    from bcl_b200.distributed import ProcessGroups, exchange_operands, owned_input_tiles, spgemm_owned
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        torch.cuda.set_device(0)
        tdist.init_process_group("nccl", rank=0, world_size=1, timeout=timedelta(seconds=60))
        a = gen.rmat(11, seed=77)
        tm, tk, tn = 300, 200, 250
        dev = torch.device("cuda", 0)
        groups = ProcessGroups(1, 1, 1)
        a_own = owned_input_tiles(a, tm, tk, 0, 1, 1, device=dev)
        b_own = owned_input_tiles(a, tk, tn, 0, 1, 1, device=dev)
        a_rows, b_cols, I, J = exchange_operands(a_own, (a.m, a.n), b_own, (a.m, a.n), tm, tk, tn, 0,
                                                 groups, device=dev)
        on_device = all(t[0].is_cuda and t[1].is_cuda and t[2].is_cuda for t in list(a_rows.values()) +
                        list(b_cols.values()))
        C = spgemm_owned(a_rows, b_cols, I, J, (a.m, a.n), (a.m, a.n), tm, tk, tn, device=0)
        n = C.nnz()
        part = (I, J, C.tile_row_ptr.cpu().numpy(), C.tile_offset.cpu().numpy(), C.col_ind[:n].cpu().numpy(),
                C.vals[:n].cpu().numpy())
        whole = assemble_tiles(a.m, a.n, tm, tn, [part])
        rp, ci, cv = O.gemm_tiled(a, a, tm, tk, tn)
        same = (np.array_equal(whole.row_ptr.astype(np.int64), rp) and np.array_equal(whole.col_ind, ci)
                and np.array_equal(whole.vals.view(np.uint32), cv.view(np.uint32)))
        q.put((on_device, same))
    except Exception as e:  # reported to the parent
        q.put(repr(e))
    finally:
        if tdist.is_initialized():
            tdist.destroy_process_group()


def test_exchange_over_nccl_one_rank():
    """The device path of the operand exchange over NCCL on one GPU (one
    rank: the owner's broadcasts of its own tiles; the receiving side is
    covered by the gloo ranks on CPU), then the owned product from the
    device tiles, bit-identical to the whole product."""
    import multiprocessing
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = multiprocessing.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_nccl_exchange_one_rank, args=(port, q))
    p.start()
    p.join(240)
    if p.is_alive():
        p.kill()
        p.join()
        pytest.fail("the one-rank NCCL exchange did not finish in 240 s")
    res = q.get(timeout=5)
    assert res == (True, True), res


def _dense_grids(a, b, c0, tiles, dtype):
    import torch
    from bcl_b200.containers import BlockCustom, DMatrix, SPMatrix
    tm, tk, tn = tiles
    A = SPMatrix.from_csr(a, BlockCustom((tm, tk)))
    if dtype == "f32":
        B = DMatrix.from_array(torch.from_numpy(b), BlockCustom((tk, tn)))
        C = DMatrix.from_array(torch.from_numpy(c0), BlockCustom((tm, tn)))
    else:
        as_bf16 = lambda x: torch.from_numpy(x.view(np.int16)).view(torch.bfloat16)
        B = DMatrix.from_array(as_bf16(b), BlockCustom((tk, tn)), dtype=torch.bfloat16)
        C = DMatrix.from_array(as_bf16(c0), BlockCustom((tm, tn)), dtype=torch.bfloat16)
    return A, B, C


def _dense_out(C, dtype):
    import torch
    out = C.get_matrix().cpu()
    return out.numpy() if dtype == "f32" else out.view(torch.int16).numpy().view(np.uint16)


@pytest.mark.parametrize("dtype", ["f32", "bf16"])
@pytest.mark.parametrize("case", ["rmat_2x2", "rmat_3x1_ragged", "long_rows_4x1"])
def test_spmm_sub_grids_cover_the_whole_product(monkeypatch, dtype, case):
    """Every process's C tiles of the sparse x dense product computed in turn
    on one GPU (bclx_spmm_grid_sub: one launch per process, each C tile in
    the rotated stage order of its global position), in place in the whole
    C: the result is the whole product bit for bit (FP32 against the oracle,
    BF16 storage against the oracle's BF16 restatement).  Covers ragged
    tiles, 12 tiles along k, and rows long enough for the long-row kernel."""
    from bcl_b200.containers import owned_tiles, spmm_sub
    from test_gpu_spmm import heavy_rows_matrix
    if case == "rmat_2x2":
        a, tiles, pgrid, n = gen.rmat(13, seed=81), (4096, 4096, 128), (2, 2), 256
    elif case == "rmat_3x1_ragged":
        a, tiles, pgrid, n = gen.rmat(13, seed=82), (1000, 700, 64), (3, 1), 200
    else:
        monkeypatch.setenv("BCLX_SPMM_LONG_MIN_ROWS", "0")
        a, tiles, pgrid, n = heavy_rows_matrix(), (4096, 4096, 256), (4, 1), 256
    b = gen.dense(a.n, n, seed=83, dist="normal")
    c0 = gen.dense(a.m, n, seed=84)
    if dtype == "bf16":
        b, c0 = O.to_bf16(b), O.to_bf16(c0)
    A, B, C = _dense_grids(a, b, c0, tiles, dtype)
    pm, pn = pgrid
    for p in range(pm * pn):
        rows, cols = owned_tiles(C.gm, C.gn, p, pm, pn)
        spmm_sub(A, B, C, rows, cols)
    got = _dense_out(C, dtype)
    if dtype == "f32":
        want = O.spmm_tiled(a, b, c0, *tiles)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    else:
        assert np.array_equal(got, O.spmm_tiled_bf16(a, b, c0, *tiles))


def test_spmm_owned_from_fetched_operands():
    """Each process's C tiles from its received operands (A's tile rows I as
    a compact sparse grid, B's tile columns J and its own C tiles as compact
    dense grids; bcl_b200.distributed.spmm_owned), 2 x 2 processes, ragged
    tiles: the tiles assemble to the whole product bit for bit."""
    import torch
    from bcl_b200.distributed import host_tile, owned_dense_tiles, spmm_owned
    a = gen.rmat(13, seed=85)
    n = 200
    b = gen.dense(a.n, n, seed=86, dist="normal")
    c0 = gen.dense(a.m, n, seed=87)
    tm, tk, tn = 1000, 700, 64
    gm, gk, gn = -(-a.m // tm), -(-a.n // tk), -(-n // tn)
    pm, pn = 2, 2
    whole = np.array(c0, copy=True)
    for p in range(pm * pn):
        r, c = divmod(p, pn)
        I = [i for i in range(gm) if i % pm == r]
        J = [j for j in range(gn) if j % pn == c]
        a_rows = {(i, k): tuple(torch.from_numpy(x) for x in host_tile(a, tm, tk, i, k)) for i in I for k in range(gk)}
        b_all = owned_dense_tiles(b, tk, tn, 0, 1, 1)
        b_cols = {(k, j): b_all[(k, j)] for k in range(gk) for j in J}
        c_tiles = owned_dense_tiles(c0, tm, tn, p, pm, pn)
        out = spmm_owned(a_rows, b_cols, c_tiles, I, J, (a.m, a.n), (a.n, n), tm, tk, tn, device=0)
        assert set(out) == set(c_tiles)
        for (i, j), t in out.items():
            blk = whole[i * tm:(i + 1) * tm, j * tn:(j + 1) * tn]
            blk[...] = t.cpu().numpy()[:blk.shape[0], :blk.shape[1]]
    want = O.spmm_tiled(a, b, c0, tm, tk, tn)
    assert np.array_equal(whole.view(np.uint32), want.view(np.uint32))
