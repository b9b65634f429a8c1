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
