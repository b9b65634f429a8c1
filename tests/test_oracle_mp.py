"""The reference's own distributed BCL::gemm on several ranks (CPU).

oracle/_ref/bcl_ref_mp is the reference's SUMMA loop compiled from its
unmodified headers over the shared-memory MPI subset (oracle/ref_stubs_mp):
tiles on their block-cyclic owners (SPMatrix.hpp:230-237, DMatrix.hpp:75-90),
remote tiles fetched one-sidedly, pointers broadcast, barriers between the
phases (spgemm.hpp:153-242).  Its result on 2, 3, 4 and 6 ranks equals the
oracle bit for bit: the per-tile order of sums does not depend on the
process grid, which is what lets every process of the GPU path compute its
own C tiles (bclx_spgemm_symbolic_sub, bclx_spmm_grid_sub) and match."""
import numpy as np
import pytest

from bcl_b200 import gen
from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.ref_mp_available(),
                                reason="the multi-rank reference binary oracle/_ref/bcl_ref_mp is not built")


@pytest.mark.parametrize("pgrid,mode", [((1, 2), "f32"), ((2, 2), "f32"), ((3, 1), "i32"), ((2, 3), "f32"),
                                        ((2, 2), "i32")])
def test_distributed_reference_spgemm_matches_oracle(pgrid, mode):
    a = gen.rmat(10, seed=41, value_type=mode)
    b = gen.rmat(10, seed=42, value_type=mode)
    tiles = (200, 150, 250)  # ragged in every dimension
    c, res = O.ref_spgemm_mp(a, b, *tiles, pgrid, mode=mode)
    assert res["ranks"] == pgrid[0] * pgrid[1]
    rp, ci, cv = O.gemm_tiled(a, b, *tiles, mode=mode)
    assert np.array_equal(c.row_ptr.astype(np.int64), rp) and np.array_equal(c.col_ind, ci)
    assert np.array_equal(c.vals.view(np.uint32), cv.view(np.uint32))


@pytest.mark.parametrize("pgrid", [(2, 2), (3, 1), (1, 3)])
def test_distributed_reference_spmm_matches_oracle(pgrid):
    a = gen.rmat(10, seed=43)
    n = 96
    b = gen.dense(a.n, n, seed=44)
    tiles = (200, 150, 40)
    c, res = O.ref_spmm_mp(a, b, *tiles, pgrid)
    assert res["ranks"] == pgrid[0] * pgrid[1]
    want = O.spmm_tiled(a, b, np.zeros((a.m, n), np.float32), *tiles)
    assert np.array_equal(c.view(np.uint32), want.view(np.uint32))


def test_distributed_reference_same_as_one_rank():
    """The distributed run and the one-rank reference agree bit for bit
    (timing fields aside), and more ranks than C tiles leave ranks idle."""
    a = gen.rmat(9, seed=45)
    c1, _ = O.ref_spgemm(a, a, 256, 256, 256)
    c4, res = O.ref_spgemm_mp(a, a, 256, 256, 256, (2, 3))  # a 2 x 2 tile grid on 6 ranks
    assert res["ranks"] == 6
    assert np.array_equal(c1.row_ptr, c4.row_ptr) and np.array_equal(c1.col_ind, c4.col_ind)
    assert np.array_equal(c1.vals.view(np.uint32), c4.vals.view(np.uint32))


def test_failing_rank_ends_the_run(tmp_path):
    """A rank that cannot start (its input is missing) ends the call with an
    error instead of leaving the other ranks waiting."""
    a = gen.rmat(8, seed=46)
    fa = tmp_path / "a.binary"
    gen.write_binary(str(fa), a)
    with pytest.raises(RuntimeError):
        O.run_ref_mp(["spgemm", str(fa), str(tmp_path / "missing.binary"), 64, 64, 64, 1, 2, "f32", "-", 0, 1], 2,
                     timeout=120)
