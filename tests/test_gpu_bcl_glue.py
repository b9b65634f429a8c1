"""The drop-in at the reference's own container level (include/bclx_bcl.hpp).

oracle/_ref/bcl_glue_check is compiled against the unmodified reference
headers (oracle/Makefile): on the same BCL::SPMatrix / BCL::DMatrix objects
it runs the reference's BCL::gemm on the host and BCL::bclx::gemm (tiles read
through their GlobalPtr handles, multiplied on the GPU through the C ABI,
written back with assign_tile / into the C tiles) and compares every output
tile bit for bit.  Ragged tile grids, FP32 and int32, and the SpMM overload
with a nonzero starting C."""
import json
import os
import subprocess

import pytest

from bcl_b200 import gen

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GLUE = os.path.join(ROOT, "oracle", "_ref", "bcl_glue_check")


@pytest.fixture(scope="module", autouse=True)
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not os.path.exists(GLUE):
        pytest.skip("bcl_glue_check not built (needs the reference tree at build time)")


@pytest.mark.parametrize("value_type,tiles,n", [("f32", (256, 256, 256), 64), ("f32", (300, 700, 260), 40),
                                                ("i32", (512, 333, 600), 0)])
def test_reference_containers_through_the_glue(tmp_path, value_type, tiles, n):
    a = gen.rmat(11, seed=91, value_type=value_type)
    fa = str(tmp_path / "a.binary")
    gen.write_binary(fa, a)
    out = subprocess.run([GLUE, fa, *map(str, tiles), value_type, str(n)], capture_output=True, text=True,
                         timeout=300)
    line = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert line, out.stdout + out.stderr
    res = json.loads(line[-1])
    assert out.returncode == 0, res
    assert res["spgemm_identical"] and res["spmm_identical"] and res["nnz"] > 0


GLUE_MP = os.path.join(ROOT, "oracle", "_ref", "bcl_glue_check_mp")


@pytest.mark.parametrize("pgrid,value_type,tiles,n", [((1, 2), "f32", (300, 700, 260), 40),
                                                      ((2, 2), "f32", (256, 256, 256), 64),
                                                      ((2, 1), "i32", (512, 333, 600), 0)])
def test_reference_containers_through_the_glue_on_ranks(tmp_path, pgrid, value_type, tiles, n):
    """The reference's containers distributed over a process grid, each rank
    a process on this GPU (over the shared-memory MPI subset): every rank
    fetches its operand tiles through get_tile and computes its own C tiles
    in one sub-grid call; rank 0 compares every tile with the reference's
    distributed BCL::gemm, bit for bit."""
    from oracle import oracle as O
    if not os.path.exists(GLUE_MP):
        pytest.skip("bcl_glue_check_mp not built (needs the reference tree at build time)")
    a = gen.rmat(11, seed=92, value_type=value_type)
    fa = str(tmp_path / "a.binary")
    gen.write_binary(fa, a)
    pm, pn = pgrid
    res = O.run_ref_mp([fa, *tiles, value_type, n, pm, pn], pm * pn, timeout=300, binary=GLUE_MP)
    assert res["ranks"] == pm * pn
    assert res["spgemm_identical"] and res["spmm_identical"] and res["nnz"] > 0
