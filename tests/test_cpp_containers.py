"""The header-only C++ containers (include/bclx_containers.hpp): BCL's
SPMatrix / DMatrix / gemm names over the C ABI, used from a C++ program that
reads the reference's binary CSR format.  The CPU tests compile it and check
its MatrixMarket reader against the reference's reader (golden fixtures); the
GPU test runs it (device slicing, gemm, dot, the tile members) and compares
both products with the oracle bit for bit."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from bcl_b200 import gen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def compile_program(out_dir):
    exe = os.path.join(out_dir, "test_containers")
    libdir = os.path.join(ROOT, "bcl_b200")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), "-I",
           os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "cpp", "test_containers.cpp"), "-o", exe,
           "-L", libdir, "-lbclx", "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{libdir}",
           f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    from bcl_b200 import _lib
    _lib.load()  # builds libbclx.so if it is missing
    return compile_program(str(tmp_path_factory.mktemp("cpp")))


def test_cpp_containers_compile(program):
    assert os.path.exists(program)


@pytest.mark.parametrize("name", ["general_real_dups", "symmetric_real", "pattern_general", "integer_general"])
def test_cpp_matrix_market_reader_golden(program, tmp_path, name):
    """The header's MatrixMarket reader (CSR<T>::read, host only) against
    what the reference's own reader made of the same files."""
    from gpu_util import GOLD
    d = np.load(os.path.join(GOLD, f"mm_{name}.npz"))
    dt = str(d["dtype"])
    out = str(tmp_path / "c.binary")
    r = subprocess.run([program, "mmread", os.path.join(GOLD, f"mm_{name}.mtx"), dt, out], capture_output=True,
                       text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    vt = np.float32 if dt == "f32" else np.int32
    c = gen.read_binary(out, vt)
    assert (c.m, c.n) == tuple(int(x) for x in d["c_shape"])
    assert np.array_equal(c.row_ptr, d["c_row_ptr"]) and np.array_equal(c.col_ind, d["c_col_ind"])
    assert np.array_equal(c.vals.view(np.uint32), d["c_vals"].astype(vt).view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("tiles", [(256, 256, 256), (300, 700, 260)])
def test_cpp_containers_match_oracle(program, tmp_path, tiles):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from oracle import oracle as O
    a = gen.rmat(10, seed=7)
    b = gen.dense(a.n, 40, seed=8)
    gen.write_binary(str(tmp_path / "a.binary"), a)
    gen.write_dense(str(tmp_path / "b.dense"), b)
    r = subprocess.run([program, str(tmp_path)] + [str(t) for t in tiles], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    c = gen.read_binary(str(tmp_path / "c.binary"))
    rp, ci, cv = O.gemm_tiled(a, a, *tiles)
    assert np.array_equal(c.row_ptr, rp) and np.array_equal(c.col_ind, ci)
    assert np.array_equal(c.vals.view(np.uint32), cv.view(np.uint32))
    e = gen.read_binary(str(tmp_path / "e.binary"))  # A rebuilt tile by tile with assign_tile
    assert np.array_equal(e.row_ptr, a.row_ptr) and np.array_equal(e.col_ind, a.col_ind)
    assert np.array_equal(e.vals.view(np.uint32), a.vals.view(np.uint32))
    d = gen.read_dense(str(tmp_path / "c.dense"))
    want = O.spmm_tiled(a, b, np.zeros((a.m, 40), np.float32), tiles[0], tiles[1], 40)
    assert np.array_equal(d.view(np.uint32), want.view(np.uint32))
