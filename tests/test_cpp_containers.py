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


def _random_mtx(path, rng, m, n, count, field, symmetric):
    i = rng.integers(1, m + 1, count)
    j = rng.integers(1, n + 1, count)
    if symmetric:
        i, j = np.maximum(i, j), np.minimum(i, j)
    rep = rng.random(count) < 0.15  # repeated indices with other values
    src = rng.integers(0, count, count)
    i, j = np.where(rep, i[src], i), np.where(rep, j[src], j)
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate {field} {'symmetric' if symmetric else 'general'}\n% seeded\n")
        f.write(f"{m} {n} {count}\n")
        for a, b in zip(i, j):
            if field == "pattern":
                f.write(f"{a} {b}\n")
            elif field == "integer":
                f.write(f"{a} {b} {int(rng.integers(-50, 51))}\n")
            else:
                f.write(f"{a} {b} {rng.normal():.7g}\n")


@pytest.mark.parametrize("seed,field,symmetric", [(1, "real", False), (2, "real", True), (3, "pattern", False),
                                                  (4, "pattern", True), (5, "integer", False), (6, "integer", True)])
def test_matrix_market_readers_match_live_reference(program, tmp_path, seed, field, symmetric):
    """Fresh seeded MatrixMarket files (repeated indices, symmetric,
    pattern, integer): the reference's own reader (the compiled reference
    binary), the Python reader and the C++ header's reader agree bit for
    bit."""
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("reference binary not built")
    rng = np.random.default_rng(seed)
    path = str(tmp_path / "x.mtx")
    m = int(rng.integers(20, 90))
    n = m if symmetric else int(rng.integers(20, 90))  # symmetric files are square
    _random_mtx(path, rng, m, n, 400, field, symmetric)
    dt = "i32" if field == "integer" else "f32"
    vt = np.float32 if dt == "f32" else np.int32
    subprocess.run([O.REF_BIN, "mmread", path, dt, str(tmp_path / "ref.binary")], check=True, timeout=60)
    r = subprocess.run([program, "mmread", path, dt, str(tmp_path / "cpp.binary")], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode == 0, r.stderr
    ref = gen.read_binary(str(tmp_path / "ref.binary"), vt)
    for got in (gen.read_binary(str(tmp_path / "cpp.binary"), vt), gen.read_matrix_market(path, vt)):
        assert (got.m, got.n) == (ref.m, ref.n)
        assert np.array_equal(got.row_ptr, ref.row_ptr) and np.array_equal(got.col_ind, ref.col_ind)
        assert np.array_equal(np.asarray(got.vals, vt).view(np.uint32), ref.vals.view(np.uint32))


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
