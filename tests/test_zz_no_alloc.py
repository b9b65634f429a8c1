"""GPU test of bclx_spgemm_tile_noalloc, the tile product for callers that
cannot allocate device memory when they call (a framework that has reserved
the device's memory for its own allocator, or code that must not call
cudaMalloc/cudaFree because those synchronize the device).

It is checked through the C ABI against the regular two-phase entry points
(bclx_spgemm_symbolic/_numeric on 1x1 grids) and against the oracle (the CPU
restatement of the reference's local product) on two calls in a row with
different inputs, so that the second call also shows that whatever the
first call left in the shared scratch array does not leak into its result.
The tolerance is the one the other SpGEMM tests use: bit-for-bit.  Further
cases: an empty A (row pointer written as zeros), the two rejections (B wider
than 16384 columns, a product whose work arrays exceed the 32 MiB scratch)
leaving the output arrays untouched, a B too tall for the B-row table in
what is left of the scratch (binary-search fallback), and a check that a
call leaves the device's free memory unchanged.  This file is collected last
so that a run stopping at the first failure has already run every other
test; it passes alone in a fresh process as well."""
import ctypes

import numpy as np
import pytest

from bcl_b200 import gen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def desc(mat, tensors):
    import torch
    from bcl_b200 import _lib
    rp = torch.from_numpy(mat.row_ptr.astype(np.int32)).cuda()
    ci = torch.from_numpy(mat.col_ind.astype(np.int32) if mat.nnz else np.zeros(1, np.int32)).cuda()
    v = torch.from_numpy(np.ascontiguousarray(mat.vals) if mat.nnz else np.zeros(1, mat.vals.dtype)).cuda()
    tensors += [rp, ci, v]
    dt = _lib.F32 if mat.vals.dtype == np.float32 else _lib.I32
    return _lib.CSRDesc(mat.m, mat.n, mat.nnz, rp.data_ptr(), ci.data_ptr(), v.data_ptr(), dt, 0)


def noalloc_product(a, b, capacity=None, raw=False):
    """Returns (status, nnz, row_ptr, col_ind, vals) from the no-allocation
    call; with raw=True col_ind and vals are the whole output arrays (to see
    that a rejected call left them untouched)."""
    import torch
    from bcl_b200 import _lib
    keep = []
    da, db = desc(a, keep), desc(b, keep)
    if capacity is None:
        from oracle import oracle as O
        capacity = int(O.spgemm_count(a, b).sum())
    c_rp = torch.full((a.m + 1,), -1, dtype=torch.int32, device="cuda")
    c_ci = torch.full((max(capacity, 1),), -7, dtype=torch.int32, device="cuda")
    c_v = torch.full((max(capacity, 1),), -7, dtype=torch.float32 if a.vals.dtype == np.float32 else torch.int32,
                     device="cuda")
    nnz = ctypes.c_int64(-1)
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    rc = _lib.load().bclx_spgemm_tile_noalloc(ctypes.byref(da), ctypes.byref(db), ctypes.c_void_p(c_rp.data_ptr()),
                                              ctypes.c_void_p(c_ci.data_ptr()), ctypes.c_void_p(c_v.data_ptr()),
                                              capacity, ctypes.byref(nnz), ctypes.c_void_p(stream))
    torch.cuda.synchronize()
    k = int(nnz.value)
    if raw:
        return rc, k, c_rp.cpu().numpy(), c_ci.cpu().numpy(), c_v.cpu().numpy()
    return (rc, k, c_rp.cpu().numpy(), c_ci[:k].cpu().numpy() if k <= capacity else None,
            c_v[:k].cpu().numpy() if k <= capacity else None)


def oracle_product(a, b):
    from oracle import oracle as O
    mode = "f32" if a.vals.dtype == np.float32 else "i32"
    return O.spgemm_local(a, b, mode=mode)


def two_phase_product(a, b):
    """The existing entry points on 1x1 grids (one tile each)."""
    from bcl_b200.containers import BlockCustom, SPMatrix, spgemm
    A = SPMatrix.from_csr(a, BlockCustom((a.m, a.n)))
    B = SPMatrix.from_csr(b, BlockCustom((b.m, b.n)))
    return spgemm(A, B).get_tile((0, 0))


def bits(x):
    return x.view(np.uint32) if x.dtype == np.float32 else x


def test_no_alloc_matches_two_phase_on_two_calls_in_a_row():
    from bcl_b200 import _lib
    # first call: R-MAT s12, FP32 (light and heavy rows); second: a different
    # shape and int32 values, after the first left its data in the scratch
    cases = [(gen.rmat(12, seed=41), None), (gen.rmat(11, seed=42, value_type="i32"), None)]
    a2 = gen.rmat(11, seed=43, value_type="i32")
    cases[1] = (cases[1][0], a2)
    for a, b in cases:
        b = a if b is None else b
        rc, nnz, rp, ci, v = noalloc_product(a, b)
        assert rc == _lib.OK, _lib.load().bclx_last_error()
        ref = two_phase_product(a, b)
        assert nnz == ref.nnz
        assert np.array_equal(rp, ref.row_ptr)
        assert np.array_equal(ci, ref.col_ind)
        assert np.array_equal(bits(v), bits(ref.vals))
        orp, oci, ov = oracle_product(a, b)
        assert np.array_equal(rp.astype(np.int64), orp)
        assert np.array_equal(ci, oci)
        assert np.array_equal(bits(v), bits(ov))


def test_no_alloc_reports_too_small_output():
    from bcl_b200 import _lib
    a = gen.rmat(10, seed=44)
    ref = two_phase_product(a, a)
    rc, nnz, rp, _, _ = noalloc_product(a, a, capacity=ref.nnz - 1)
    assert rc == _lib.ERR_INVALID
    assert nnz == ref.nnz and np.array_equal(rp, ref.row_ptr)
    # the next call with enough room still agrees
    rc, nnz, rp, ci, v = noalloc_product(a, a, capacity=ref.nnz)
    assert rc == _lib.OK and np.array_equal(ci, ref.col_ind) and np.array_equal(bits(v), bits(ref.vals))


def test_no_alloc_empty_a_writes_zero_row_ptr():
    from bcl_b200 import _lib
    b = gen.rmat(8, seed=45)
    a = gen.CSR(0, b.m, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32))
    rc, nnz, rp, _, _ = noalloc_product(a, b, capacity=0)
    assert rc == _lib.OK and nnz == 0
    assert rp.tolist() == [0]


def test_no_alloc_rejects_wide_b_and_leaves_output():
    from bcl_b200 import _lib
    rng = np.random.default_rng(46)
    a = gen.rmat(8, seed=46)
    n = 16385
    rp = np.arange(a.n + 1, dtype=np.int32)
    b = gen.CSR(a.n, n, rp, rng.integers(0, n, a.n).astype(np.int32), rng.uniform(-1, 1, a.n).astype(np.float32))
    rc, nnz, crp, ci, v = noalloc_product(a, b, capacity=64, raw=True)
    assert rc == _lib.ERR_INVALID
    assert "16384" in _lib.load().bclx_last_error().decode()
    assert (ci == -7).all() and (v == -7).all()


def test_no_alloc_rejects_oversized_work_and_leaves_output():
    """A tall A (2^21 rows): the row lists alone exceed the 32 MiB scratch."""
    from bcl_b200 import _lib
    m, k = 1 << 21, 64
    rng = np.random.default_rng(47)
    rp = np.zeros(m + 1, np.int32)
    rp[1:] = np.minimum(np.arange(1, m + 1), 4096)   # the first 4096 rows hold one entry each
    a = gen.CSR(m, k, rp, rng.integers(0, k, 4096).astype(np.int32), rng.uniform(-1, 1, 4096).astype(np.float32))
    b = gen.CSR(k, k, np.arange(k + 1, dtype=np.int32), np.arange(k, dtype=np.int32), np.ones(k, np.float32))
    rc, nnz, crp, ci, v = noalloc_product(a, b, capacity=8192, raw=True)
    assert rc == _lib.ERR_INVALID
    assert "scratch" in _lib.load().bclx_last_error().decode()
    assert (ci == -7).all() and (v == -7).all()


def test_no_alloc_b_too_tall_for_the_row_table():
    """B with 2^21 rows and 16384 columns: its B-row table (65 entries per B
    row) does not fit in the scratch, so heavy items binary-search B rows;
    the result is still the oracle's, bit for bit."""
    from bcl_b200 import _lib
    rng = np.random.default_rng(48)
    k, n, m = 1 << 21, 16384, 300
    per_b = 2
    b_rp = np.arange(0, per_b * k + 1, per_b, dtype=np.int32)
    b_ci = np.sort(rng.integers(0, n, (k, per_b)), axis=1).astype(np.int32)
    b_ci[:, 1] = np.maximum(b_ci[:, 1], b_ci[:, 0] + 1)
    b_ci = np.minimum(b_ci, n - 1)
    b_ci[:, 0] = np.minimum(b_ci[:, 0], b_ci[:, 1] - 1)
    b = gen.CSR(k, n, b_rp, b_ci.reshape(-1), rng.uniform(-1, 1, per_b * k).astype(np.float32))
    per_a = 600
    a_ci = np.sort(np.stack([rng.choice(k, per_a, replace=False) for _ in range(m)]), axis=1).astype(np.int32)
    a = gen.CSR(m, k, np.arange(0, per_a * m + 1, per_a, dtype=np.int32), a_ci.reshape(-1),
                rng.uniform(-1, 1, per_a * m).astype(np.float32))
    rc, nnz, rp, ci, v = noalloc_product(a, b)
    assert rc == _lib.OK, _lib.load().bclx_last_error()
    orp, oci, ov = oracle_product(a, b)
    assert np.array_equal(rp.astype(np.int64), orp)
    assert np.array_equal(ci, oci)
    assert np.array_equal(bits(v), bits(ov))


def test_no_alloc_allocates_nothing():
    """After a first call (which may load the library's kernels), another
    call leaves the device's free memory exactly as it was."""
    import torch
    from bcl_b200 import _lib
    a = gen.rmat(11, seed=49)
    assert noalloc_product(a, a)[0] == _lib.OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    rc, *_ = noalloc_product(a, a)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert rc == _lib.OK
    # noalloc_product's own output tensors come from torch's cache, already
    # reserved by the first call
    assert free1 == free0
