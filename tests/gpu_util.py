"""Helpers shared by the GPU parity tests."""
import os

import numpy as np

from bcl_b200 import gen

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_csr(d, prefix):
    m, n = (int(x) for x in d[f"{prefix}_shape"])
    return gen.CSR(m, n, d[f"{prefix}_row_ptr"], d[f"{prefix}_col_ind"], d[f"{prefix}_vals"])


def bits(x):
    x = np.asarray(x)
    return x.view(np.uint32) if x.dtype == np.float32 else x


def assert_csr_identical(got, row_ptr, col_ind, vals):
    """Structure and values bit-for-bit (FP32 compared as bit patterns)."""
    assert np.array_equal(np.asarray(got.row_ptr, np.int64), np.asarray(row_ptr, np.int64)), "row_ptr differs"
    assert np.array_equal(got.col_ind, col_ind), "col_ind differs"
    assert np.array_equal(bits(got.vals), bits(vals)), "values differ"


def assert_rel_close(got, want, rtol):
    """|got - want| <= rtol * |want| per entry (+ a tiny absolute floor for exact zeros)."""
    got, want = np.asarray(got, np.float64), np.asarray(want, np.float64)
    err = np.abs(got - want)
    bound = rtol * np.abs(want) + 1e-30
    bad = err > bound
    assert not bad.any(), f"{int(bad.sum())} entries off; worst {float((err / (np.abs(want) + 1e-30)).max())}"
