"""Seeded synthetic inputs for the sparse tile multiply, and the reference's
binary CSR file format.

The reference ships no generators or fixtures for its matrix path; its only
synthetic generator (examples/matrix/generate_spmat.hpp:58-116) draws uniform
or zipf columns with drand48 and injects tiles through
``SPMatrix::assign_tile``.  The inputs named for this path are:

* Erdos-Renyi: ``n x n`` with exactly ``nnz_per_row`` distinct uniform columns
  per row (sampled without replacement), values U(-1, 1) FP32.
* R-MAT: ``2**scale`` square, ``edge_factor * n`` edges, quadrant
  probabilities a/b/c/d, duplicates merged and self-loops kept.  Values are
  FP32 U(-1, 1) or int32 uniform in [-8, 8].
* 3-D 27-point stencil Laplacian on a ``g**3`` grid: 26 on the diagonal and -1
  on each of the (up to) 26 neighbours.
* Dense row-major blocks: U(-1, 1) or N(0, 1) FP32.

Every matrix is returned as a :class:`CSR` with sorted, unique column indices
per row, which is the form ``CSRMatrix::assign`` produces
(bcl/containers/sequential/CSRMatrix.hpp:107-165).
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np


@dataclasses.dataclass
class CSR:
    """Host CSR matrix: int32 ``row_ptr[m+1]``, int32 ``col_ind[nnz]`` (sorted
    within each row) and ``vals[nnz]`` (float32 or int32)."""

    m: int
    n: int
    row_ptr: np.ndarray
    col_ind: np.ndarray
    vals: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[-1])

    @property
    def dtype(self):
        return self.vals.dtype

    def row_nnz(self) -> np.ndarray:
        return np.diff(self.row_ptr)

    def copy(self) -> "CSR":
        return CSR(self.m, self.n, self.row_ptr.copy(), self.col_ind.copy(), self.vals.copy())

    def astype(self, dtype) -> "CSR":
        return CSR(self.m, self.n, self.row_ptr, self.col_ind, self.vals.astype(dtype))


def _csr_from_sorted_keys(keys: np.ndarray, m: int, n: int, vals: np.ndarray) -> CSR:
    rows = keys // n
    cols = (keys - rows * n).astype(np.int32)
    counts = np.bincount(rows, minlength=m)
    row_ptr = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    if row_ptr[-1] >= 2**31:
        raise ValueError("matrix has more than 2**31-1 nonzeros; int32 row_ptr cannot hold it")
    return CSR(m, n, row_ptr.astype(np.int32), cols, vals)


def _sorted_unique(keys: np.ndarray) -> np.ndarray:
    """Sorted distinct values (np.unique, without its slow path on large int64 arrays)."""
    keys.sort()
    if keys.size == 0:
        return keys
    keep = np.empty(keys.size, dtype=bool)
    keep[0] = True
    np.not_equal(keys[1:], keys[:-1], out=keep[1:])
    return keys[keep]


def _values(rng: np.random.Generator, count: int, value_type: str) -> np.ndarray:
    if value_type == "f32":
        return rng.uniform(-1.0, 1.0, count).astype(np.float32)
    if value_type == "i32":
        return rng.integers(-8, 9, count, dtype=np.int64).astype(np.int32)
    raise ValueError(f"unknown value type {value_type!r}")


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
         seed: int = 0, value_type: str = "f32", chunk: int = 1 << 22) -> CSR:
    """R-MAT graph adjacency matrix (Chakrabarti, Zhan, Faloutsos 2004).

    Each of ``edge_factor * 2**scale`` edges descends ``scale`` levels of the
    recursive quadrant split with probabilities ``a`` (top-left), ``b``
    (top-right), ``c`` (bottom-left), ``d = 1 - a - b - c``.  Duplicate edges
    are merged (one entry) and self-loops are kept.
    """
    n = 1 << scale
    n_edges = edge_factor * n
    rng = np.random.default_rng(seed)
    keys = np.empty(n_edges, dtype=np.int64)
    ab, abc = a + b, a + b + c
    r = np.empty(chunk, dtype=np.float64)
    m1 = np.empty(chunk, dtype=bool)
    m2 = np.empty(chunk, dtype=bool)
    for start in range(0, n_edges, chunk):
        cnt = min(chunk, n_edges - start)
        rows = np.zeros(cnt, dtype=np.int64)
        cols = np.zeros(cnt, dtype=np.int64)
        rr, d, rt = r[:cnt], m1[:cnt], m2[:cnt]
        for level in range(scale):
            rng.random(out=rr)
            bit = np.int64(1) << np.int64(scale - 1 - level)
            # quadrant: [0,a) top-left, [a,a+b) top-right, [a+b,a+b+c) bottom-left, rest bottom-right
            np.greater_equal(rr, ab, out=d)
            np.add(rows, bit, out=rows, where=d)
            np.greater_equal(rr, a, out=rt)
            rt &= ~d
            rt |= rr >= abc
            np.add(cols, bit, out=cols, where=rt)
        keys[start:start + cnt] = rows * n + cols
    keys = _sorted_unique(keys)
    return _csr_from_sorted_keys(keys, n, n, _values(rng, keys.size, value_type))


def erdos_renyi(n: int, nnz_per_row: int = 16, seed: int = 0, value_type: str = "f32") -> CSR:
    """``n x n`` matrix with exactly ``nnz_per_row`` distinct uniform columns per
    row (sampled without replacement), values U(-1, 1)."""
    if nnz_per_row > n:
        raise ValueError("nnz_per_row exceeds the number of columns")
    rng = np.random.default_rng(seed)
    cols = rng.integers(0, n, size=(n, nnz_per_row), dtype=np.int64)
    while True:
        cols.sort(axis=1)
        dup = np.zeros_like(cols, dtype=bool)
        dup[:, 1:] = cols[:, 1:] == cols[:, :-1]
        nd = int(dup.sum())
        if nd == 0:
            break
        cols[dup] = rng.integers(0, n, size=nd, dtype=np.int64)
    keys = (np.arange(n, dtype=np.int64)[:, None] * n + cols).ravel()
    return _csr_from_sorted_keys(keys, n, n, _values(rng, keys.size, value_type))


def stencil27(g: int, value_type: str = "f32") -> CSR:
    """3-D 27-point Laplacian on a ``g x g x g`` grid (lexicographic x fastest):
    26 on the diagonal, -1 for every neighbour inside the grid."""
    n = g ** 3
    idx = np.arange(n, dtype=np.int64)
    x = idx % g
    y = (idx // g) % g
    z = idx // (g * g)
    col_blocks = []
    mask_blocks = []
    # Offsets in increasing linear offset order, so each row comes out sorted.
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                ok = ((x + dx >= 0) & (x + dx < g) & (y + dy >= 0) & (y + dy < g)
                      & (z + dz >= 0) & (z + dz < g))
                col_blocks.append(idx + dx + dy * g + dz * g * g)
                mask_blocks.append(ok)
    cols = np.stack(col_blocks, axis=1)
    mask = np.stack(mask_blocks, axis=1)
    diag = cols == idx[:, None]
    vals_full = np.where(diag, 26, -1)
    counts = mask.sum(axis=1)
    row_ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    vt = np.float32 if value_type == "f32" else np.int32
    return CSR(n, n, row_ptr.astype(np.int32), cols[mask].astype(np.int32), vals_full[mask].astype(vt))


def dense(m: int, n: int, seed: int = 0, dist: str = "uniform") -> np.ndarray:
    """Row-major FP32 ``m x n`` block: U(-1, 1) (``uniform``) or N(0, 1) (``normal``)."""
    rng = np.random.default_rng(seed)
    if dist == "uniform":
        return rng.uniform(-1.0, 1.0, size=(m, n)).astype(np.float32)
    if dist == "normal":
        return rng.standard_normal(size=(m, n), dtype=np.float32)
    raise ValueError(f"unknown distribution {dist!r}")


def intermediate_products(a: CSR, b: CSR) -> int:
    """Number of scalar multiply-adds of the row-by-row (Gustavson) product
    A*B: sum over A's entries (i, k) of nnz(B[k, :])."""
    blen = np.diff(b.row_ptr.astype(np.int64))
    return int(blen[a.col_ind].sum())


# ---- the reference's binary CSR format (CSRMatrix.hpp:489-530) ------------

def write_binary(path: str, mat: CSR) -> None:
    """``size_t m, n, nnz``; ``T vals[nnz]``; ``int col_ind[nnz]``; ``int row_ptr[m+1]``."""
    with open(path, "wb") as f:
        np.array([mat.m, mat.n, mat.nnz], dtype=np.uint64).tofile(f)
        mat.vals.tofile(f)
        mat.col_ind.astype(np.int32).tofile(f)
        mat.row_ptr.astype(np.int32).tofile(f)


def read_binary(path: str, value_dtype=np.float32) -> CSR:
    with open(path, "rb") as f:
        m, n, nnz = (int(v) for v in np.fromfile(f, dtype=np.uint64, count=3))
        vals = np.fromfile(f, dtype=value_dtype, count=nnz)
        col_ind = np.fromfile(f, dtype=np.int32, count=nnz)
        row_ptr = np.fromfile(f, dtype=np.int32, count=m + 1)
    return CSR(m, n, row_ptr, col_ind, vals)


# ---- MatrixMarket (matrix_io.hpp:218-356, CSRMatrix.hpp:370-410, 533-547) ----

def read_matrix_market(path: str, value_dtype=np.float32, one_indexed: bool = True) -> CSR:
    """Read a coordinate MatrixMarket file as the reference's mmread does:
    `general` or `symmetric` (an off-diagonal entry is also stored
    transposed), `pattern` values read as 1; an index repeated later in the
    file is ignored (the first one stays); entries sorted by (row, column).
    Other formats, indices out of range and more entries than announced are
    errors."""
    with open(path, "r") as f:
        header = f.readline().split()
        if len(header) < 5 or header[0] != "%%MatrixMarket" or header[1] != "matrix" or header[2] != "coordinate":
            raise RuntimeError(f"{path} could not be parsed as a Matrix Market file.")
        pattern = header[3] == "pattern"
        if header[4] == "general":
            symmetric = False
        elif header[4] == "symmetric":
            symmetric = True
        else:
            raise RuntimeError(f"{path} has an unsupported matrix type")
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        m, n, nnz = (int(x) for x in line.split()[:3])
        body = f.read()
    ncol = 2 if pattern else 3
    tok = np.array(body.split(), dtype=object)
    if tok.size % ncol:
        raise RuntimeError(f"read_MatrixMarket: malformed entry lines in {path}")
    tok = tok.reshape(-1, ncol)
    if tok.shape[0] > nnz:
        raise RuntimeError("read_MatrixMarket: error reading Matrix Market file, file has more nonzeros than reported.")
    i = tok[:, 0].astype(np.int64)
    j = tok[:, 1].astype(np.int64)
    if one_indexed:
        i -= 1
        j -= 1
    if ((i < 0) | (i >= m) | (j < 0) | (j >= n)).any():
        raise RuntimeError("read_MatrixMarket: file has nonzero out of bounds.")
    if pattern:
        v = np.ones(i.size, dtype=value_dtype)
    elif np.dtype(value_dtype).kind == "f":
        v = tok[:, 2].astype(np.float64).astype(value_dtype)
    else:
        v = tok[:, 2].astype(np.float64).astype(np.int64).astype(value_dtype)
    if symmetric:  # each line inserts (i, j), then (j, i) off the diagonal
        off = i != j
        k = np.arange(i.size, dtype=np.int64)
        i = np.concatenate([i, j[off]])
        j2 = np.concatenate([j, i[: k.size][off]])
        order_key = np.concatenate([2 * k, 2 * k[off] + 1])  # insertion order
        v = np.concatenate([v, v[off]])
        j = j2
    else:
        order_key = np.arange(i.size, dtype=np.int64)
    key = i * n + j
    # first insertion of every index wins
    o = np.lexsort((order_key, key))
    keep = np.ones(o.size, dtype=bool)
    keep[1:] = key[o][1:] != key[o][:-1]
    o = o[keep]
    return _csr_from_sorted_keys(key[o], m, n, v[o])


def write_matrix_market(path: str, mat: CSR) -> None:
    """CSRMatrix::write_MatrixMarket: an `integer general` header, then one
    `row col value` line per entry (1-based, value printed with %f)."""
    rows = np.repeat(np.arange(mat.m, dtype=np.int64), np.diff(mat.row_ptr.astype(np.int64)))
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate integer general\n")
        f.write(f"{mat.m} {mat.n} {mat.nnz}\n")
        for r, c, x in zip(rows + 1, mat.col_ind.astype(np.int64) + 1, mat.vals):
            f.write(f"{r} {c} {float(x):f}\n")


def read_matrix(path: str, value_dtype=np.float32) -> CSR:
    """By suffix, as matrix_io::detect_file_type: .mtx or .binary."""
    if path.endswith(".mtx"):
        return read_matrix_market(path, value_dtype)
    if path.endswith(".binary"):
        return read_binary(path, value_dtype)
    raise RuntimeError(f"matrix_info: Could not detect file format for \"{path}\"")


def write_dense(path: str, arr: np.ndarray) -> None:
    """``int64 m, n``; ``T data[m*n]`` row-major."""
    with open(path, "wb") as f:
        np.array(arr.shape, dtype=np.int64).tofile(f)
        np.ascontiguousarray(arr).tofile(f)


def read_dense(path: str, dtype=np.float32) -> np.ndarray:
    with open(path, "rb") as f:
        m, n = (int(v) for v in np.fromfile(f, dtype=np.int64, count=2))
        return np.fromfile(f, dtype=dtype, count=m * n).reshape(m, n)


def cache_dir() -> str:
    d = os.environ.get("BCLX_CACHE", os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), ".cache"))
    os.makedirs(d, exist_ok=True)
    return d
