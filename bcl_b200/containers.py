"""Device-resident tile containers and the gemm calls of BCL's matrix path,
over the bclx C ABI.

Python mirror of the reference's interface for this path
(bcl/containers/SPMatrix.hpp, DMatrix.hpp, algorithms/spgemm.hpp): the same
names and argument meaning — ``SPMatrix`` / ``DMatrix`` with a tile grid
chosen by a ``BlockCustom`` policy, ``grid_shape`` / ``tile_shape`` /
``tile_nnz`` / ``tile_rank`` / ``get_tile`` / ``assign_tile`` / ``get`` /
``dot``, and ``gemm(a, b, c)`` for sparse x sparse and sparse x dense.  Every
tile lives on one GPU (rank 0); torch supplies device memory and the current
stream, and all arithmetic runs in the CUDA kernels behind the C ABI.

Storage.  An SPMatrix keeps its CSR tiles packed in four device arrays, tile
t = i*grid_n + j owning ``col_ind/vals[tile_offset[t]:tile_offset[t+1]]`` and
``tile_row_ptr[t]`` (tile_m+1 local offsets), plus a device array of
``bclx_csr_t`` descriptors, one per tile, that the kernels read.  This is the
format the sparse product writes, so a product is again an SPMatrix without a
copy.  A DMatrix keeps ``grid_m*grid_n`` padded row-major tiles of
tile_m x tile_n in one allocation, as DMatrix does (DMatrix.hpp:55-95).
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from ._lib import CSRDesc, DGrid, SpGrid, SpGridOut, call
from .gen import CSR

_NP_TO_DT = {np.dtype(np.float32): _lib.F32, np.dtype(np.int32): _lib.I32}
_TORCH_OF = {_lib.F32: torch.float32, _lib.I32: torch.int32, _lib.BF16: torch.bfloat16}


def _ceil_div(a: int, b: int) -> int:
    return (a + b - 1) // b


# ---- context ------------------------------------------------------------------


class Context:
    """A bclx context on one device; every call runs on torch's current stream."""

    def __init__(self, device: int = 0):
        if not torch.cuda.is_available():
            raise RuntimeError("bcl_b200 needs a CUDA device (B200, sm_100a); none is visible")
        self.device = device
        h = ctypes.c_void_p()
        call("bclx_context_create", device, ctypes.byref(h))
        self.h = h

    def use_current_stream(self):
        s = torch.cuda.current_stream(self.device).cuda_stream
        if s != getattr(self, "_stream", None):  # the C call only when the stream changes
            call("bclx_context_set_stream", self.h, ctypes.c_void_p(s))
            self._stream = s
        return self.h

    def release_cached(self):
        """Return the scratch pool's cached device memory to the driver."""
        call("bclx_context_release_cached", self.use_current_stream())

    def synchronize(self):
        """Wait for the current stream (bclx_context_synchronize)."""
        call("bclx_context_synchronize", self.use_current_stream())

    TUNING_KEYS = {"light_ub": _lib.TUNE_LIGHT_UB, "learn_target": _lib.TUNE_LEARN_TARGET,
                   "btable_max_bytes": _lib.TUNE_BTABLE_MAX_BYTES, "spmm_rows": _lib.TUNE_SPMM_ROWS,
                   "spmm_long_row": _lib.TUNE_SPMM_LONG_ROW, "spmm_long_blocks": _lib.TUNE_SPMM_LONG_BLOCKS,
                   "spmm_schedule": _lib.TUNE_SPMM_SCHEDULE, "item_outputs": _lib.TUNE_ITEM_OUTPUTS,
                   "wide_light": _lib.TUNE_WIDE_LIGHT, "spmm_panel_major": _lib.TUNE_SPMM_PANEL_MAJOR}

    def set_tuning(self, **knobs) -> None:
        """bclx_context_set_tuning for each name=value (None: the default)."""
        for k, v in knobs.items():
            call("bclx_context_set_tuning", self.h, self.TUNING_KEYS[k], -1 if v is None else int(v))

    def get_tuning(self, name: str) -> int:
        v = ctypes.c_int64()
        call("bclx_context_get_tuning", self.h, self.TUNING_KEYS[name], ctypes.byref(v))
        return int(v.value)

    def tuned(self, **knobs):
        """Context manager: the knobs set inside the block, the previous values after."""
        import contextlib

        @contextlib.contextmanager
        def cm():
            old = {k: self.get_tuning(k) for k in knobs}
            self.set_tuning(**knobs)
            try:
                yield self
            finally:
                self.set_tuning(**old)
        return cm()

    def __del__(self):
        try:
            if getattr(self, "h", None):
                _lib.load().bclx_context_destroy(self.h)
        except Exception:
            pass


_contexts = {}


def context(device: Optional[int] = None) -> Context:
    d = torch.cuda.current_device() if device is None else int(device)
    if d not in _contexts:
        _contexts[d] = Context(d)
    return _contexts[d]


# ---- blocking ------------------------------------------------------------------


@dataclasses.dataclass
class BlockCustom:
    """Tile-grid policy (bcl/containers/detail/Blocking.hpp:215-245): a tile
    shape and a processor grid.  On one GPU the processor grid is {1, 1}, so
    every tile is owned by rank 0.  A tile dimension of 0 (``Tile::div``)
    divides that dimension evenly over the processor grid."""

    tile_shape: Tuple[int, int]
    grid_shape: Tuple[int, int] = (1, 1)

    def seed(self, m: int, n: int) -> Tuple[int, int]:
        tm, tn = self.tile_shape
        if tm == 0:
            tm = _ceil_div(m, self.grid_shape[0])
        if tn == 0:
            tn = _ceil_div(n, self.grid_shape[1])
        if tm <= 0 or tn <= 0:
            raise ValueError("tile shape must be positive")
        return int(tm), int(tn)


# ---- host-side tiling ------------------------------------------------------------


def split_tiles(a: CSR, tm: int, tn: int):
    """Cut a host CSR into a tm x tn tile grid, packed (the result of
    SPMatrix::init_ / get_slice_impl_, SPMatrix.hpp:211-271, CSRMatrix.hpp:238-276):
    returns (tile_row_ptr [ntiles, tm+1] int32 local offsets, tile_offset
    [ntiles+1] int64, col_ind int32 tile-local, vals)."""
    gm, gn = _ceil_div(a.m, tm), _ceil_div(a.n, tn)
    ntiles = gm * gn
    rp = a.row_ptr.astype(np.int64)
    rows = np.repeat(np.arange(a.m, dtype=np.int64), np.diff(rp))
    cols = a.col_ind.astype(np.int64)
    ti, tj = rows // tm, cols // tn
    t = ti * gn + tj
    order = np.argsort(t, kind="stable")  # keeps (row, col) order inside every tile
    t_sorted = t[order]
    lrow = rows[order] - ti[order] * tm
    counts = np.bincount(t, minlength=ntiles)
    tile_offset = np.zeros(ntiles + 1, dtype=np.int64)
    np.cumsum(counts, out=tile_offset[1:])
    per_row = np.bincount(t_sorted * tm + lrow, minlength=ntiles * tm).reshape(ntiles, tm)
    tile_rp = np.zeros((ntiles, tm + 1), dtype=np.int64)
    np.cumsum(per_row, axis=1, out=tile_rp[:, 1:])
    if counts.size and counts.max(initial=0) >= 2**31:
        raise OverflowError("a tile has more than 2**31-1 nonzeros")
    col_local = (cols[order] - tj[order] * tn).astype(np.int32)
    return tile_rp.astype(np.int32), tile_offset, col_local, a.vals[order]


_BINARY_OPS = {"plus": 0, "minus": 1, "multiplies": 2, "divides": 3, "min": 4, "max": 5, "second": 6}


def _binary_op_code(fn) -> int:
    import operator
    if isinstance(fn, str):
        if fn not in _BINARY_OPS:
            raise ValueError(f"unknown binary op {fn!r}")
        return _BINARY_OPS[fn]
    table = {operator.add: 0, operator.sub: 1, operator.mul: 2, operator.truediv: 3, operator.floordiv: 3,
             min: 4, max: 5}
    if fn in table:
        return table[fn]
    raise ValueError("binary_op_inplace runs on the device: pass one of " + ", ".join(_BINARY_OPS))


def _nonempty(t: torch.Tensor) -> torch.Tensor:
    return t if t.numel() > 0 else torch.zeros(1, dtype=t.dtype, device=t.device)


# ---- SPMatrix ----------------------------------------------------------------------


class _Future:
    """A deferred value with BCL::future's get() (core/future.hpp:13-72)."""

    def __init__(self, fn):
        self._fn, self._done, self._value = fn, False, None

    def get(self):
        if not self._done:
            self._value, self._done, self._fn = self._fn(), True, None
        return self._value

    def wait(self) -> None:
        self.get()


class SPMatrix:
    """Distributed sparse matrix with every tile on this GPU
    (BCL::SPMatrix<T, int>, bcl/containers/SPMatrix.hpp:69-659)."""

    def __init__(self, m: int, n: int, tile_m: int, tile_n: int, dtype, device: int,
                 tile_row_ptr: torch.Tensor, tile_offset: torch.Tensor, col_ind: torch.Tensor,
                 vals: torch.Tensor):
        self.m, self.n = int(m), int(n)
        self.tm, self.tn = int(tile_m), int(tile_n)
        self.gm, self.gn = _ceil_div(self.m, self.tm), _ceil_div(self.n, self.tn)
        self.dtype = np.dtype(dtype)
        self.device = device
        self.tile_row_ptr = tile_row_ptr
        self.tile_offset = tile_offset
        self.col_ind = _nonempty(col_ind)
        self.vals = _nonempty(vals)
        self._offsets_host = None
        self._build_desc()

    # -- construction
    @classmethod
    def from_csr(cls, a: CSR, blocking: BlockCustom, device: Optional[int] = None) -> "SPMatrix":
        """Upload a host matrix and tile it on the device (the SPMatrix(fname,
        blocking) constructor's slicing, SPMatrix.hpp:211-271, from an
        in-memory CSR whose columns are ascending within each row)."""
        dev = torch.cuda.current_device() if device is None else device
        tm, tn = blocking.seed(a.m, a.n)
        td = torch.device("cuda", dev)
        rp = torch.from_numpy(a.row_ptr.astype(np.int32)).to(td)
        ci = torch.from_numpy(a.col_ind.astype(np.int32)).to(td)
        v = torch.from_numpy(np.ascontiguousarray(a.vals)).to(td)
        return cls.from_device_csr(a.m, a.n, rp, ci, v, (tm, tn), device=dev)

    @classmethod
    def from_device_csr(cls, m: int, n: int, row_ptr: torch.Tensor, col_ind: torch.Tensor, vals: torch.Tensor,
                        tile_shape: Tuple[int, int], device: Optional[int] = None) -> "SPMatrix":
        """Tile a CSR matrix already in device memory (int32 row_ptr [m+1] and
        col_ind, FP32 or int32 vals; columns ascending within each row)
        into a tile_m x tile_n grid, on the device (bclx_csr_to_tiles)."""
        dev = torch.cuda.current_device() if device is None else device
        tm, tn = int(tile_shape[0]), int(tile_shape[1])
        gm, gn = _ceil_div(m, tm), _ceil_div(n, tn)
        td = torch.device("cuda", dev)
        nnz = int(col_ind.numel())
        np_dtype = np.dtype(np.float32) if vals.dtype == torch.float32 else np.dtype(np.int32)
        dt = _NP_TO_DT[np_dtype]
        trp = torch.empty((gm * gn, tm + 1), dtype=torch.int32, device=td)
        toff = torch.zeros(gm * gn + 1, dtype=torch.int64, device=td)
        oci = torch.empty(max(nnz, 1), dtype=torch.int32, device=td)
        ov = torch.empty(max(nnz, 1), dtype=vals.dtype, device=td)
        desc = CSRDesc(m, n, nnz, row_ptr.data_ptr(), col_ind.data_ptr() if nnz else 0,
                       vals.data_ptr() if nnz else 0, dt, 0)
        out = SpGridOut(m, n, tm, tn, gm, gn, trp.data_ptr(), toff.data_ptr(), oci.data_ptr(), ov.data_ptr(), dt, 0)
        call("bclx_csr_to_tiles", context(dev).use_current_stream(), ctypes.byref(desc), ctypes.byref(out))
        return cls(m, n, tm, tn, np_dtype, dev, trp, toff, oci[:nnz], ov[:nnz])

    @classmethod
    def from_file(cls, path: str, blocking: BlockCustom, value_dtype=np.float32,
                  device: Optional[int] = None) -> "SPMatrix":
        """SPMatrix(fname, blocking) (SPMatrix.hpp:108-113, 194-271): a
        MatrixMarket (.mtx) or binary (.binary) file, tiled on the device."""
        from . import gen
        return cls.from_csr(gen.read_matrix(path, value_dtype), blocking, device)

    @classmethod
    def zeros(cls, shape: Tuple[int, int], blocking: BlockCustom, dtype=np.float32,
              device: Optional[int] = None) -> "SPMatrix":
        """An all-zero matrix (SPMatrix(dim, blocking), init_with_zero)."""
        dev = torch.cuda.current_device() if device is None else device
        m, n = shape
        tm, tn = blocking.seed(m, n)
        ntiles = _ceil_div(m, tm) * _ceil_div(n, tn)
        td = torch.device("cuda", dev)
        return cls(m, n, tm, tn, dtype, dev, torch.zeros((ntiles, tm + 1), dtype=torch.int32, device=td),
                   torch.zeros(ntiles + 1, dtype=torch.int64, device=td),
                   torch.zeros(0, dtype=torch.int32, device=td),
                   torch.zeros(0, dtype=_TORCH_OF[_NP_TO_DT[np.dtype(dtype)]], device=td))

    def _build_desc(self):
        """Device array of bclx_csr_t, one per tile, computed on the device."""
        ntiles = self.gm * self.gn
        td = self.tile_row_ptr.device
        ti = torch.arange(self.gm, device=td).repeat_interleave(self.gn)
        tj = torch.arange(self.gn, device=td).repeat(self.gm)
        d = torch.empty((ntiles, 6), dtype=torch.int64, device=td)
        d[:, 0] = torch.clamp(self.m - ti * self.tm, max=self.tm)
        d[:, 1] = torch.clamp(self.n - tj * self.tn, max=self.tn)
        d[:, 2] = self.tile_offset[1:] - self.tile_offset[:-1]
        d[:, 3] = self.tile_row_ptr.data_ptr() + torch.arange(ntiles, device=td) * (self.tm + 1) * 4
        d[:, 4] = self.col_ind.data_ptr() + self.tile_offset[:-1] * 4
        d[:, 5] = self.vals.data_ptr() + self.tile_offset[:-1] * self.vals.element_size()
        self.desc = torch.empty((ntiles, 7), dtype=torch.int64, device=td)
        self.desc[:, :6] = d
        self.desc[:, 6] = _NP_TO_DT[self.dtype]  # dtype (low 32 bits) and pad
        self.desc = self.desc.contiguous()
        self._offsets_host = None

    # -- the reference's accessors
    def shape(self):
        return (self.m, self.n)

    def grid_shape(self):
        return (self.gm, self.gn)

    def tile_shape(self, index=None):
        if index is None:
            return (self.tm, self.tn)
        i, j = index
        return (min(self.tm, self.m - i * self.tm), min(self.tn, self.n - j * self.tn))

    def tile_rank(self, index) -> int:
        return 0

    def _offsets(self) -> np.ndarray:
        if self._offsets_host is None:
            self._offsets_host = self.tile_offset.cpu().numpy()
        return self._offsets_host

    def tile_nnz(self, index) -> int:
        t = index[0] * self.gn + index[1]
        o = self._offsets()
        return int(o[t + 1] - o[t])

    def nnz(self) -> int:
        return int(self._offsets()[-1])

    def spgrid(self) -> SpGrid:
        key = self.desc.data_ptr()
        g = getattr(self, "_spgrid", None)
        if g is None or g[0] != key:  # built once per descriptor array
            g = (key, SpGrid(self.m, self.n, self.tm, self.tn, self.gm, self.gn, key, _NP_TO_DT[self.dtype], 0))
            self._spgrid = g
        return g[1]

    def tile_desc_ptr(self, index) -> int:
        """Device address of one tile's bclx_csr_t (a 1x1 grid view of it)."""
        return self.desc.data_ptr() + (index[0] * self.gn + index[1]) * 56

    def get_tile(self, index) -> CSR:
        """Copy one tile to the host (SPMatrix::get_tile, SPMatrix.hpp:476-494)."""
        t = index[0] * self.gn + index[1]
        o = self._offsets()
        m, n = self.tile_shape(index)
        rp = self.tile_row_ptr[t, : m + 1].cpu().numpy()
        ci = self.col_ind[o[t]:o[t + 1]].cpu().numpy() if o[t + 1] > o[t] else np.zeros(0, np.int32)
        v = self.vals[o[t]:o[t + 1]].cpu().numpy() if o[t + 1] > o[t] else np.zeros(0, self.dtype)
        return CSR(m, n, rp, ci, v)

    def arget_tile(self, index) -> "_Future":
        """SPMatrix::arget_tile (SPMatrix.hpp:496-514): the tile copy as a
        future; its get() makes the copy (once)."""
        return _Future(lambda: self.get_tile(index))

    def get(self) -> CSR:
        """Gather the whole matrix in global coordinates on the device
        (bclx_tiles_to_csr) and return it on the host (SPMatrix::get,
        SPMatrix.hpp:516-546)."""
        rp, ci, v = self.get_device()
        return CSR(self.m, self.n, rp.cpu().numpy(), ci.cpu().numpy(), v.cpu().numpy())

    def get_device(self):
        """The whole matrix as device CSR arrays (row_ptr, col_ind, vals)."""
        nnz = int(self._offsets()[-1])
        td = self.tile_row_ptr.device
        rp = torch.empty(self.m + 1, dtype=torch.int32, device=td)
        ci = torch.empty(max(nnz, 1), dtype=torch.int32, device=td)
        v = torch.empty(max(nnz, 1), dtype=self.vals.dtype, device=td)
        call("bclx_tiles_to_csr", context(self.device).use_current_stream(), ctypes.byref(self.spgrid()),
             ctypes.c_void_p(rp.data_ptr()), ctypes.c_void_p(ci.data_ptr()), ctypes.c_void_p(v.data_ptr()))
        return rp, ci[:nnz], v[:nnz]

    def get_host_gather(self) -> CSR:
        """The same gather done with numpy on the host (kept for checks)."""
        o = self._offsets()
        nnz = int(o[-1])
        trp = self.tile_row_ptr.cpu().numpy().astype(np.int64)
        ci = self.col_ind.cpu().numpy()[:nnz].astype(np.int64)
        v = self.vals.cpu().numpy()[:nnz]
        t_of = np.repeat(np.arange(self.gm * self.gn), np.diff(o))
        ti, tj = t_of // self.gn, t_of % self.gn
        # local row of each entry
        lrow = np.empty(nnz, dtype=np.int64)
        for t in range(self.gm * self.gn):
            if o[t + 1] > o[t]:
                cnt = np.diff(trp[t])
                lrow[o[t]:o[t + 1]] = np.repeat(np.arange(self.tm), cnt)
        grow = ti * self.tm + lrow
        gcol = tj * self.tn + ci
        key = grow * self.n + gcol
        order = np.argsort(key, kind="stable")
        counts = np.bincount(grow, minlength=self.m)
        rp = np.zeros(self.m + 1, dtype=np.int64)
        np.cumsum(counts, out=rp[1:])
        vals = v[order]
        if vals.dtype == np.float32:  # as SPMatrix::get adds each value to 0: -0.0 -> +0.0
            vals = np.float32(0) + vals
        return CSR(self.m, self.n, rp.astype(np.int32), gcol[order].astype(np.int32), vals)

    def binary_op_inplace(self, other: "DMatrix", fn) -> "SPMatrix":
        """Every stored entry a(i, j) becomes fn(a(i, j), other(i, j))
        (SPMatrix::binary_op_inplace, SPMatrix.hpp:571-616), on the device.
        fn: one of "plus", "minus", "multiplies", "divides", "min", "max",
        "second", or operator.add / sub / mul / truediv / floordiv, or the
        builtins min / max."""
        code = _binary_op_code(fn)
        if other.m != self.m or other.n != self.n:
            raise RuntimeError("BCL::SPMatrix::binary_op_inplace: shape mismatch")
        call("bclx_spmatrix_binary_op", context(self.device).use_current_stream(), ctypes.byref(self.spgrid()),
             ctypes.byref(other.dgrid()), code)
        return self

    def assign_tile(self, index, tile: CSR) -> None:
        """Replace one tile (SPMatrix::assign_tile, SPMatrix.hpp:277-308)."""
        if tile.m != self.tile_shape(index)[0] or tile.n != self.tile_shape(index)[1]:
            raise RuntimeError("BCL::SpMatrix::assign_tile: tile shape mismatch")
        t = index[0] * self.gn + index[1]
        o = self._offsets()
        td = self.tile_row_ptr.device
        nnz = int(o[-1])
        old_n = int(o[t + 1] - o[t])
        new_n = tile.nnz
        ci = torch.cat([self.col_ind[: o[t]], torch.from_numpy(tile.col_ind.astype(np.int32)).to(td),
                        self.col_ind[o[t + 1]:nnz]])
        v = torch.cat([self.vals[: o[t]], torch.from_numpy(np.ascontiguousarray(tile.vals, self.dtype)).to(td),
                       self.vals[o[t + 1]:nnz]])
        rp = self.tile_row_ptr.clone()
        rp[t].zero_()
        rp[t, : tile.m + 1] = torch.from_numpy(tile.row_ptr.astype(np.int32)).to(td)
        rp[t, tile.m + 1:] = new_n
        toff = self.tile_offset.clone()
        toff[t + 1:] += new_n - old_n
        self.tile_row_ptr, self.tile_offset = rp, toff
        self.col_ind, self.vals = _nonempty(ci), _nonempty(v)
        self._build_desc()

    def dot(self, other):
        """C = self * other (SPMatrix::dot -> gemm)."""
        if isinstance(other, SPMatrix):
            return spgemm(self, other)
        if isinstance(other, DMatrix):
            c = DMatrix.zeros((self.m, other.n), BlockCustom((self.tm, other.tn)), dtype=other.torch_dtype,
                              device=self.device)
            gemm(self, other, c)
            return c
        raise TypeError("dot: unsupported operand")


# ---- DMatrix -------------------------------------------------------------------------


class DMatrix:
    """Distributed dense matrix with every tile on this GPU (BCL::DMatrix<T>,
    bcl/containers/DMatrix.hpp:27-587): grid_m*grid_n tiles of tile_m x tile_n,
    row-major, padded to full size at the edges.  FP32, or bfloat16 storage."""

    def __init__(self, m: int, n: int, tile_m: int, tile_n: int, tiles: torch.Tensor):
        self.m, self.n, self.tm, self.tn = int(m), int(n), int(tile_m), int(tile_n)
        self.gm, self.gn = _ceil_div(self.m, self.tm), _ceil_div(self.n, self.tn)
        assert tiles.shape == (self.gm * self.gn, self.tm, self.tn) and tiles.is_contiguous()
        self.tiles = tiles
        self.torch_dtype = tiles.dtype
        self.device = tiles.device.index
        nt = self.gm * self.gn
        self.ptrs = (tiles.data_ptr() + torch.arange(nt, dtype=torch.int64, device=tiles.device)
                     * (self.tm * self.tn * tiles.element_size())).contiguous()

    @classmethod
    def zeros(cls, shape, blocking: BlockCustom, dtype=torch.float32, device=None) -> "DMatrix":
        dev = torch.cuda.current_device() if device is None else device
        m, n = shape
        tm, tn = blocking.seed(m, n)
        nt = _ceil_div(m, tm) * _ceil_div(n, tn)
        return cls(m, n, tm, tn, torch.zeros((nt, tm, tn), dtype=dtype, device=torch.device("cuda", dev)))

    @classmethod
    def from_array(cls, arr, blocking: BlockCustom, dtype=torch.float32, device=None) -> "DMatrix":
        """Tile a full row-major array (host numpy or torch)."""
        dev = torch.cuda.current_device() if device is None else device
        full = torch.as_tensor(arr)
        m, n = full.shape
        d = cls.zeros((m, n), blocking, dtype=dtype, device=dev)
        d.set_matrix(full)
        return d

    def set_matrix(self, full: torch.Tensor) -> None:
        src = full.to(device=self.tiles.device, dtype=self.torch_dtype)
        mp, np_ = self.gm * self.tm, self.gn * self.tn
        pad = torch.zeros((mp, np_), dtype=self.torch_dtype, device=self.tiles.device)
        pad[: self.m, : self.n] = src
        self.tiles.copy_(pad.view(self.gm, self.tm, self.gn, self.tn).permute(0, 2, 1, 3)
                         .reshape(self.gm * self.gn, self.tm, self.tn))

    def get_matrix(self) -> torch.Tensor:
        """The whole matrix as one row-major tensor (DMatrix::get_matrix)."""
        full = (self.tiles.view(self.gm, self.gn, self.tm, self.tn).permute(0, 2, 1, 3)
                .reshape(self.gm * self.tm, self.gn * self.tn))
        return full[: self.m, : self.n]

    def fill_(self, value) -> "DMatrix":
        """DMatrix::operator=(value) (DMatrix.hpp:226-242)."""
        self.tiles.fill_(value)
        return self

    def shape(self):
        return (self.m, self.n)

    def grid_shape(self):
        return (self.gm, self.gn)

    def tile_shape(self, index=None):
        if index is None:
            return (self.tm, self.tn)
        i, j = index
        return (min(self.tm, self.m - i * self.tm), min(self.tn, self.n - j * self.tn))

    def tile_rank(self, index) -> int:
        return 0

    def tile_size(self) -> int:
        """Elements of one (padded) tile storage (DMatrix::tile_size)."""
        return self.tm * self.tn

    def tile_ptr(self, index) -> int:
        return int(self.tiles[index[0] * self.gn + index[1]].data_ptr())

    def get_tile(self, index) -> torch.Tensor:
        """The padded tile, row-major, copied to the host (DMatrix::get_tile,
        DMatrix.hpp:169-173)."""
        return self.tiles[index[0] * self.gn + index[1]].reshape(-1).cpu()

    @property
    def bclx_dtype(self) -> int:
        if self.torch_dtype == torch.float32:
            return _lib.F32
        if self.torch_dtype == torch.bfloat16:
            return _lib.BF16
        if self.torch_dtype == torch.int32:
            return _lib.I32
        raise TypeError("DMatrix tiles must be float32, bfloat16 or int32")

    def sum(self):
        """Sum of every element (DMatrix::sum, DMatrix.hpp:537-554), on the
        device: int32 exact (modulo 2^32); FP32/BF16 accumulated in FP64 and
        rounded once to FP32 (the reference's sequential FP32 sum agrees
        within its own rounding error)."""
        out = (ctypes.c_int32 if self.torch_dtype == torch.int32 else ctypes.c_float)()
        call("bclx_dmatrix_sum", context(self.device).use_current_stream(), ctypes.byref(self.dgrid()),
             ctypes.byref(out))
        return out.value

    def dgrid(self) -> DGrid:
        key = self.ptrs.data_ptr()
        g = getattr(self, "_dgrid", None)
        if g is None or g[0] != key:  # built once per tile-pointer array
            g = (key, DGrid(self.m, self.n, self.tm, self.tn, self.gm, self.gn, key, self.bclx_dtype, 0))
            self._dgrid = g
        return g[1]


# ---- products -----------------------------------------------------------------------


def _out_grid(a: SPMatrix, b: SPMatrix):
    td = a.tile_row_ptr.device
    gm, gn = a.gm, b.gn
    trp = torch.empty((gm * gn, a.tm + 1), dtype=torch.int32, device=td)
    toff = torch.empty(gm * gn + 1, dtype=torch.int64, device=td)
    out = SpGridOut(a.m, b.n, a.tm, b.tn, gm, gn, trp.data_ptr(), toff.data_ptr(), None, None,
                    _NP_TO_DT[a.dtype], 0)
    return out, trp, toff


class SpgemmPlan:
    """Holds a symbolic-phase plan (work decomposition and row offsets)."""

    def __init__(self, handle):
        self.h = handle

    def stats(self) -> dict:
        arr = (ctypes.c_int64 * 6)()
        call("bclx_spgemm_plan_stats", self.h, arr)
        keys = ["products", "light_rows", "heavy_rows", "heavy_items", "stages", "nnz"]
        return dict(zip(keys, [int(x) for x in arr]))

    def tune(self, grab: int, blocks_per_sm: int, long_seg: int) -> None:
        """Numeric-pass parameters (see bclx_spgemm_plan_tune)."""
        call("bclx_spgemm_plan_tune", self.h, int(grab), int(blocks_per_sm), int(long_seg))

    def close(self):
        if getattr(self, "h", None):
            lib = _lib._lib
            if lib is not None:  # (at interpreter exit the library may be gone already)
                lib.bclx_spgemm_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def _check_grids(a: SPMatrix, b: SPMatrix):
    if a.n != b.m:
        raise RuntimeError("BCL::gemm: inner dimensions differ")
    if a.tn != b.tm:
        raise RuntimeError("BCL::gemm: A's tile width must equal B's tile height")
    if a.dtype != b.dtype:
        raise TypeError("BCL::gemm: A and B value types differ")


def spgemm_symbolic(a: SPMatrix, b: SPMatrix):
    """Symbolic phase: returns (plan, out descriptor, tile_row_ptr, tile_offset, nnz)."""
    _check_grids(a, b)
    ctx = context(a.device)
    h = ctx.use_current_stream()
    out, trp, toff = _out_grid(a, b)
    plan = ctypes.c_void_p()
    nnz = ctypes.c_int64()
    ag, bg = a.spgrid(), b.spgrid()
    call("bclx_spgemm_symbolic", h, ctypes.byref(ag), ctypes.byref(bg), ctypes.byref(out), ctypes.byref(plan),
         ctypes.byref(nnz))
    return SpgemmPlan(plan), out, trp, toff, int(nnz.value)


def spgemm(a: SPMatrix, b: SPMatrix, stages: str = "fused", keep_plan: bool = False, tuning=None):
    """C = A * B over the tile grids (BCL::gemm(SPMatrix, SPMatrix, SPMatrix&),
    spgemm.hpp:182-242).  ``stages="fused"`` runs every SUMMA stage in one
    numeric launch; ``"per_stage"`` / ``"batched"`` run one launch per stage
    (all G*G tile products of that stage), adding into C between them;
    ``"batched_graph"`` does the same through a CUDA graph kept by the plan.
    All forms are bit-identical.  ``tuning`` = (grab, blocks_per_sm,
    long_seg), a dict of those and "light_ub", or "auto" for the autotuner's
    cached choice."""
    params = None
    if tuning == "auto":
        from . import autotune
        params = autotune.lookup(a, b)
    elif isinstance(tuning, dict):
        params = tuning
    elif tuning:
        params = dict(zip(("grab", "blocks_per_sm", "long_seg"), tuning))
    sym_knobs = {k: params[k] for k in ("light_ub", "item_outputs", "wide_light") if params and k in params}
    if sym_knobs:
        with context(a.device).tuned(**sym_knobs):
            plan, out, trp, toff, nnz = spgemm_symbolic(a, b)
    else:
        plan, out, trp, toff, nnz = spgemm_symbolic(a, b)
    if params:
        plan.tune(params.get("grab", 1), params.get("blocks_per_sm", 4), params.get("long_seg", 32))
    td = a.tile_row_ptr.device
    ci = torch.empty(max(nnz, 1), dtype=torch.int32, device=td)
    v = torch.empty(max(nnz, 1), dtype=_TORCH_OF[_NP_TO_DT[a.dtype]], device=td)
    out.col_ind, out.vals = ci.data_ptr(), v.data_ptr()
    spgemm_numeric(plan, a, b, out, stages)
    c = SPMatrix(a.m, b.n, a.tm, b.tn, a.dtype, a.device, trp, toff, ci, v)
    if keep_plan:
        return c, plan
    plan.close()
    return c


# ---- distributed products (one process per GPU) ------------------------------------


def process_grid(world: int) -> Tuple[int, int]:
    """pm x pn process grid for `world` processes, as square as possible
    (pm <= pn), the shape of the reference's default BlockSquare layout."""
    pm = int(world ** 0.5)
    while world % pm:
        pm -= 1
    return pm, world // pm


def owned_tiles(gm: int, gn: int, rank: int, pm: int, pn: int):
    """Tile rows and columns whose C tiles process `rank` owns in the
    reference's block-cyclic layout: tile (i, j) belongs to process
    (j % pn) + (i % pm) * pn (SPMatrix.hpp:230-237).  The owned tiles are the
    Cartesian product of the two lists."""
    r, c = divmod(rank, pn)
    return [i for i in range(gm) if i % pm == r], [j for j in range(gn) if j % pn == c]


def _sub_spgrid(x: SPMatrix, rows, cols):
    """Tile rows `rows` x tile columns `cols` of x as a grid view: a gathered
    descriptor array (the tiles themselves are not copied)."""
    td = x.desc.device
    r = torch.as_tensor(list(rows), dtype=torch.int64, device=td)
    c = torch.as_tensor(list(cols), dtype=torch.int64, device=td)
    desc = x.desc[(r[:, None] * x.gn + c[None, :]).reshape(-1)].contiguous()
    m = sum(min(x.tm, x.m - i * x.tm) for i in rows)
    n = sum(min(x.tn, x.n - j * x.tn) for j in cols)
    return SpGrid(m, n, x.tm, x.tn, len(rows), len(cols), desc.data_ptr(), _NP_TO_DT[x.dtype], 0), desc


def spgemm_sub(a: SPMatrix, b: SPMatrix, tile_rows, tile_cols, form: str = "fused", predictor="default",
               keep_plan: bool = False):
    """The C tiles (i, j), i in tile_rows, j in tile_cols (increasing global
    tile indices), of C = A * B, bit-identical to those tiles of the whole
    product (each keeps its stage order k = (k_ + i + j) mod G): what one
    process of the reference's stationary-C loop computes
    (spgemm.hpp:194-224), or one block of a product computed block by block.
    The result is an SPMatrix of those tiles in sub-grid order
    (bclx_spgemm_symbolic_sub, or bclx_spgemm_learned_run_sub with
    form="learned")."""
    _check_grids(a, b)
    if form == "learned":
        return _spgemm_learned_sub(a, b, tile_rows, tile_cols, predictor, keep_plan)
    tile_rows, tile_cols = list(tile_rows), list(tile_cols)
    if any(q <= p for p, q in zip(tile_rows, tile_rows[1:])) or any(q <= p for p, q in zip(tile_cols, tile_cols[1:])):
        raise ValueError("tile rows and columns must be increasing")
    ag, adesc = _sub_spgrid(a, tile_rows, range(a.gn))
    bg, bdesc = _sub_spgrid(b, range(b.gm), tile_cols)
    c = _sub_product(a, b, ag, bg, tile_rows, tile_cols)
    del adesc, bdesc  # (the numeric pass is ordered on the stream before any reuse)
    return c


def spgemm_compact(a: SPMatrix, b: SPMatrix, tile_rows, tile_cols):
    """The C tiles (tile_rows[x], tile_cols[y]) of a product whose operands
    are held as compact grids: `a` holds exactly A's tile rows `tile_rows`
    (its tile (x, k) is global tile (tile_rows[x], k)) and `b` exactly B's
    tile columns `tile_cols` (as a process of a distributed product holds
    them after fetching them from their owners, bcl_b200.distributed).  Every
    tile is bit-identical to that tile of the whole product."""
    _check_grids(a, b)
    tile_rows, tile_cols = list(tile_rows), list(tile_cols)
    if a.gm != len(tile_rows) or b.gn != len(tile_cols):
        raise RuntimeError("BCL::gemm: compact operand grids do not match the tile lists")
    if any(q <= p for p, q in zip(tile_rows, tile_rows[1:])) or any(q <= p for p, q in zip(tile_cols, tile_cols[1:])):
        raise ValueError("tile rows and columns must be increasing")
    return _sub_product(a, b, a.spgrid(), b.spgrid(), tile_rows, tile_cols)


def _sub_product(a: SPMatrix, b: SPMatrix, ag, bg, tile_rows, tile_cols):
    """bclx_spgemm_symbolic_sub + numeric on the grid views ag (A's rows
    tile_rows) and bg (B's columns tile_cols)."""
    h = context(a.device).use_current_stream()
    td = a.tile_row_ptr.device
    gm, gn = len(tile_rows), len(tile_cols)
    trp = torch.empty((gm * gn, a.tm + 1), dtype=torch.int32, device=td)
    toff = torch.empty(gm * gn + 1, dtype=torch.int64, device=td)
    out = SpGridOut(ag.m, bg.n, a.tm, b.tn, gm, gn, trp.data_ptr(), toff.data_ptr(), None, None,
                    _NP_TO_DT[a.dtype], 0)
    rows_arr = (ctypes.c_int64 * max(gm, 1))(*tile_rows)
    cols_arr = (ctypes.c_int64 * max(gn, 1))(*tile_cols)
    plan = ctypes.c_void_p()
    nnz = ctypes.c_int64()
    call("bclx_spgemm_symbolic_sub", h, ctypes.byref(ag), ctypes.byref(bg), ctypes.byref(out), rows_arr, cols_arr,
         ctypes.byref(plan), ctypes.byref(nnz))
    pl = SpgemmPlan(plan)
    ci = torch.empty(max(nnz.value, 1), dtype=torch.int32, device=td)
    v = torch.empty(max(nnz.value, 1), dtype=_TORCH_OF[_NP_TO_DT[a.dtype]], device=td)
    out.col_ind, out.vals = ci.data_ptr(), v.data_ptr()
    call("bclx_spgemm_numeric", h, pl.h, ctypes.byref(ag), ctypes.byref(bg), ctypes.byref(out), 0, 0)
    pl.close()
    return SPMatrix(ag.m, bg.n, a.tm, b.tn, a.dtype, a.device, trp, toff, ci, v)


def _spgemm_learned_sub(a, b, tile_rows, tile_cols, predictor, keep_plan):
    if predictor == "default":
        from . import learned
        predictor = learned.get_default()
    tile_rows, tile_cols = list(tile_rows), list(tile_cols)
    h = context(a.device).use_current_stream()
    ag, adesc = _sub_spgrid(a, tile_rows, range(a.gn))
    bg, bdesc = _sub_spgrid(b, range(b.gm), tile_cols)
    td = a.tile_row_ptr.device
    gm, gn = len(tile_rows), len(tile_cols)
    trp = torch.empty((gm * gn, a.tm + 1), dtype=torch.int32, device=td)
    toff = torch.empty(gm * gn + 1, dtype=torch.int64, device=td)
    out = SpGridOut(ag.m, bg.n, a.tm, b.tn, gm, gn, trp.data_ptr(), toff.data_ptr(), None, None,
                    _NP_TO_DT[a.dtype], 0)
    rows_arr = (ctypes.c_int64 * max(gm, 1))(*tile_rows)
    cols_arr = (ctypes.c_int64 * max(gn, 1))(*tile_cols)
    prm = ctypes.c_void_p(predictor.params.data_ptr()) if predictor is not None else None
    plan = ctypes.c_void_p()
    nnz = ctypes.c_int64()
    call("bclx_spgemm_learned_run_sub", h, ctypes.byref(ag), ctypes.byref(bg), ctypes.byref(out), rows_arr,
         cols_arr, prm, ctypes.byref(plan), ctypes.byref(nnz))
    pl = SpgemmPlan(plan)
    k = int(nnz.value)
    ci = torch.empty(max(k, 1), dtype=torch.int32, device=td)
    v = torch.empty(max(k, 1), dtype=_TORCH_OF[_NP_TO_DT[a.dtype]], device=td)
    out.col_ind, out.vals = ci.data_ptr(), v.data_ptr()
    call("bclx_spgemm_learned_finish", h, pl.h, ctypes.byref(out))
    del adesc, bdesc
    c = SPMatrix(ag.m, bg.n, a.tm, b.tn, a.dtype, a.device, trp, toff, ci, v)
    if keep_plan:
        return c, pl
    pl.close()
    return c


def spgemm_blocks(a: SPMatrix, b: SPMatrix, block_rows: int, form: str = "fused", predictor="default"):
    """C = A * B computed one block of `block_rows` C tile rows at a time
    (for products whose working space does not fit beside the whole C):
    yields (tile rows, SPMatrix of that block's tiles).  The blocks together
    are the whole product, bit for bit."""
    for i0 in range(0, a.gm, block_rows):
        rows = list(range(i0, min(i0 + block_rows, a.gm)))
        yield rows, spgemm_sub(a, b, rows, range(b.gn), form=form, predictor=predictor)


def spgemm_to_host(a: SPMatrix, b: SPMatrix, block_rows: int = 1, host: Optional[dict] = None):
    """C = A * B delivered to pinned host memory with the device-to-host copy
    overlapped with the product: C is computed one block of `block_rows`
    tile rows at a time (spgemm_sub) and each finished block's arrays are
    copied back on a second stream while the next block is computed.
    `host`: a dict of pinned buffers reused across calls (grown as needed).
    Returns (host dict, [(tile rows, nnz, tile_row_ptr, tile_offset,
    col_ind, vals) host views per block]), valid once the call returns (it
    waits for the copies)."""
    host = {} if host is None else host
    copy_stream = host.get("_stream")
    if copy_stream is None:
        copy_stream = host["_stream"] = torch.cuda.Stream(device=a.tile_row_ptr.device)
    compute = torch.cuda.current_stream()
    blocks, keep = [], []
    for q, i0 in enumerate(range(0, a.gm, block_rows)):
        rows = list(range(i0, min(i0 + block_rows, a.gm)))
        C = spgemm_sub(a, b, rows, range(b.gn))
        nnz = C.nnz()
        ev = torch.cuda.Event()
        ev.record(compute)
        views = []
        with torch.cuda.stream(copy_stream):
            copy_stream.wait_event(ev)
            for name, t in (("tile_row_ptr", C.tile_row_ptr.reshape(-1)), ("tile_offset", C.tile_offset),
                            ("col_ind", C.col_ind[:nnz]), ("vals", C.vals[:nnz])):
                buf = host.get((q, name))
                if buf is None or buf.numel() < t.numel() or buf.dtype != t.dtype:
                    buf = host[(q, name)] = torch.empty(max(t.numel(), 1), dtype=t.dtype).pin_memory()
                dst = buf[:t.numel()]
                dst.copy_(t, non_blocking=True)
                views.append(dst)
        keep.append(C)  # the device arrays stay alive until their copies finish
        blocks.append((rows, nnz, *views))
    copy_stream.synchronize()
    del keep
    return host, blocks


def spgemm_distributed(a: SPMatrix, b: SPMatrix, rank: int, world: int, pgrid=None):
    """This process's C tiles of C = A * B under the reference's block-cyclic
    ownership, A's tile rows and B's tile columns being available here (A
    and B replicated, as for A * A with A loaded on every process): no data
    exchange is needed.  Returns (C sub-grid, tile rows, tile columns)."""
    pm, pn = pgrid or process_grid(world)
    rows, cols = owned_tiles(a.gm, b.gn, rank, pm, pn)
    if not rows or not cols:
        return None, rows, cols
    return spgemm_sub(a, b, rows, cols), rows, cols


def assemble_tiles(m: int, n: int, tm: int, tn: int, parts) -> CSR:
    """The whole matrix on the host from sub-grid results: parts is a list of
    (tile_rows, tile_cols, tile_row_ptr, tile_offset, col_ind, vals) host
    arrays, one per process (SPMatrix::get of a distributed matrix)."""
    gm, gn = _ceil_div(m, tm), _ceil_div(n, tn)
    tiles = {}
    if sum(len(p[0]) * len(p[1]) for p in parts) != gm * gn:
        raise RuntimeError("the parts do not cover every tile exactly once")
    for rows, cols, trp, toff, ci, v in parts:
        trp = np.asarray(trp).reshape(len(rows) * len(cols), tm + 1)
        for a_, i in enumerate(rows):
            for b_, j in enumerate(cols):
                t = a_ * len(cols) + b_
                tiles[(i, j)] = (trp[t], ci[toff[t]:toff[t + 1]], v[toff[t]:toff[t + 1]])
    if len(tiles) != gm * gn:
        raise RuntimeError("the parts do not cover every tile exactly once")
    rp = [0]
    cis, vs = [], []
    for i in range(gm):
        for r in range(min(tm, m - i * tm)):
            for j in range(gn):
                trow, ci, v = tiles[(i, j)]
                s, e = int(trow[r]), int(trow[r + 1])
                cis.append(np.asarray(ci[s:e], np.int64) + j * tn)
                vs.append(np.asarray(v[s:e]))
            rp.append(rp[-1] + sum(len(x) for x in cis[len(cis) - gn:]))
    ci = np.concatenate(cis).astype(np.int32) if cis else np.zeros(0, np.int32)
    val = np.concatenate(vs) if vs else np.zeros(0, np.float32)
    return CSR(m, n, np.asarray(rp, np.int32), ci, val)


def spgemm_learned(a: SPMatrix, b: SPMatrix, predictor="default", keep_plan: bool = False):
    """C = A * B through the learned product: a row-nnz predictor sizes the
    work instead of a symbolic pass; rows it mispredicts are redone exactly,
    so the result is bit-identical to spgemm().  ``predictor``: a
    learned.RowNnzPredictor, "default" (the cached trained model), or None
    (size the work from the product counts instead of a prediction)."""
    _check_grids(a, b)
    if predictor == "default":
        from . import learned
        predictor = learned.get_default()
    h = context(a.device).use_current_stream()
    out, trp, toff = _out_grid(a, b)
    plan = ctypes.c_void_p()
    nnz = ctypes.c_int64()
    ag, bg = a.spgrid(), b.spgrid()
    prm = ctypes.c_void_p(predictor.params.data_ptr()) if predictor is not None else None
    call("bclx_spgemm_learned_run", h, ctypes.byref(ag), ctypes.byref(bg), ctypes.byref(out), prm,
         ctypes.byref(plan), ctypes.byref(nnz))
    pl = SpgemmPlan(plan)
    k = int(nnz.value)
    td = a.tile_row_ptr.device
    ci = torch.empty(max(k, 1), dtype=torch.int32, device=td)
    v = torch.empty(max(k, 1), dtype=_TORCH_OF[_NP_TO_DT[a.dtype]], device=td)
    out.col_ind, out.vals = ci.data_ptr(), v.data_ptr()
    call("bclx_spgemm_learned_finish", h, pl.h, ctypes.byref(out))
    c = SPMatrix(a.m, b.n, a.tm, b.tn, a.dtype, a.device, trp, toff, ci, v)
    if keep_plan:
        return c, pl
    pl.close()
    return c


def learned_stats(plan: "SpgemmPlan") -> dict:
    arr = (ctypes.c_int64 * 6)()
    call("bclx_spgemm_learned_stats", plan.h, arr)
    keys = ["heavy_rows", "heavy_items", "rows_redone", "temp_entries", "nnz", "redo_items"]
    return dict(zip(keys, [int(x) for x in arr]))


def spgemm_numeric(plan: SpgemmPlan, a: SPMatrix, b: SPMatrix, out: SpGridOut, stages: str = "fused"):
    h = context(a.device).use_current_stream()
    ag, bg = a.spgrid(), b.spgrid()
    if stages == "fused":
        call("bclx_spgemm_numeric", h, plan.h, ctypes.byref(ag), ctypes.byref(bg), ctypes.byref(out), 0, 0)
    elif stages == "per_stage":
        for s in range(a.gn):
            call("bclx_spgemm_numeric", h, plan.h, ctypes.byref(ag), ctypes.byref(bg), ctypes.byref(out), s, s + 1)
    elif stages in ("batched", "batched_graph"):
        call("bclx_spgemm_numeric_staged", h, plan.h, ctypes.byref(ag), ctypes.byref(bg), ctypes.byref(out),
             1 if stages == "batched_graph" else 0)
    else:
        raise ValueError(stages)


def tile_accumulate(parts: Sequence[SPMatrix]) -> SPMatrix:
    """Sum 1x1-grid partial tiles in list order (SparseHashAccumulator::
    accumulate + get_matrix, SparseHashAccumulator.hpp:86-183)."""
    p0 = parts[0]
    m, n = p0.m, p0.n
    td = p0.tile_row_ptr.device
    descs = torch.cat([p.desc[0:1] for p in parts]).contiguous()
    h = context(p0.device).use_current_stream()
    rp = torch.empty((1, m + 1), dtype=torch.int32, device=td)
    plan = ctypes.c_void_p()
    nnz = ctypes.c_int64()
    dt = _NP_TO_DT[p0.dtype]
    call("bclx_tile_accumulate_symbolic", h, ctypes.c_void_p(descs.data_ptr()), len(parts), m, n, dt,
         ctypes.c_void_p(rp.data_ptr()), ctypes.byref(plan), ctypes.byref(nnz))
    pl = SpgemmPlan(plan)
    k = int(nnz.value)
    ci = torch.empty(max(k, 1), dtype=torch.int32, device=td)
    v = torch.empty(max(k, 1), dtype=_TORCH_OF[dt], device=td)
    out = CSRDesc(m, n, k, rp.data_ptr(), ci.data_ptr(), v.data_ptr(), dt, 0)
    call("bclx_tile_accumulate_numeric", h, pl.h, ctypes.c_void_p(descs.data_ptr()), len(parts), ctypes.byref(out))
    pl.close()
    toff = torch.tensor([0, k], dtype=torch.int64, device=td)
    return SPMatrix(m, n, m, n, p0.dtype, p0.device, rp, toff, ci, v)


def _tile_view(a: SPMatrix, index) -> SPMatrix:
    """A 1x1-grid SPMatrix sharing one tile's storage (no copy)."""
    t = index[0] * a.gn + index[1]
    o = a._offsets()
    m, n = a.tile_shape(index)
    lo, hi = int(o[t]), int(o[t + 1])
    td = a.tile_row_ptr.device
    rp = a.tile_row_ptr[t:t + 1, : m + 1].contiguous() if m + 1 != a.tm + 1 else a.tile_row_ptr[t:t + 1]
    toff = torch.tensor([0, hi - lo], dtype=torch.int64, device=td)
    return SPMatrix(m, n, m, n, a.dtype, a.device, rp, toff, a.col_ind[lo:hi] if hi > lo else a.col_ind[:0],
                    a.vals[lo:hi] if hi > lo else a.vals[:0])


def spgemm_plain(a: SPMatrix, b: SPMatrix) -> SPMatrix:
    """The reference's loop structure, one call per tile product: for every C
    tile (i, j), the partials A_ik * B_kj for k = (k_ + i + j) mod G each by a
    two-phase product, then their tile accumulation (spgemm.hpp:200-235)."""
    _check_grids(a, b)
    G = a.gn
    td = a.tile_row_ptr.device
    tiles = []
    for i in range(a.gm):
        for j in range(b.gn):
            parts = []
            for k_ in range(G):
                k = (k_ + i + j) % G
                parts.append(spgemm(_tile_view(a, (i, k)), _tile_view(b, (k, j))))
            tiles.append(tile_accumulate(parts))
    # pack the per-tile results into one SPMatrix
    tm, tn = a.tm, b.tn
    counts = [t.nnz() for t in tiles]
    toff = np.zeros(len(tiles) + 1, dtype=np.int64)
    np.cumsum(counts, out=toff[1:])
    trp = torch.empty((len(tiles), tm + 1), dtype=torch.int32, device=td)
    for t, tile in enumerate(tiles):
        mt = tile.m
        trp[t, : mt + 1] = tile.tile_row_ptr[0, : mt + 1]
        trp[t, mt + 1:] = counts[t]
    ci = torch.cat([t.col_ind[: c] for t, c in zip(tiles, counts)])
    v = torch.cat([t.vals[: c] for t, c in zip(tiles, counts)])
    return SPMatrix(a.m, b.n, tm, tn, a.dtype, a.device, trp, torch.from_numpy(toff).to(td), ci, v)


def spmm(a: SPMatrix, b: DMatrix, c: DMatrix, tuning=None) -> None:
    """C += A * B over tile grids in one launch (BCL::gemm(SPMatrix, DMatrix,
    DMatrix&), spgemm.hpp:153-179).  ``tuning``: a dict of SpMM context
    knobs (spmm_rows, spmm_long_row, spmm_long_blocks, spmm_schedule) or
    "auto" for the autotuner's cached choice; results do not depend on it."""
    if a.n != b.m or a.m != c.m or b.n != c.n:
        raise RuntimeError("BCL::gemm: shape mismatch")
    if a.dtype != np.float32:
        raise TypeError("SpMM needs FP32 sparse values")
    if tuning == "auto":
        from . import autotune
        tuning = autotune.lookup(a, b, "spmm")
    ctx = context(a.device)
    h = ctx.use_current_stream()
    ag, bg, cg = a.spgrid(), b.dgrid(), c.dgrid()
    if tuning:
        with ctx.tuned(**tuning):
            call("bclx_spmm_grid", h, ctypes.byref(ag), ctypes.byref(bg), ctypes.byref(cg))
    else:
        call("bclx_spmm_grid", h, ctypes.byref(ag), ctypes.byref(bg), ctypes.byref(cg))


def _sub_dgrid(x: DMatrix, rows, cols):
    """Tile rows `rows` x tile columns `cols` of x as a grid view: a gathered
    tile-pointer array (the tiles themselves are not copied)."""
    td = x.ptrs.device
    r = torch.as_tensor(list(rows), dtype=torch.int64, device=td)
    c = torch.as_tensor(list(cols), dtype=torch.int64, device=td)
    ptrs = x.ptrs[(r[:, None] * x.gn + c[None, :]).reshape(-1)].contiguous()
    m = sum(min(x.tm, x.m - i * x.tm) for i in rows)
    n = sum(min(x.tn, x.n - j * x.tn) for j in cols)
    return DGrid(m, n, x.tm, x.tn, len(rows), len(cols), ptrs.data_ptr(), x.bclx_dtype, 0), ptrs


def _check_spmm(a: SPMatrix, b: DMatrix, c: DMatrix):
    if a.n != b.m or a.m != c.m or b.n != c.n:
        raise RuntimeError("BCL::gemm: shape mismatch")
    if a.dtype != np.float32:
        raise TypeError("SpMM needs FP32 sparse values")


def _increasing(tile_rows, tile_cols):
    tile_rows, tile_cols = list(tile_rows), list(tile_cols)
    if any(q <= p for p, q in zip(tile_rows, tile_rows[1:])) or any(q <= p for p, q in zip(tile_cols, tile_cols[1:])):
        raise ValueError("tile rows and columns must be increasing")
    return tile_rows, tile_cols


def _spmm_grid_sub(device, ag, bg, cg, tile_rows, tile_cols):
    h = context(device).use_current_stream()
    rows_arr = (ctypes.c_int64 * max(len(tile_rows), 1))(*tile_rows)
    cols_arr = (ctypes.c_int64 * max(len(tile_cols), 1))(*tile_cols)
    call("bclx_spmm_grid_sub", h, ctypes.byref(ag), ctypes.byref(bg), ctypes.byref(cg), rows_arr, cols_arr)


def spmm_sub(a: SPMatrix, b: DMatrix, c: DMatrix, tile_rows, tile_cols) -> None:
    """C += A * B for the C tiles (i, j), i in tile_rows, j in tile_cols
    (increasing global tile indices), in place in c's tiles, each over all k
    in the rotated order of its global position: what one process of the
    reference's stationary-C loop computes (spgemm.hpp:153-179 under
    c.tile_rank), in one launch (bclx_spmm_grid_sub); bit-identical to those
    tiles of spmm(a, b, c)."""
    _check_spmm(a, b, c)
    tile_rows, tile_cols = _increasing(tile_rows, tile_cols)
    if not tile_rows or not tile_cols:
        return
    ag, adesc = _sub_spgrid(a, tile_rows, range(a.gn))
    bg, bptr = _sub_dgrid(b, range(b.gm), tile_cols)
    cg, cptr = _sub_dgrid(c, tile_rows, tile_cols)
    _spmm_grid_sub(a.device, ag, bg, cg, tile_rows, tile_cols)
    del adesc, bptr, cptr  # (the launches are ordered on the stream before any reuse)


def spmm_compact(a: SPMatrix, b: DMatrix, c: DMatrix, tile_rows, tile_cols) -> None:
    """C += A * B on operands held as compact grids: `a` holds exactly A's
    tile rows tile_rows (its tile (x, k) is global tile (tile_rows[x], k)),
    `b` B's tile columns tile_cols and `c` the C tiles tile_rows x
    tile_cols (as a process of a distributed product holds them after
    fetching its operands, bcl_b200.distributed).  Every C tile is
    bit-identical to that tile of the whole product."""
    _check_spmm(a, b, c)
    tile_rows, tile_cols = _increasing(tile_rows, tile_cols)
    if a.gm != len(tile_rows) or c.gm != len(tile_rows) or c.gn != len(tile_cols) or b.gn != len(tile_cols):
        raise RuntimeError("BCL::gemm: compact operand grids do not match the tile lists")
    if not tile_rows or not tile_cols:
        return
    _spmm_grid_sub(a.device, a.spgrid(), b.dgrid(), c.dgrid(), tile_rows, tile_cols)


def rowwise_gemm(a: SPMatrix, b: DMatrix, c: DMatrix) -> None:
    """C += A * B with C in one tile column, every C tile row taking the k
    tiles in ascending order (rowwise_gemm, experimental_gemm.hpp:83-123)."""
    if a.n != b.m or a.m != c.m or b.n != c.n:
        raise RuntimeError("BCL::rowwise_gemm: shape mismatch")
    if c.gn != 1:
        raise RuntimeError("BCL::rowwise_gemm: C must have one tile column")
    h = context(a.device).use_current_stream()
    call("bclx_spmm_grid_rowwise", h, ctypes.byref(a.spgrid()), ctypes.byref(b.dgrid()), ctypes.byref(c.dgrid()))


def cached_rowwise_gemm(a: SPMatrix, b: DMatrix, c: DMatrix, cache_size: int = 0) -> None:
    """cached_rowwise_gemm (experimental_gemm.hpp:125-165): the reference
    caches fetched B rows in `cache_size` bytes; here B is resident in HBM,
    so the cache size does not matter and the sums are rowwise_gemm's."""
    rowwise_gemm(a, b, c)


def batched_rowwise_gemm(a: SPMatrix, b: DMatrix, c: DMatrix) -> None:
    """batched_rowwise_gemm (experimental_gemm.hpp:167-212): the reference
    sorts a tile's entries by B row to fetch each once; entries of one C row
    keep their order, so the sums are rowwise_gemm's."""
    rowwise_gemm(a, b, c)


def spmm_plain(a: SPMatrix, b: DMatrix, c: DMatrix) -> None:
    """The reference's loop, one spmm_wrapper call per tile product
    (spgemm.hpp:153-179)."""
    if a.n != b.m or a.m != c.m or b.n != c.n:
        raise RuntimeError("BCL::gemm: shape mismatch")
    h = context(a.device).use_current_stream()
    o = a._offsets()
    G = a.gn
    es = b.tiles.element_size()
    for i in range(c.gm):
        for j in range(c.gn):
            for k_ in range(G):
                k = (k_ + i + j) % G
                t = i * a.gn + k
                m, n = c.tile_shape((i, j))
                call("bclx_spmm_tile", h, m, n, a.tile_shape((i, k))[1], int(o[t + 1] - o[t]),
                     ctypes.c_void_p(c.tile_ptr((i, j))), ctypes.c_void_p(b.tile_ptr((k, j))),
                     ctypes.c_void_p(a.vals.data_ptr() + int(o[t]) * 4),
                     ctypes.c_void_p(a.tile_row_ptr[t].data_ptr()),
                     ctypes.c_void_p(a.col_ind.data_ptr() + int(o[t]) * 4), b.tn, c.tn, c.bclx_dtype)
    del es


def gemm(a, b, c=None):
    """BCL::gemm(a, b, c): sparse x sparse returns the product SPMatrix (c, if
    given, is replaced tile by tile, as assign_tile does); sparse x dense
    accumulates into the DMatrix c in place."""
    if isinstance(a, SPMatrix) and isinstance(b, SPMatrix):
        res = spgemm(a, b)
        if c is not None:
            if (c.m, c.n, c.tm, c.tn) != (res.m, res.n, res.tm, res.tn):
                raise RuntimeError("BCL::gemm: C has a different tile grid")
            c.tile_row_ptr, c.tile_offset, c.col_ind, c.vals = res.tile_row_ptr, res.tile_offset, res.col_ind, res.vals
            c._build_desc()
            return c
        return res
    if isinstance(a, SPMatrix) and isinstance(b, DMatrix):
        if c is None:
            raise TypeError("sparse x dense gemm needs the output DMatrix")
        spmm(a, b, c)
        return c
    raise TypeError("BCL::gemm: unsupported operand types")
