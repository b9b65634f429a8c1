"""Distributed inputs for the stationary-C SUMMA product: each process holds
only the A and B tiles it owns, and fetches the others it needs.

The reference places tile (i, j) of every SPMatrix on process
(j % pn) + (i % pm) * pn of a pm x pn process grid (SPMatrix.hpp:230-237),
and its product loop fetches each remote A_ik / B_kj tile from its owner
(spgemm.hpp:194-224; the GPU driver broadcasts them,
cuda/algorithms/spgemm.hpp:164-292).  Process (r, c) owns the C tiles
I x J with I = {i : i % pm = r} and J = {j : j % pn = c}; it needs the A
tiles (i, k), i in I, whose owners (r, k % pn) are in its process row, and
the B tiles (k, j), j in J, whose owners (k % pm, c) are in its process
column.  So one exchange serves the whole product: every owner broadcasts
its tiles once within its process row (A) and its process column (B), sparse
tiles packed into three buffers (per-tile entry counts, then the int32 row
pointers and column indices, then the values), dense tiles into one.  Over
NCCL the buffers are device tensors and land in local HBM, where the
sub-grid products read them (`spgemm_owned`, `spmm_owned`); over gloo they
are host tensors.  The sparse x dense product (spgemm.hpp:153-179; its GPU
driver cuda/algorithms/spmm.hpp:20-115) places dense tiles the same way
(DMatrix.hpp:75-90), so the same exchange serves it with B dense.
"""
from __future__ import annotations

from typing import Dict, List, Optional, Tuple

import numpy as np
import torch

Tile = Tuple[torch.Tensor, torch.Tensor, torch.Tensor]  # row_ptr [rows+1] int32, col_ind int32, vals


def tile_owner(i: int, j: int, pm: int, pn: int) -> int:
    """Process holding tile (i, j) (SPMatrix.hpp:230-237)."""
    return (j % pn) + (i % pm) * pn


def _ceil_div(a: int, b: int) -> int:
    return -(-a // b)


def host_tile(mat, tm: int, tn: int, i: int, j: int) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Tile (i, j) of a host CSR matrix (columns ascending within rows): row
    pointers from 0, tile-local columns, values (SPMatrix's slicing,
    CSRMatrix.hpp:238-276)."""
    r0, r1 = i * tm, min((i + 1) * tm, mat.m)
    c0, c1 = j * tn, min((j + 1) * tn, mat.n)
    rp = [0]
    cis, vs = [], []
    for r in range(r0, r1):
        s, e = int(mat.row_ptr[r]), int(mat.row_ptr[r + 1])
        cols = mat.col_ind[s:e]
        lo, hi = np.searchsorted(cols, c0), np.searchsorted(cols, c1)
        cis.append(cols[lo:hi] - c0)
        vs.append(mat.vals[s + lo:s + hi])
        rp.append(rp[-1] + int(hi - lo))
    ci = np.concatenate(cis).astype(np.int32) if cis else np.zeros(0, np.int32)
    v = np.concatenate(vs) if vs else np.zeros(0, mat.vals.dtype)
    return np.asarray(rp, np.int32), ci, np.ascontiguousarray(v)


def owned_input_tiles(mat, tm: int, tn: int, rank: int, pm: int, pn: int, device="cpu") -> Dict[Tuple[int, int], Tile]:
    """The tiles of `mat` that process `rank` holds when the matrix is
    distributed as the reference distributes it (what SPMatrix(fname,
    blocking) keeps on each process)."""
    from .containers import split_tiles
    gm, gn = _ceil_div(mat.m, tm), _ceil_div(mat.n, tn)
    trp, toff, ci, v = split_tiles(mat, tm, tn)  # every tile at once, packed in grid order
    out = {}
    for i in range(gm):
        for j in range(gn):
            if tile_owner(i, j, pm, pn) == rank:
                t = i * gn + j
                rows = min(tm, mat.m - i * tm)
                lo, hi = int(toff[t]), int(toff[t + 1])
                out[(i, j)] = (torch.from_numpy(np.ascontiguousarray(trp[t, :rows + 1])).to(device),
                               torch.from_numpy(np.ascontiguousarray(ci[lo:hi])).to(device),
                               torch.from_numpy(np.ascontiguousarray(v[lo:hi])).to(device))
    return out


class ProcessGroups:
    """The row and column communicators of a pm x pn process grid.  Every
    process must create them, in the same order (torch.distributed.new_group)."""

    def __init__(self, world: int, pm: int, pn: int):
        import torch.distributed as tdist
        assert pm * pn == world
        self.pm, self.pn = pm, pn
        self.rows = [tdist.new_group([r * pn + c for c in range(pn)]) for r in range(pm)]
        self.cols = [tdist.new_group([r * pn + c for r in range(pm)]) for c in range(pn)]


def _broadcast_tiles(keys: List[Tuple[int, int]], rows_of, owned: Dict, src: int, me: int, group, device,
                     val_dtype) -> Dict[Tuple[int, int], Tile]:
    """Tiles `keys` from process `src` to every member of `group`: the entry
    counts, then the int32 row pointers and column indices in one buffer,
    then the values."""
    import torch.distributed as tdist
    if not keys:
        return {}
    nrows = [rows_of(k) for k in keys]
    if me == src:
        tiles = [owned[k] for k in keys]
        nnz = torch.tensor([int(t[1].numel()) for t in tiles], dtype=torch.int64, device=device)
    else:
        nnz = torch.empty(len(keys), dtype=torch.int64, device=device)
    tdist.broadcast(nnz, src=src, group=group)
    counts = nnz.cpu().tolist()
    n_int = sum(r + 1 for r in nrows) + sum(counts)
    if me == src:
        ints = torch.cat([t[0] for t in tiles] + [t[1] for t in tiles]).to(torch.int32).contiguous()
        vals = torch.cat([t[2] for t in tiles]).contiguous() if sum(counts) else torch.zeros(1, dtype=val_dtype,
                                                                                          device=device)
    else:
        ints = torch.empty(n_int, dtype=torch.int32, device=device)
        vals = torch.empty(max(sum(counts), 1), dtype=val_dtype, device=device)
    tdist.broadcast(ints, src=src, group=group)
    tdist.broadcast(vals, src=src, group=group)
    if me == src:
        return {k: owned[k] for k in keys}
    out = {}
    p = 0
    q = sum(r + 1 for r in nrows)
    vpos = 0
    for k, r, c in zip(keys, nrows, counts):
        out[k] = (ints[p:p + r + 1], ints[q:q + c], vals[vpos:vpos + c])
        p += r + 1
        q += c
        vpos += c
    return out


def exchange_operands(a_own: Dict, a_shape: Tuple[int, int], b_own: Dict, b_shape: Tuple[int, int],
                      tm: int, tk: int, tn: int, rank: int, groups: ProcessGroups, device="cpu",
                      val_dtype=torch.float32):
    """Fetch the A tiles of this process's C tile rows and the B tiles of its
    C tile columns from their owners.  a_own / b_own: the tiles this process
    holds ({(i, j): (row_ptr, col_ind, vals)}).  Returns (a_rows, b_cols, I,
    J): a_rows[(i, k)] for i in I and every k, b_cols[(k, j)] for every k and
    j in J, I and J this process's C tile rows and columns.  Every process of
    the grid calls it (the broadcasts are collective within process rows and
    columns); a process that owns no tile still takes part."""
    I, J, gk = _owned_lines(a_shape, b_shape, tm, tk, tn, rank, groups)
    a_rows = _exchange_a_rows(a_own, a_shape[0], tm, gk, I, rank, groups, device, val_dtype)
    pm, pn = groups.pm, groups.pn
    c = rank % pn
    kdim = a_shape[1]
    b_cols: Dict = {}
    for rr in range(pm):  # B along the process column, owner by owner
        keys = [(k, j) for k in range(gk) if k % pm == rr for j in J]
        b_cols.update(_broadcast_tiles(keys, lambda key: min(tk, kdim - key[0] * tk), b_own, rr * pn + c, rank,
                                       groups.cols[c], device, val_dtype))
    return a_rows, b_cols, I, J


def _owned_lines(a_shape, b_shape, tm: int, tk: int, tn: int, rank: int, groups: ProcessGroups):
    """This process's C tile rows I and columns J, and the number of k tiles."""
    r, c = divmod(rank, groups.pn)
    m, kdim = a_shape
    n = b_shape[1]
    I = [i for i in range(_ceil_div(m, tm)) if i % groups.pm == r]
    J = [j for j in range(_ceil_div(n, tn)) if j % groups.pn == c]
    return I, J, _ceil_div(kdim, tk)


def _exchange_a_rows(a_own: Dict, m: int, tm: int, gk: int, I: List[int], rank: int, groups: ProcessGroups, device,
                     val_dtype) -> Dict:
    """A's tiles (i, k), i in I, every k, along the process row: process
    (r, cc) broadcasts the tiles with k % pn == cc that the row needs."""
    pn = groups.pn
    r = rank // pn
    a_rows: Dict = {}
    for cc in range(pn):
        keys = [(i, k) for i in I for k in range(gk) if k % pn == cc]
        a_rows.update(_broadcast_tiles(keys, lambda key: min(tm, m - key[0] * tm), a_own, r * pn + cc, rank,
                                       groups.rows[r], device, val_dtype))
    return a_rows


def owned_dense_tiles(arr, tm: int, tn: int, rank: int, pm: int, pn: int, dtype=torch.float32,
                      device="cpu") -> Dict[Tuple[int, int], torch.Tensor]:
    """The tiles of a dense m x n matrix that process `rank` holds in the
    reference's layout (DMatrix.hpp:75-90: tile (i, j) on process
    (j % pn) + (i % pm) * pn), each tm x tn row-major and zero-padded at the
    edges as a DMatrix tile is."""
    full = torch.as_tensor(arr)
    m, n = full.shape
    out = {}
    for i in range(_ceil_div(m, tm)):
        for j in range(_ceil_div(n, tn)):
            if tile_owner(i, j, pm, pn) == rank:
                t = torch.zeros((tm, tn), dtype=dtype, device=device)
                blk = full[i * tm:(i + 1) * tm, j * tn:(j + 1) * tn]
                t[:blk.shape[0], :blk.shape[1]] = blk.to(device=device, dtype=dtype)
                out[(i, j)] = t
    return out


def _broadcast_dense(keys: List[Tuple[int, int]], owned: Dict, src: int, me: int, group, shape, dtype,
                     device) -> Dict[Tuple[int, int], torch.Tensor]:
    """Dense tiles `keys` from process `src` to every member of `group`, in
    one buffer."""
    import torch.distributed as tdist
    if not keys:
        return {}
    if me == src:
        buf = torch.stack([owned[k] for k in keys]).contiguous()
    else:
        buf = torch.empty((len(keys),) + tuple(shape), dtype=dtype, device=device)
    tdist.broadcast(buf, src=src, group=group)
    if me == src:
        return {k: owned[k] for k in keys}
    return {k: buf[x] for x, k in enumerate(keys)}


def exchange_spmm_operands(a_own: Dict, a_shape: Tuple[int, int], b_own: Dict, b_shape: Tuple[int, int],
                           tm: int, tk: int, tn: int, rank: int, groups: ProcessGroups, device="cpu",
                           b_dtype=torch.float32):
    """The operands of this process's C tiles for the sparse x dense product
    (spgemm.hpp:153-179; the GPU driver's broadcasts,
    cuda/algorithms/spmm.hpp:20-115): the sparse A tiles of its C tile rows
    along its process row, and the dense B tiles (tk x tn, padded) of its C
    tile columns along its process column.  The C tiles I x J are this
    process's own (the same layout) and do not move.  Returns (a_rows,
    b_cols, I, J); every process of the grid calls it."""
    I, J, gk = _owned_lines(a_shape, b_shape, tm, tk, tn, rank, groups)
    a_rows = _exchange_a_rows(a_own, a_shape[0], tm, gk, I, rank, groups, device, torch.float32)
    pm, pn = groups.pm, groups.pn
    c = rank % pn
    b_cols: Dict = {}
    for rr in range(pm):  # dense B along the process column
        keys = [(k, j) for k in range(gk) if k % pm == rr for j in J]
        b_cols.update(_broadcast_dense(keys, b_own, rr * pn + c, rank, groups.cols[c], (tk, tn), b_dtype, device))
    return a_rows, b_cols, I, J


def pack_tiles(tiles: Dict, rows: List[int], cols: List[int], tm: int, val_dtype, device):
    """The tiles (rows[a], cols[b]) in that order, packed as an SPMatrix
    packs its grid: tile_row_ptr [ntiles, tm+1] int32 (an edge tile's last
    entries repeat its nnz), tile_offset [ntiles+1] int64, col_ind, vals."""
    td = torch.device(device)
    gm, gn = len(rows), len(cols)
    trp = torch.empty((gm * gn, tm + 1), dtype=torch.int32, device=td)
    offs = [0]
    cis, vs = [], []
    for a_, i in enumerate(rows):
        for b_, j in enumerate(cols):
            rp, ci, v = tiles[(i, j)]
            nr = rp.numel() - 1
            t = a_ * gn + b_
            trp[t, :nr + 1] = rp.to(td)
            trp[t, nr + 1:] = int(rp[-1])
            cis.append(ci.to(td))
            vs.append(v.to(td))
            offs.append(offs[-1] + int(ci.numel()))
    toff = torch.tensor(offs, dtype=torch.int64, device=td)
    ci = torch.cat(cis) if cis else torch.zeros(0, dtype=torch.int32, device=td)
    v = torch.cat(vs) if vs else torch.zeros(0, dtype=val_dtype, device=td)
    return trp, toff, ci, v


def pack_grid(tiles: Dict, rows: List[int], cols: List[int], tm: int, tn: int, m: int, n: int, dtype,
              device: int):
    """An SPMatrix of the tiles (rows[a], cols[b]) in that order (a compact
    grid: its tile (a, b) is global tile (rows[a], cols[b])), packed on the
    device.  m, n: the global shape (for the edge tiles; only the last tile
    row or column of the global grid can be short, and it stays last)."""
    from .containers import _NP_TO_DT, _TORCH_OF, SPMatrix
    trp, toff, ci, v = pack_tiles(tiles, rows, cols, tm, _TORCH_OF[_NP_TO_DT[np.dtype(dtype)]],
                                  torch.device("cuda", device))
    mm = sum(min(tm, m - i * tm) for i in rows)
    nn = sum(min(tn, n - j * tn) for j in cols)
    return SPMatrix(mm, nn, tm, tn, dtype, device, trp, toff, ci, v)


def spmm_owned(a_rows: Dict, b_cols: Dict, c_tiles: Dict, I: List[int], J: List[int], a_shape, b_shape, tm: int,
               tk: int, tn: int, device: Optional[int] = None):
    """C += A * B for this process's C tiles I x J on the GPU, from the
    fetched operand tiles: A's rows I packed as a compact sparse grid, B's
    columns J and the C tiles (c_tiles[(i, j)], tm x tn) stacked as compact
    dense grids, one launch through bclx_spmm_grid_sub with the global tile
    indices.  Returns the C tiles ({(i, j): tm x tn tensor on the device},
    bit-identical to those tiles of the whole product), or {} for a process
    that owns no C tile."""
    from .containers import DMatrix, spmm_compact
    if not I or not J:
        return {}
    dev = torch.cuda.current_device() if device is None else device
    td = torch.device("cuda", dev)
    m, kdim = a_shape
    _, n = b_shape
    gk = _ceil_div(kdim, tk)
    A = pack_grid(a_rows, I, list(range(gk)), tm, tk, m, kdim, np.float32, dev)
    kk = list(range(gk))
    bt = torch.stack([b_cols[(k, j)].to(td) for k in kk for j in J]).contiguous()
    ct = torch.stack([c_tiles[(i, j)].to(td) for i in I for j in J]).contiguous()
    nn = sum(min(tn, n - j * tn) for j in J)
    mm = sum(min(tm, m - i * tm) for i in I)
    B = DMatrix(kdim, nn, tk, tn, bt)
    C = DMatrix(mm, nn, tm, tn, ct)
    spmm_compact(A, B, C, I, J)
    return {(i, j): C.tiles[x * len(J) + y] for x, i in enumerate(I) for y, j in enumerate(J)}


def spgemm_owned(a_rows: Dict, b_cols: Dict, I: List[int], J: List[int], a_shape, b_shape, tm: int, tk: int,
                 tn: int, dtype=np.float32, device: Optional[int] = None):
    """This process's C tiles I x J from the fetched operand tiles, on the
    GPU: A's rows I and B's columns J packed into compact grids, the product
    through bclx_spgemm_symbolic_sub with the global tile indices (so every
    tile keeps the stage order k = (k_ + i + j) mod G of its global
    position).  Returns the C sub-grid (an SPMatrix in I x J order), or None
    for a process that owns no C tile (more processes than tile rows or
    columns)."""
    from .containers import spgemm_compact
    if not I or not J:
        return None
    dev = torch.cuda.current_device() if device is None else device
    m, kdim = a_shape
    _, n = b_shape
    gk = _ceil_div(kdim, tk)
    A = pack_grid(a_rows, I, list(range(gk)), tm, tk, m, kdim, dtype, dev)
    B = pack_grid(b_cols, list(range(gk)), J, tk, tn, kdim, n, dtype, dev)
    return spgemm_compact(A, B, I, J)
