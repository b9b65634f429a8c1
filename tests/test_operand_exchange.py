"""Distributed operands on CPU (gloo ranks): every process holds only the A
and B tiles it owns in the reference's block-cyclic layout
(SPMatrix.hpp:230-237), fetches the A tiles of its C tile rows along its
process row and the B tiles of its C tile columns along its process column
(bcl_b200.distributed.exchange_operands), computes its C tiles from what it
received (the oracle stands in for the device kernels), and rank 0 gathers
the sub-grids: the assembled product equals the whole product bit for bit."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _operands(value_type, tiles=(100, 70, 90)):
    """Two 512 x 512 R-MAT matrices; the default tiles are ragged at the
    edge in every dimension."""
    from bcl_b200 import gen
    a = gen.rmat(9, seed=31, value_type=value_type)
    b = gen.rmat(9, seed=32, value_type=value_type)
    return (a, b) + tuple(tiles)


def _from_tiles(tiles, rows, cols, tr, tc, m, n, dtype):
    """A host CSR of shape m x n holding the tiles (i, j), i in rows, j in
    cols (global positions), and nothing else."""
    from bcl_b200.gen import CSR
    rows, cols = set(rows), sorted(cols)
    rp, cis, vs = [0], [], []
    for r in range(m):
        i, lr = divmod(r, tr)
        added = 0
        if i in rows:
            for j in cols:
                trp, tci, tv = (t.numpy() for t in tiles[(i, j)])
                s, e = int(trp[lr]), int(trp[lr + 1])
                cis.append(tci[s:e].astype(np.int32) + j * tc)
                vs.append(tv[s:e])
                added += e - s
        rp.append(rp[-1] + added)
    ci = np.concatenate(cis) if cis else np.zeros(0, np.int32)
    v = np.concatenate(vs) if vs else np.zeros(0, dtype)
    return CSR(m, n, np.asarray(rp, np.int32), ci.astype(np.int32), v.astype(dtype))


def _owned_part(rp, ci, cv, rows, cols, tm, tn, m, n):
    """The C tiles rows x cols of a host product, packed as a sub-grid
    (rows, cols, tile_row_ptr, tile_offset, col_ind, vals)."""
    trp, toff, cis, vs = [], [0], [], []
    for i in rows:
        for j in cols:
            loc = [0]
            for r in range(i * tm, min((i + 1) * tm, m)):
                seg = slice(rp[r], rp[r + 1])
                sel = (ci[seg] >= j * tn) & (ci[seg] < min((j + 1) * tn, n))
                cis.append(ci[seg][sel] - j * tn)
                vs.append(cv[seg][sel])
                loc.append(loc[-1] + int(sel.sum()))
            loc += [loc[-1]] * (tm + 1 - len(loc))
            trp.append(loc)
            toff.append(toff[-1] + loc[-1])
    return (rows, cols, np.asarray(trp, np.int32).reshape(-1, tm + 1), np.asarray(toff, np.int64),
            np.concatenate(cis).astype(np.int32) if cis else np.zeros(0, np.int32),
            np.concatenate(vs) if vs else np.zeros(0, cv.dtype))


def _exchange_rank(rank, world, pgrid, value_type, tiles, port, out):
    import torch.distributed as tdist
    from bcl_b200.containers import assemble_tiles
    from bcl_b200.distributed import ProcessGroups, exchange_operands, host_tile, owned_input_tiles
    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        a, b, tm, tk, tn = _operands(value_type, tiles)
        pm, pn = pgrid
        groups = ProcessGroups(world, pm, pn)
        a_own = owned_input_tiles(a, tm, tk, rank, pm, pn)
        b_own = owned_input_tiles(b, tk, tn, rank, pm, pn)
        vdt = torch.float32 if value_type == "f32" else torch.int32
        a_rows, b_cols, I, J = exchange_operands(a_own, (a.m, a.n), b_own, (b.m, b.n), tm, tk, tn, rank, groups,
                                                 val_dtype=vdt)
        gk = -(-a.n // tk)
        # every tile received is the owner's tile, bit for bit
        ok = set(a_rows) == {(i, k) for i in I for k in range(gk)}
        ok &= set(b_cols) == {(k, j) for k in range(gk) for j in J}
        for (i, k), t in a_rows.items():
            ref = host_tile(a, tm, tk, i, k)
            ok &= all(np.array_equal(x.numpy().view(np.uint32) if x.dtype != torch.int32 else x.numpy(),
                                     y.view(np.uint32) if y.dtype != np.int32 else y) for x, y in zip(t, ref))
        for (k, j), t in b_cols.items():
            ref = host_tile(b, tk, tn, k, j)
            ok &= all(np.array_equal(x.numpy().view(np.uint32) if x.dtype != torch.int32 else x.numpy(),
                                     y.view(np.uint32) if y.dtype != np.int32 else y) for x, y in zip(t, ref))
        fetched = sum(1 for key in a_rows if key not in a_own) + sum(1 for key in b_cols if key not in b_own)
        # this process's C tiles from the received operands only
        ar = _from_tiles(a_rows, I, range(gk), tm, tk, a.m, a.n, a.vals.dtype)
        bc = _from_tiles(b_cols, range(gk), J, tk, tn, b.m, b.n, b.vals.dtype)
        if I and J:
            rp, ci, cv = O.gemm_tiled(ar, bc, tm, tk, tn, mode=value_type)
            part = _owned_part(rp, ci, cv, I, J, tm, tn, a.m, b.n)
        else:  # no C tile here; the process still served its tiles to the others
            part = None
        gathered = [None] * world if rank == 0 else None
        tdist.gather_object((part, ok, fetched), gathered, dst=0)
        if rank == 0:
            whole = assemble_tiles(a.m, b.n, tm, tn, [g[0] for g in gathered if g[0] is not None])
            wrp, wci, wcv = O.gemm_tiled(a, b, tm, tk, tn, mode=value_type)
            out["ok"] = all(g[1] for g in gathered)
            out["fetched"] = [g[2] for g in gathered]
            out["idle"] = sum(g[0] is None for g in gathered)
            out["same"] = (np.array_equal(whole.row_ptr.astype(np.int64), wrp) and np.array_equal(whole.col_ind, wci)
                           and np.array_equal(whole.vals.view(np.uint32), wcv.view(np.uint32)))
            out["nnz"] = int(wrp[-1])
    finally:
        tdist.destroy_process_group()


def _run(world, pgrid, value_type, tiles):
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_exchange_rank, args=(world, pgrid, value_type, tiles, port, out), nprocs=world, join=True)
        return dict(out)


@pytest.mark.parametrize("world,pgrid,value_type", [(2, (1, 2), "f32"), (4, (2, 2), "f32"), (3, (3, 1), "i32"),
                                                    (4, (2, 2), "i32")])
def test_exchange_serves_the_whole_product(world, pgrid, value_type):
    res = _run(world, pgrid, value_type, (100, 70, 90))
    assert res["ok"], "a received tile differs from its owner's"
    assert all(f > 0 for f in res["fetched"]), "every process needs tiles it does not own"
    assert res["same"] and res["nnz"] > 0 and res["idle"] == 0


def test_exchange_with_processes_that_own_no_c_tile():
    """One tile row and one tile column of C on a 2 x 2 process grid: three
    processes own no C tile but hold operand tiles (k is cut in 8) and must
    still serve them; rank 0 computes the whole product."""
    res = _run(4, (2, 2), "f32", (512, 70, 512))
    assert res["ok"] and res["same"] and res["idle"] == 3


def test_pack_tiles_matches_the_grid_layout():
    """pack_tiles lays out a compact grid exactly as an SPMatrix packs the
    same tiles (split_tiles of the matrix that holds them): tile row
    pointers with edge tiles padded by their nnz, offsets, columns, values."""
    from bcl_b200.containers import split_tiles
    from bcl_b200.distributed import host_tile, pack_tiles
    a, _, tm, tk, _ = _operands("f32")
    gm, gk = -(-a.m // tm), -(-a.n // tk)
    rows = [i for i in range(gm) if i % 2 == 1]  # includes the short last tile row
    assert rows[-1] == gm - 1
    tiles = {(i, k): tuple(torch.from_numpy(x) for x in host_tile(a, tm, tk, i, k)) for i in rows for k in range(gk)}
    trp, toff, ci, v = pack_tiles(tiles, rows, list(range(gk)), tm, torch.float32, "cpu")
    # the same tiles as one host matrix: rows of tile rows `rows`, stacked
    keep = np.concatenate([np.arange(i * tm, min((i + 1) * tm, a.m)) for i in rows])
    rp = np.concatenate([[0], np.cumsum(np.diff(a.row_ptr)[keep])]).astype(np.int32)
    sel = np.concatenate([np.arange(a.row_ptr[r], a.row_ptr[r + 1]) for r in keep]).astype(np.int64)
    from bcl_b200.gen import CSR
    sub = CSR(len(keep), a.n, rp, a.col_ind[sel], a.vals[sel])
    etrp, etoff, eci, ev = split_tiles(sub, tm, tk)
    assert np.array_equal(trp.numpy(), etrp) and np.array_equal(toff.numpy(), etoff)
    assert np.array_equal(ci.numpy(), eci) and np.array_equal(v.numpy().view(np.uint32), ev.view(np.uint32))


def test_owned_input_tiles_partition_the_matrix():
    """Every tile of the matrix is held by exactly one process, the one the
    reference's formula names."""
    from bcl_b200.distributed import owned_input_tiles, tile_owner
    a, _, tm, tk, _ = _operands("f32")
    pm, pn = 2, 3
    seen = {}
    for p in range(pm * pn):
        for key, t in owned_input_tiles(a, tm, tk, p, pm, pn).items():
            assert key not in seen and tile_owner(*key, pm, pn) == p
            seen[key] = int(t[1].numel())
    assert len(seen) == (-(-a.m // tm)) * (-(-a.n // tk)) and sum(seen.values()) == a.nnz


def _spmm_exchange_rank(rank, world, pgrid, port, out):
    """The sparse x dense product with distributed operands: A sparse and B,
    C dense, every tile on its owner; A along process rows, dense B along
    process columns; each process's C tiles from what it received (oracle)."""
    import torch.distributed as tdist
    from bcl_b200 import gen
    from bcl_b200.distributed import (ProcessGroups, exchange_spmm_operands, host_tile, owned_dense_tiles,
                                      owned_input_tiles)
    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        a = gen.rmat(9, seed=33)
        n = 200
        b = gen.dense(a.n, n, seed=34)
        c0 = gen.dense(a.m, n, seed=35)
        tm, tk, tn = 100, 70, 64  # ragged in every dimension
        pm, pn = pgrid
        groups = ProcessGroups(world, pm, pn)
        a_own = owned_input_tiles(a, tm, tk, rank, pm, pn)
        b_own = owned_dense_tiles(b, tk, tn, rank, pm, pn)
        c_own = owned_dense_tiles(c0, tm, tn, rank, pm, pn)
        a_rows, b_cols, I, J = exchange_spmm_operands(a_own, (a.m, a.n), b_own, (b.shape[0], n), tm, tk, tn, rank,
                                                      groups)
        gk = -(-a.n // tk)
        ok = set(c_own) == {(i, j) for i in I for j in J}  # C tiles stay with their owner
        ok &= set(b_cols) == {(k, j) for k in range(gk) for j in J}
        for (k, j), t in b_cols.items():
            want = np.zeros((tk, tn), np.float32)
            blk = b[k * tk:(k + 1) * tk, j * tn:(j + 1) * tn]
            want[:blk.shape[0], :blk.shape[1]] = blk
            ok &= np.array_equal(t.numpy().view(np.uint32), want.view(np.uint32))
        for (i, k), t in a_rows.items():
            ref = host_tile(a, tm, tk, i, k)
            ok &= all(np.array_equal(x.numpy().view(np.uint32) if x.dtype != torch.int32 else x.numpy(),
                                     y.view(np.uint32) if y.dtype != np.int32 else y) for x, y in zip(t, ref))
        # C tiles I x J from the received operands only: A's rows I, B's columns J
        ar = _from_tiles(a_rows, I, range(gk), tm, tk, a.m, a.n, np.float32)
        bc = np.zeros_like(b)
        for (k, j), t in b_cols.items():
            blk = bc[k * tk:(k + 1) * tk, j * tn:(j + 1) * tn]
            blk[...] = t.numpy()[:blk.shape[0], :blk.shape[1]]
        tiles = {}
        if I and J:
            cc = O.spmm_tiled(ar, bc, c0, tm, tk, tn)
            tiles = {(i, j): cc[i * tm:(i + 1) * tm, j * tn:(j + 1) * tn].copy() for i in I for j in J}
        gathered = [None] * world if rank == 0 else None
        tdist.gather_object((tiles, ok), gathered, dst=0)
        if rank == 0:
            whole = np.array(c0, copy=True)
            seen = 0
            for part, _ in gathered:
                for (i, j), blk in part.items():
                    whole[i * tm:(i + 1) * tm, j * tn:(j + 1) * tn] = blk
                    seen += 1
            want = O.spmm_tiled(a, b, c0, tm, tk, tn)
            out["ok"] = all(g[1] for g in gathered)
            out["tiles"] = seen
            out["same"] = np.array_equal(whole.view(np.uint32), want.view(np.uint32))
    finally:
        tdist.destroy_process_group()


@pytest.mark.parametrize("world,pgrid", [(2, (1, 2)), (4, (2, 2)), (3, (3, 1))])
def test_spmm_exchange_serves_the_whole_product(world, pgrid):
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_spmm_exchange_rank, args=(world, pgrid, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res["ok"], "a received tile differs from its owner's, or C tiles moved"
    assert res["tiles"] == 6 * 4 and res["same"]


def _rank_leaves(rank, world, port, out):
    """Rank 1 leaves before the exchange (between steps, nothing in
    flight); rank 0 must get an error from its next collective, within the
    process group's timeout, instead of waiting for ever."""
    from datetime import timedelta
    import time
    import torch.distributed as tdist
    from bcl_b200.distributed import ProcessGroups, exchange_operands, owned_input_tiles
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    tdist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=10))
    groups = ProcessGroups(world, 1, world)
    a, b, tm, tk, tn = _operands("f32")
    if rank == 1:
        out["left"] = True
        return  # leaves without destroying the group: its peers see it gone
    t0 = time.time()
    try:
        exchange_operands(owned_input_tiles(a, tm, tk, rank, 1, world), (a.m, a.n),
                          owned_input_tiles(b, tk, tn, rank, 1, world), (b.m, b.n), tm, tk, tn, rank, groups)
        out["error"] = None
    except RuntimeError as e:
        out["error"] = type(e).__name__
    out["seconds"] = time.time() - t0


def test_exchange_fails_fast_when_a_rank_leaves():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_leaves, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res["left"] and res["error"] is not None
    assert res["seconds"] < 60
