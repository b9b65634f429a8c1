"""The N>1 path of bench.py on CPU: two gloo ranks (torchrun-style env).
Each rank multiplies its own independent matrix, so the only collectives are
the barrier and the max of the ranks' times; rank 0 alone reports, and the
reference arm runs on rank 0 only."""
import importlib.util
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    bench = _bench()
    dist = bench.Dist(backend="gloo")
    try:
        dist.barrier()
        # rank r "took" 1 + r seconds; the job takes the slowest
        t = dist.max(1.0 + rank)
        rate = bench.job_rate(dist.world, 10.0, 4, t)

        class Args:
            workload, seed, steps, warmup, gpus = "spgemm_rmat16", 1, 1, 0, world

        ref = bench.run_reference(Args, dist) if rank != 0 else "rank0-skipped"
        out[rank] = (dist.world, t, rate, ref)
        dist.barrier()
    finally:
        dist.close()


def test_two_gloo_ranks_max_time_and_rank0_only():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        w, t, rate, ref = res[r]
        assert w == world
        assert t == 2.0                 # max over ranks
        assert rate == world * 10.0 * 4 / 2.0
    assert res[1][3] is None            # the reference arm prints on rank 0 only


def test_single_process_needs_no_group():
    bench = _bench()
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    d = bench.Dist()
    assert d.world == 1 and d.pg is None and d.max(3.5) == 3.5
    d.close()


def _owned_tile_products(rank, world, port, out):
    """A distributed product's host logic on CPU: every gloo rank takes its
    block-cyclic C tiles (the reference's ownership), computes them with the
    oracle (standing in for the device kernels), and rank 0 gathers the
    sub-grids and assembles the whole matrix."""
    import numpy as np
    import torch.distributed as tdist
    from bcl_b200 import gen
    from bcl_b200.containers import assemble_tiles, owned_tiles, process_grid
    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        a = gen.rmat(9, seed=23)
        tm = tk = tn = 100
        gm = gn = -(-a.m // tm)
        pm, pn = process_grid(world)
        rows, cols = owned_tiles(gm, gn, rank, pm, pn)
        # the owned tiles of the oracle's whole product, packed as the device sub-grid would be
        rp, ci, cv = O.gemm_tiled(a, a, tm, tk, tn)
        trp, toff, cis, vs = [], [0], [], []
        for i in rows:
            for j in cols:
                r0, r1 = i * tm, min((i + 1) * tm, a.m)
                loc = [0]
                for r in range(r0, r1):
                    seg = slice(rp[r], rp[r + 1])
                    sel = (ci[seg] >= j * tn) & (ci[seg] < (j + 1) * tn)
                    cis.append(ci[seg][sel] - j * tn)
                    vs.append(cv[seg][sel])
                    loc.append(loc[-1] + int(sel.sum()))
                loc += [loc[-1]] * (tm + 1 - len(loc))
                trp.append(loc)
                toff.append(toff[-1] + loc[-1])
        part = (rows, cols, np.asarray(trp, np.int32), np.asarray(toff, np.int64),
                np.concatenate(cis) if cis else np.zeros(0, np.int32),
                np.concatenate(vs) if vs else np.zeros(0, np.float32))
        gathered = [None] * world if rank == 0 else None
        tdist.gather_object(part, gathered, dst=0)
        if rank == 0:
            whole = assemble_tiles(a.m, a.m, tm, tn, gathered)
            out["ok"] = (np.array_equal(whole.row_ptr.astype(np.int64), rp) and np.array_equal(whole.col_ind, ci)
                         and np.array_equal(whole.vals.view(np.uint32), cv.view(np.uint32)))
            out["tiles"] = sum(len(p[0]) * len(p[1]) for p in gathered)
    finally:
        tdist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_block_cyclic_ownership_covers_and_gathers(world):
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_owned_tile_products, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res["ok"] and res["tiles"] == 6 * 6


def test_ownership_matches_the_reference_formula():
    from bcl_b200.containers import owned_tiles, process_grid
    for world in (1, 2, 3, 4, 6, 8):
        pm, pn = process_grid(world)
        assert pm * pn == world and pm <= pn
        seen = {}
        for p in range(world):
            rows, cols = owned_tiles(7, 9, p, pm, pn)
            for i in rows:
                for j in cols:
                    assert (j % pn) + (i % pm) * pn == p    # SPMatrix.hpp:230-237
                    seen[(i, j)] = p
        assert len(seen) == 7 * 9
