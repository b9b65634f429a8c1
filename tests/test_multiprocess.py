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
