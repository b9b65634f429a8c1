"""bench.py's reference arm on CPU: the sample rows dealt to one process per
core cover the sample exactly once, and the reference line keeps the JSON
contract (impl, cpu_baseline, e2e with no copies).  Needs the reference
binary built from the reference headers (oracle/_ref/bcl_ref)."""
import importlib.util
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_ref_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_split_rows_deals_every_row_once():
    from bcl_b200 import gen
    bench = _bench()
    a = gen.rmat(9, seed=5)
    s = bench.row_sample(a, 3)
    parts = bench.split_rows(s, 4)
    assert len(parts) == 4
    assert sum(p.m for p in parts) == s.m and sum(p.nnz for p in parts) == s.nnz
    for p, part in enumerate(parts):
        rows = np.arange(p, s.m, 4)
        for i, r in enumerate(rows[:20]):
            lo, hi = s.row_ptr[r], s.row_ptr[r + 1]
            plo, phi = part.row_ptr[i], part.row_ptr[i + 1]
            assert np.array_equal(part.col_ind[plo:phi], s.col_ind[lo:hi])
            assert np.array_equal(part.vals[plo:phi], s.vals[lo:hi])


def test_reference_arm_line():
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("the reference binary oracle/_ref/bcl_ref is not built")
    bench = _bench()

    class Args:
        workload, seed, steps, warmup, gpus = "spmm_er16k", 1, 1, 0, 1

    class OneRank:
        rank, world = 0, 1

    line = bench.run_reference(Args, OneRank)
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["value"] == line["value"]
    assert line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": "GFLOP/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["higher_is_better"] is True and line["gpu_launches"] == 0
