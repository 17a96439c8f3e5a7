"""The autotuner: with tuning on, the first call per (operator, shape, size class) times
every variant and later calls run the fastest; every variant gives the same results."""
import numpy as np
import pytest

from redfox_b200 import plans as PL
from redfox_b200 import rfx as R
from redfox_b200 import workloads as WL

from helpers import to_np


def test_tune_table_without_gpu_work():
    R.tune(0)
    R.tune_reset()
    assert R.tune_table() == []


@pytest.mark.gpu
def test_tuned_operators_give_default_results(cuda):
    import torch
    rows = R.gen_uniform_rows(300_000, WL.FACT_WIDTHS, 7, WL.FACT_LO, WL.FACT_HI, device=cuda)
    r, s = PL.gen_join_aggregate(20_000, 80_000, key_domain=5000)
    R.sort_pairs(r, begin_bit=32, end_bit=64)
    R.sort_pairs(s, begin_bit=64, end_bit=96)
    jout, total = R.join_tuples_two_step(r, 32, s, 64, 16)
    a = R.gen_uniform_rows(400_000, [32], 11, [0], [1 << 22], device=cuda).view(torch.int32).view(-1).clone()
    b = R.gen_uniform_rows(150_000, [32], 12, [0], [1 << 22], device=cuda).view(torch.int32).view(-1).clone()
    R.sort_pairs(a)
    R.sort_pairs(b)

    def run_all():
        sel, _ = R.select(rows, WL.FACT_WIDTHS, WL.fact_predicate())
        red = R.reduce_tuples(jout, 96, 0, 64, 4, n=total)
        sets = [R.set_op(op, a, b) for op in (R.SET_INTERSECTION, R.SET_DIFFERENCE, R.SET_UNION)]
        return [to_np(sel)] + [to_np(x) for x in red[:3]] + [to_np(x) for x in sets]

    R.tune(0)
    R.tune_reset()
    base = run_all()
    try:
        R.tune(1)
        first = run_all()      # tunes every class
        table = R.tune_table()
        second = run_all()     # uses the decisions
    finally:
        R.tune(0)
        R.tune_reset()
    ops = {e["op"] for e in table}
    assert {"select_compact", "reduce_tuples", "set_filter"} <= ops
    for e in table:
        assert 0 <= e["variant"] < len(e["ms"])
        assert e["ms"][e["variant"]] == min(m for m in e["ms"] if m >= 0)
    for x, y, z in zip(base, first, second):
        assert np.array_equal(x, y) and np.array_equal(x, z)
    assert R.device_status() == R.OK
