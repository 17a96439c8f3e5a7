"""Select / arith / project / filter-aggregate kernels against the oracle (bit-exact)."""
import numpy as np
import pytest

import oracle as O
from redfox_b200 import rfx as R
from redfox_b200 import workloads as WL

from helpers import fact_oracle, fact_rows_oracle, oracle_arith, oracle_cmps, to_np

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True, params=["jit", "interp"])
def kernel_path(request, monkeypatch):
    """Every case runs on the plan-specialised (runtime-compiled) kernels and on the
    interpreting kernels (RFX_JIT=0)."""
    if request.param == "interp":
        monkeypatch.setenv("RFX_JIT", "0")
    else:
        monkeypatch.delenv("RFX_JIT", raising=False)
    return request.param


def _rows_to_dev(rows, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(rows)).to(cuda)


@pytest.mark.parametrize("n", [1, 1000, 262144 + 17])
def test_generator_matches_oracle(cuda, n):
    dev = WL.gen_fact(n)
    assert np.array_equal(to_np(dev), fact_rows_oracle(n))
    assert R.device_status() == R.OK


SHAPES = [
    ([8], [(R.LT, (R.OPND_VAR, 0), (R.OPND_CONST, 100), R.I8)]),
    ([3, 13], [(R.GE, (R.OPND_VAR, 1), (R.OPND_CONST, 4000), R.I16)]),
    ([32], [(R.NE, (R.OPND_VAR, 0), (R.OPND_CONST, 7), R.I32)]),
    ([32, 32], [(R.LE, (R.OPND_VAR, 0), (R.OPND_CONST, 2**31), R.I32),
                (R.GT, (R.OPND_VAR, 1), (R.OPND_VAR, 0), R.I32)]),
    ([32, 64], [(R.EQ, (R.OPND_VAR, 0), (R.OPND_CONST, 5), R.I32)]),
    ([7, 33, 64, 40, 21], [(R.SGT, (R.OPND_CONST, 2**39), (R.OPND_VAR, 3), R.I64)]),
    (WL.FACT_WIDTHS, [(R.LE, (R.OPND_VAR, 0), (R.OPND_CONST, 2475), R.I32)]),
]


def _random_rows(widths, n, seed, small=False):
    rng = np.random.default_rng(seed)
    cols = []
    for w in widths:
        hi = min(2**w, 2**63) if not small else min(2**w, 16)
        c = rng.integers(0, hi, n, dtype=np.uint64) if hi < 2**63 else rng.integers(0, 2**63, n, dtype=np.uint64) * np.uint64(2)
        cols.append(c)
    return O.pack(widths, cols)


@pytest.mark.parametrize("shape", range(len(SHAPES)))
@pytest.mark.parametrize("n", [0, 1, 31, 33, 511, 512, 513, 100003])
def test_select_matches_oracle(cuda, shape, n):
    widths, cmps = SHAPES[shape]
    rows = _random_rows(widths, n, seed=shape * 1000 + n, small=(shape == 3))
    got, k = R.select(_rows_to_dev(rows, cuda), widths, cmps)
    exp = O.select(rows, widths, oracle_cmps(cmps))
    assert k == len(exp)
    assert np.array_equal(to_np(got), exp)
    assert R.device_status() == R.OK


def _arith_cases():
    # (widths, expr) -- C integer semantics incl. 32-bit wrap, signed int promotion, div/mod
    return [
        ([32, 32], R.make_arith([(R.NODE_OP, R.MUL, 0, 1, 2, 0), (R.NODE_INDEX, 0, R.I32, -1, -1, 0),
                                 (R.NODE_INDEX, 0, R.I32, -1, -1, 1)], 0, R.I32, 32)),
        ([8, 16], R.make_arith([(R.NODE_OP, R.SUB, 0, 1, 2, 0), (R.NODE_INDEX, 0, R.I8, -1, -1, 0),
                                (R.NODE_INDEX, 0, R.I16, -1, -1, 1)], 0, R.I64, 40)),
        ([16, 16], R.make_arith([(R.NODE_OP, R.DIV, 0, 1, 2, 0),
                                 (R.NODE_OP, R.SUB, 0, 3, 4, 0), (R.NODE_INDEX, 0, R.I16, -1, -1, 1),
                                 (R.NODE_INDEX, 0, R.I16, -1, -1, 0), (R.NODE_CONST, 0, R.I32, -1, -1, 30000)],
                                0, R.I32, 32)),
        ([32, 64], R.make_arith([(R.NODE_OP, R.MOD, 0, 1, 2, 0), (R.NODE_INDEX, 0, R.I64, -1, -1, 1),
                                 (R.NODE_INDEX, 0, R.I32, -1, -1, 0)], 0, R.I64, 64)),
        ([32, 64], R.make_arith([(R.NODE_OP, R.ADD, 0, 1, 2, 0), (R.NODE_INDEX, 0, R.I32, -1, -1, 0),
                                 (R.NODE_CONST, 0, R.I64, -1, -1, 2**63 + 5)], 0, R.I64, 64)),
        (WL.FACT_WIDTHS, WL.fact_ariths()[1]),
    ]


@pytest.mark.parametrize("case", range(6))
@pytest.mark.parametrize("n", [1, 513, 70001])
def test_arith_matches_oracle(cuda, case, n):
    widths, expr = _arith_cases()[case]
    rows = _random_rows(widths, n, seed=case * 77 + n)
    got = R.arith(_rows_to_dev(rows, cuda), widths, expr)
    exp = O.arith(rows, widths, oracle_arith(expr))
    assert np.array_equal(to_np(got), exp)


@pytest.mark.parametrize("n", [1, 1000, 65537])
def test_project_matches_oracle(cuda, n):
    rows = fact_rows_oracle(n)
    for out_w, fmap in (([8, 8, 64], [5, 6, 2]), ([32], [0]), ([64, 32, 8], [1, 0, 100]), ([8, 8], [6, 5])):
        got = R.project(_rows_to_dev(rows, cuda), WL.FACT_WIDTHS, out_w, fmap)
        exp = O.project(rows, WL.FACT_WIDTHS, out_w, fmap)
        assert np.array_equal(to_np(got), exp), (out_w, fmap)


@pytest.mark.parametrize("n", [0, 5, 1023, 200001])
def test_select_project_matches_composition(cuda, n):
    """select -> arith -> arith -> project in one kernel == the reference's op sequence."""
    rows = fact_rows_oracle(n)
    cmps = WL.fact_predicate()
    ariths = WL.fact_ariths()
    out_w, fmap = [8, 8, 64, 64], [5, 6, 7, 8]
    got, k = R.select_project(_rows_to_dev(rows, cuda), WL.FACT_WIDTHS, cmps, ariths, out_w, fmap)
    sel = O.select(rows, WL.FACT_WIDTHS, oracle_cmps(cmps))
    a1 = O.arith(sel, WL.FACT_WIDTHS, oracle_arith(ariths[0]))
    a2 = O.arith(a1, WL.FACT_WIDTHS + [64], oracle_arith(ariths[1]))
    exp = O.project(a2, WL.FACT_WIDTHS + [64, 64], out_w, fmap)
    assert k == len(exp)
    assert np.array_equal(to_np(got), exp)


@pytest.mark.parametrize("n", [0, 1, 4097, 1_000_003])
def test_fact_filter_aggregate_matches_oracle(cuda, n):
    dev = WL.gen_fact(n)
    plan = WL.fact_plan(n)
    plan.launch(dev)
    keys, sums, counts = plan.result()
    assert R.device_status() == R.OK
    if n == 0:
        assert len(keys) == 0
        return
    ek, es, ec = fact_oracle(to_np(dev))
    assert np.array_equal(keys, ek) and np.array_equal(sums, es) and np.array_equal(counts, ec)


def test_filter_aggregate_repeatable(cuda):
    n = 300_000
    dev = WL.gen_fact(n)
    plan = WL.fact_plan(n)
    plan.launch(dev)
    first = plan.result()
    plan.launch(dev)
    second = plan.result()
    for a, b in zip(first, second):
        assert np.array_equal(a, b)


def test_filter_aggregate_shared_table_path(cuda):
    """A larger group domain takes the shared-atomic table instead of private slots."""
    n = 200_000
    rows = _random_rows([8, 8, 32], n, seed=5, small=True)
    cmps = [(R.GE, (R.OPND_VAR, 2), (R.OPND_CONST, 3), R.I32)]
    keys, sums, counts = R.filter_aggregate(_rows_to_dev(rows, cuda), [8, 8, 32], cmps, [], [0, 1], [16, 16], [2])
    ek, es, ec = O.filter_aggregate(rows, [8, 8, 32], oracle_cmps(cmps), [], [0, 1], [2])
    assert np.array_equal(keys, ek) and np.array_equal(sums, es) and np.array_equal(counts, ec)


def test_filter_aggregate_domain_violation_reported(cuda):
    rows = _random_rows([8, 8], 1000, seed=9, small=True)   # values up to 15
    R.filter_aggregate(_rows_to_dev(rows, cuda), [8, 8], [], [], [0], [4], [1])
    assert R.device_status() == R.ERR_CAPACITY
    assert R.device_status() == R.OK   # the word is cleared by the read
