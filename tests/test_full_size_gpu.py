"""Bit-exact parity at the workloads' full sizes: every benchmark plan run on the GPU over
its full seeded inputs equals the oracle's restatement of the same plan over the same
inputs -- keys, order, sums, counts and join totals -- as the reference's own full-run
checks compare device results against the CPU join (moderngpu tests/benchmarkjoin.cu:166-190,
ra/test/TestJoin.cu:107-156).

* filter-project-aggregate: 60M rows of Tuple<32,64,64,64,64,8,8>, 6 groups;
* join + aggregate: R 1M x S 4M, ~19.3M join rows, ~2.6e5 groups;
* three-relation pipeline: D1 1.5M, D2 15M (Zipf(1) foreign keys), F 60M, lists 5M / 2M;
* batched form: 64 queries of the batched workload's size law (log-uniform 1e4..8e6 rows).

The inputs are generated on the device and checked byte for byte against the oracle's
generator first, so the oracle computes on exactly what the kernels saw.
"""
import numpy as np
import pytest

import oracle as O
from redfox_b200 import batch as B
from redfox_b200 import plans as PL
from redfox_b200 import workloads as WL

from helpers import (fact_oracle, fact_rows_oracle, join_aggregate_oracle, join_aggregate_oracle_data,
                     three_relation_oracle, three_relation_oracle_data, to_np)

pytestmark = pytest.mark.gpu


def test_filter_aggregate_60M_rows_bit_exact(cuda):
    n = WL.FACT_ROWS
    rows = WL.gen_fact(n)
    plan = WL.fact_plan(n)
    plan.launch(rows)
    keys, sums, counts = plan.result()
    host = to_np(rows)
    del rows
    assert np.array_equal(host, fact_rows_oracle(n))
    ek, es, ec = fact_oracle(host)
    assert len(ek) == 6
    assert np.array_equal(keys, ek) and np.array_equal(sums, es) and np.array_equal(counts, ec)


def test_join_aggregate_1M_x_4M_bit_exact(cuda):
    r, s = PL.gen_join_aggregate()
    er, es = join_aggregate_oracle_data(PL.C0_R_ROWS, PL.C0_S_ROWS, PL.C0_KEY_DOMAIN)
    assert np.array_equal(to_np(r), er) and np.array_equal(to_np(s), es)
    keys, sums, counts, total = PL.join_aggregate(r, s)
    ek, esum, ecnt, etot = join_aggregate_oracle(er, es)
    assert 15_000_000 < etot < 25_000_000
    assert total == etot
    assert np.array_equal(to_np(keys).view(np.uint32), ek)
    assert np.array_equal(to_np(sums), esum)
    assert np.array_equal(to_np(counts).view(np.uint32), ecnt)


def test_three_relation_full_size_bit_exact(cuda):
    d1, d2, f, li, lo = PL.gen_three_relation()
    ed1, ed2, ef, eli, elo = three_relation_oracle_data(PL.C2_D1_ROWS, PL.C2_D2_ROWS, PL.C2_F_ROWS, PL.C2_L5,
                                                        PL.C2_L2)
    assert np.array_equal(to_np(d1), ed1) and np.array_equal(to_np(d2), ed2)
    assert np.array_equal(to_np(f), ef)
    assert np.array_equal(to_np(li).view(np.uint32), eli) and np.array_equal(to_np(lo).view(np.uint32), elo)
    keys, sums, counts = PL.three_relation(d1, d2, f, li, lo)
    del d1, d2, f
    ek, es, ec = three_relation_oracle(ed1, ed2, ef, eli, elo)
    assert len(ek) > 1000
    assert np.array_equal(to_np(keys).view(np.uint32), ek)
    assert np.array_equal(to_np(sums), es)
    assert np.array_equal(to_np(counts).view(np.uint32), ec)


def test_batched_64_queries_full_size_law_bit_exact(cuda):
    """64 queries drawn by the batched workload's own size law: the batched plan's groups per
    query equal the oracle's plan over that query alone."""
    sizes = B.query_sizes(64)
    r_all, s_all, r_off, s_off = B.gen_batch(sizes)
    plan = B.BatchedPlan(r_all, s_all)
    plan.run()
    keys, sums, counts, total = plan.result()
    per = B.split_by_query(keys, sums, counts, len(sizes))
    hr, hs = to_np(r_all), to_np(s_all)
    etotal = 0
    for q in range(len(sizes)):
        ek, es, ec, et = join_aggregate_oracle(hr[r_off[q]:r_off[q + 1]], hs[s_off[q]:s_off[q + 1]])
        etotal += et
        bk, bs, bc = per[q]
        assert np.array_equal(to_np(bk).view(np.uint32), ek >> np.uint32(B.QUERY_BITS)), q
        assert np.array_equal(to_np(bs), es), q
        assert np.array_equal(to_np(bc).view(np.uint32), ec), q
    assert total == etotal


def test_oracle_generator_matches_for_batched_inputs(cuda):
    """The batched inputs of a few queries equal the oracle generator's (the same SplitMix64
    streams), so the batched parity above compares like with like."""
    sizes = B.query_sizes(3, 1000, 20_000, seed=5)
    r_all, s_all, r_off, s_off = B.gen_batch(sizes)
    hr = to_np(r_all).view(np.uint64).ravel()
    for q, (nr, ns) in enumerate(sizes):
        dom = max(1, nr // 4)
        key = O.uniform(nr, B.C3_SEED + 16 + 2 * q, 0, 0, dom)
        pay = O.uniform(nr, B.C3_SEED + 16 + 2 * q, 1, 0, 1 << 32)
        exp = (((key << np.uint64(B.QUERY_BITS)) | np.uint64(q)) << np.uint64(32)) | pay
        assert np.array_equal(hr[r_off[q]:r_off[q + 1]], exp)
