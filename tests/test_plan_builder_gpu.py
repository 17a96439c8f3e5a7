"""Plans lowered from RA by the builder, run by the executor on the GPU: the benchmark
queries give the oracle's results, and the paths the benchmark plans do not take
(projection + sort before an aggregation, unsorted set-operation inputs, unique, merge)
give what a numpy restatement of the RA gives."""
import numpy as np
import pytest
import torch

import oracle as O
from redfox_b200 import executor as X
from redfox_b200 import plan_builder as PB
from redfox_b200 import plans as PL
from redfox_b200 import rfx as R

from helpers import join_aggregate_oracle, join_aggregate_oracle_data, to_np

pytestmark = pytest.mark.gpu


def _run(builder, inputs):
    ex = X.Executor(builder.json())
    for name, t in inputs.items():
        ex.bind(name, t)
    ex.run()
    return ex


@pytest.mark.parametrize("nr,ns,dom", [(1000, 4000, 256), (50000, 200000, 12500)])
def test_join_aggregate_from_ra(cuda, nr, ns, dom):
    r, s = PL.gen_join_aggregate(nr, ns, key_domain=dom)
    ex = _run(PB.join_aggregate_ra(), {"R": r.clone(), "S": s.clone()})
    t = to_np(ex.output("T")).view(np.uint64).reshape(-1, 2)     # key << 64 | sum
    c = to_np(ex.output("C")).view(np.uint64).ravel()            # key << 32 | count
    ex.close()
    ek, esum, ecnt, _ = join_aggregate_oracle(*join_aggregate_oracle_data(nr, ns, dom))
    assert np.array_equal(t[:, 1].astype(np.uint32), ek) and np.array_equal(t[:, 0].view(np.int64), esum)
    assert np.array_equal((c >> np.uint64(32)).astype(np.uint32), ek)
    assert np.array_equal((c & np.uint64(0xFFFFFFFF)).astype(np.uint32), ecnt)


def test_three_relation_from_ra(cuda):
    n1, n2, n3, l5, l2 = (PL.C2_D1_ROWS // 100, PL.C2_D2_ROWS // 100, PL.C2_F_ROWS // 100, PL.C2_L5 // 100,
                          PL.C2_L2 // 100)
    d1, d2, f, li, lo = PL.gen_three_relation(n1, n2, n3, l5, l2)
    ek, es, ec = PL.three_relation(d1, d2, f, li, lo)
    ex = _run(PB.three_relation_ra(PL.C2_SEGMENT, PL.C2_DATE_LO, PL.C2_DATE_HI),
              {"D1": d1, "D2": d2, "F": f.clone(), "Lin": li, "Lout": lo})
    t = to_np(ex.output("T")).view(np.uint64).reshape(-1, 2)
    c = to_np(ex.output("C")).view(np.uint64).ravel()
    ex.close()
    assert np.array_equal(t[:, 1].astype(np.uint32), to_np(ek).view(np.uint32))
    assert np.array_equal(t[:, 0].view(np.int64), to_np(es))
    assert np.array_equal((c & np.uint64(0xFFFFFFFF)).astype(np.uint32), to_np(ec).view(np.uint32))


def test_aggregation_over_non_leading_fields(cuda):
    """A(x:16, y:16, v:32): SUM(v) by y and COUNT by (y, x) -- projection, sort, reduce, merge."""
    n = 200_000
    rng = np.random.default_rng(3)
    x = rng.integers(0, 50, n, dtype=np.uint64)
    y = rng.integers(0, 300, n, dtype=np.uint64)
    v = rng.integers(0, 2**32, n, dtype=np.uint64)
    a = O.pack([16, 16, 32], [x, y, v])
    b = PB.PlanBuilder().relation("A", [16, 16, 32])
    b.agg("T", "A", [1], PB.AGG_TOTAL, 2).agg("C", "A", [1, 0], PB.AGG_COUNT).output("T", "C")
    ex = _run(b, {"A": torch.from_numpy(a).to(cuda)})
    t = to_np(ex.output("T")).view(np.uint64).reshape(-1, 2)    # (y:16, sum:64) in 16 B
    c = to_np(ex.output("C")).view(np.uint64).ravel()           # (y:16, x:16, count:32)
    ex.close()
    ys = np.unique(y)
    sums = np.array([v[y == k].sum() for k in ys], np.uint64)
    assert np.array_equal(t[:, 1], ys) and np.array_equal(t[:, 0], sums)
    pairs, counts = np.unique(np.stack([y, x], 1), axis=0, return_counts=True)
    assert np.array_equal(c >> np.uint64(48), pairs[:, 0])
    assert np.array_equal((c >> np.uint64(32)) & np.uint64(0xFFFF), pairs[:, 1])
    assert np.array_equal(c & np.uint64(0xFFFFFFFF), counts.astype(np.uint64))


def test_set_operations_on_unsorted_inputs(cuda):
    rng = np.random.default_rng(4)
    a = rng.integers(0, 5000, 20000).astype(np.uint32)
    bb = rng.integers(0, 5000, 8000).astype(np.uint32)
    b = PB.PlanBuilder().relation("A", [32]).relation("B", [32])
    b.set_op("U", "A", "B", R.SET_UNION).unique("U")
    b.set_op("D", "A", "B", R.SET_DIFFERENCE)
    b.output("U", "D")
    ex = _run(b, {"A": torch.from_numpy(a.view(np.int32).copy()).to(cuda),
                  "B": torch.from_numpy(bb.view(np.int32).copy()).to(cuda)})
    u = to_np(ex.output("U")).view(np.uint32).ravel()
    d = to_np(ex.output("D")).view(np.uint32).ravel()
    ex.close()
    sa, sb = np.sort(a), np.sort(bb)
    assert np.array_equal(u, O.unique(O.set_union(sa, sb)))
    assert np.array_equal(d, O.set_difference(sa, sb))
