"""The batched form: many join + aggregate queries folded into one plan (query id below the
key, queries in order) give, per query, exactly the plain per-query plan's result and the
oracle's, eagerly and through CUDA graph replay."""
import numpy as np
import pytest

from redfox_b200 import batch as B

from helpers import join_aggregate_oracle, to_np


def test_query_sizes_are_deterministic_and_in_range():
    a = B.query_sizes(64, 1000, 50_000, seed=7)
    assert a == B.query_sizes(64, 1000, 50_000, seed=7)
    assert all(1000 <= x <= 50_000 for q in a for x in q)
    full = B.query_sizes()
    assert len(full) == B.C3_QUERIES
    # the per-query key domain |R|/4 must fit the key bits, the query ids the query bits,
    # and both the 32-bit key field
    assert max(r for r, _ in full) // 4 <= 1 << B.KEY_BITS
    assert B.C3_QUERIES - 1 <= B.QUERY_MASK
    assert B.QUERY_BITS + B.KEY_BITS <= 32
    assert B.unfold(B.fold(12345, 67)) == (12345, 67)


def _per_query(r_all, s_all, r_off, s_off, q):
    keys, sums, counts, total = B.plain_query(r_all, s_all, r_off, s_off, q)
    return B.unfold(keys)[0], sums, counts, total


@pytest.mark.gpu
def test_batched_equals_plain_and_oracle(cuda):
    sizes = B.query_sizes(16, 1000, 50_000, seed=11)
    r_all, s_all, r_off, s_off = B.gen_batch(sizes)
    plan = B.BatchedPlan(r_all, s_all)
    plan.run()
    keys, sums, counts, total = plan.result()
    per = B.split_by_query(keys, sums, counts, len(sizes))
    totals = 0
    for q in range(len(sizes)):
        pk, ps, pc, pt = _per_query(r_all, s_all, r_off, s_off, q)
        totals += pt
        bk, bs, bc = per[q]
        assert np.array_equal(to_np(bk), to_np(pk)), q
        assert np.array_equal(to_np(bs), to_np(ps)), q
        assert np.array_equal(to_np(bc), to_np(pc)), q
        if q < 3:
            ek, es, ec, et = join_aggregate_oracle(to_np(r_all[r_off[q]:r_off[q + 1]]),
                                                   to_np(s_all[s_off[q]:s_off[q + 1]]))
            assert et == pt
            assert np.array_equal(to_np(bk).view(np.uint32), ek >> np.uint32(B.QUERY_BITS))
            assert np.array_equal(to_np(bs), es)
            assert np.array_equal(to_np(bc).view(np.uint32), ec)
    assert totals == total


@pytest.mark.gpu
def test_graph_replay_reproduces_eager(cuda):
    import torch
    sizes = B.query_sizes(24, 1000, 20_000, seed=12)
    r_all, s_all, _, _ = B.gen_batch(sizes)
    plan = B.BatchedPlan(r_all, s_all)
    plan.run()
    k0, s0, c0, t0 = [x.clone() if torch.is_tensor(x) else x for x in plan.result()]
    plan.capture()
    for _ in range(3):
        plan.keys.zero_()
        plan.sums.zero_()
        plan.replay()
        k1, s1, c1, t1 = plan.result()
        assert t1 == t0
        assert torch.equal(k1, k0) and torch.equal(s1, s0) and torch.equal(c1, c0)


def test_split_by_query_on_host_tensors():
    """Groups ordered by (key, query) -- what the stable sort on the key bits leaves -- split
    into per-query groups in key order, the query bits removed (host tensors, no GPU)."""
    import torch
    pairs = sorted([(k, q) for k in (3, 9, 1 << 20, (1 << 21) - 1) for q in (0, 2, 5)])
    keys = torch.tensor([B.fold(k, q) for k, q in pairs], dtype=torch.int64).to(torch.int32)
    sums = torch.arange(len(pairs), dtype=torch.int64)
    counts = torch.arange(len(pairs), dtype=torch.int32) + 1
    per = B.split_by_query(keys, sums, counts, 6)
    for q in range(6):
        k, s, c = per[q]
        want = [i for i, (_, qq) in enumerate(pairs) if qq == q]
        assert k.tolist() == [pairs[i][0] for i in want]
        assert s.tolist() == want and c.tolist() == [i + 1 for i in want]
