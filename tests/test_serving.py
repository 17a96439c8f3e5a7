"""Admission logic of the serving loop on a virtual clock (no GPU): FIFO order, slot and
byte-budget limits, oversize queries running alone, and the effect of concurrency on
latency under Poisson arrivals."""
import math

import numpy as np

from redfox_b200 import serving as S

from helpers import three_relation_oracle_data


def _q(qid, arrival, est):
    q = S.Query(qid, arrival, 0, 0, 100, 0)
    q.est_bytes = est
    return q


def test_requests_are_seeded_and_in_range():
    a = S.gen_requests(200, 1000.0, seed=5)
    b = S.gen_requests(200, 1000.0, seed=5)
    assert [(q.arrival, q.segment, q.date_lo, q.date_hi, q.list_size) for q in a] == \
        [(q.arrival, q.segment, q.date_lo, q.date_hi, q.list_size) for q in b]
    assert all(a[i].arrival < a[i + 1].arrival for i in range(len(a) - 1))
    for q in a:
        assert S.WIDTH_MIN <= q.date_hi - q.date_lo <= S.WIDTH_MAX
        assert 0 <= q.date_lo and q.date_hi <= S.DATE_DAYS
        assert 0 <= q.segment <= 4
        assert q.list_size == 0 or S.LIST_MIN <= q.list_size <= S.LIST_MAX
        assert q.est_bytes > 0
    # mean inter-arrival ~ 1 / rate
    assert 0.5e-3 < a[-1].arrival / len(a) < 2e-3
    assert 0.3 < sum(q.list_size > 0 for q in a) / len(a) < 0.7


def test_fifo_slots_and_budget():
    sch = S.Scheduler(slots=2, budget_bytes=100)
    for i, est in enumerate([40, 40, 10, 70]):
        sch.arrive(_q(i, 0.0, est))
    first = sch.admissions()
    assert [q.qid for q, _ in first] == [0, 1]          # two slots
    assert sorted(s for _, s in first) == [0, 1]
    sch.complete(first[0][0])
    nxt = sch.admissions()
    assert [q.qid for q, _ in nxt] == [2]               # 40 + 10 within 100
    assert sch.admissions() == []                       # 50 + 70 exceeds the budget: head waits
    sch.complete(first[1][0])
    assert [q.qid for q, _ in sch.admissions()] == [3]  # 10 + 70 fits
    assert sch.inflight_bytes == 80 and sch.peak_queries == 2


def test_budget_blocks_head_and_oversize_runs_alone():
    sch = S.Scheduler(slots=4, budget_bytes=100)
    big = _q(0, 0.0, 250)
    sch.arrive(big)
    assert [q.qid for q, _ in sch.admissions()] == [0]  # larger than the budget: alone
    sch.arrive(_q(1, 0.0, 5))
    assert sch.admissions() == []                       # nothing joins an oversize query
    sch.complete(big)
    assert [q.qid for q, _ in sch.admissions()] == [1]
    assert sch.peak_bytes == 250


def test_simulated_latency_improves_with_slots():
    reqs = S.gen_requests(400, 2000.0, seed=9)
    service = lambda q, k: 1e-3 * (1 + 0.2 * (k - 1))   # mild slowdown when sharing the GPU
    one = [S.Query(q.qid, q.arrival, q.segment, q.date_lo, q.date_hi, q.list_size) for q in reqs]
    for a, b in zip(one, reqs):
        a.est_bytes = b.est_bytes
    S.simulate(one, service, slots=1)
    sch = S.simulate(reqs, service, slots=8)
    s1 = S.latency_summary(one)
    s8 = S.latency_summary(reqs)
    assert all(not math.isnan(q.done) for q in reqs + one)
    assert all(q.start >= q.arrival for q in reqs)
    assert s8["latency_ms_p99"] < s1["latency_ms_p99"]
    assert s8["queries_per_s"] > s1["queries_per_s"]
    assert sch.peak_queries <= 8 and sch.peak_bytes <= S.BUDGET_BYTES


def test_simulated_budget_limits_concurrency():
    reqs = [_q(i, 0.0, 30) for i in range(20)]
    sch = S.simulate(reqs, lambda q, k: 1.0, slots=8, budget_bytes=100)
    assert sch.peak_queries == 3 and sch.peak_bytes <= 100
    # FIFO: start times are non-decreasing in arrival (qid) order
    starts = [q.start for q in reqs]
    assert starts == sorted(starts)


def _multi_select_np(rows, field, bounds, key, val):
    """numpy restatement of rfx_multi_select: per row in order, per query in order, emit
    ((key << 8 | q) << val_width) | val when lo_q <= field < hi_q."""
    W = rows.shape[1]
    limbs = rows.view(np.uint64) if W >= 8 else rows.view(np.uint32).astype(np.uint64)
    if W == 16:
        as_int = [int(lo) | (int(hi) << 64) for lo, hi in limbs]
    else:
        as_int = [int(x) for x in limbs.ravel()]

    def bits(x, sw):
        return (x >> sw[0]) & ((1 << sw[1]) - 1)
    out = []
    for x in as_int:
        f = bits(x, field)
        for q, (lo, hi) in enumerate(bounds):
            if lo <= f < hi:
                out.append((((bits(x, key) << 8) | q) << val[1]) | bits(x, val))
    return np.array(out, dtype=np.uint64)


def test_round_plan_layout_on_oracle():
    """The batched round's bit layout (query id in the low 8 bits of every key) run with
    the oracle's operators gives every query exactly the per-query oracle plan's groups."""
    import oracle as O
    from redfox_b200 import serving as S

    from helpers import serving_query_oracle
    n1, n2, n3 = 3000, 30000, 120000
    d1, d2, f, _, _ = three_relation_oracle_data(n1, n2, n3, 10, 10)
    fs = O.sort_pairs(f, begin_bit=64, end_bit=96)
    reqs = S.gen_requests(12, 1e6, seed=5, n2=n2)
    lists = {}
    for q in reqs:
        if q.list_size:
            raw = O.uniform(q.list_size, q.list_seed, 0, 0, n2).astype(np.uint32)
            lists[q.qid] = O.unique(O.sort_pairs(raw))
    for group in ([q for q in reqs if q.list_size], [q for q in reqs if not q.list_size]):
        d1m = _multi_select_np(d1, (0, 8), [(q.segment, q.segment + 1) for q in group], (8, 32), (0, 8))
        d2m = _multi_select_np(d2, (0, 32), [(q.date_lo, q.date_hi) for q in group], (32, 24), (64, 32))
        d2m = O.sort_pairs(d2m.view(np.uint8).reshape(-1, 8), begin_bit=32, end_bit=64)
        j1 = O.join_tuples(d1m.view(np.uint8).reshape(-1, 8), 8, d2m, 32, 16)
        keys = O.project(j1, [32, 8, 8, 32], [32, 8], [3, 1])
        keys = O.sort_pairs(keys, begin_bit=0, end_bit=40)
        if group and group[0].list_size:
            folded = np.concatenate([(lists[q.qid].astype(np.uint64) << np.uint64(8)) | np.uint64(i)
                                     for i, q in enumerate(group)])
            folded = O.sort_pairs(folded, begin_bit=0, end_bit=40)
            keys = O.set_intersection(keys.view(np.uint64).ravel(), folded).view(np.uint8).reshape(-1, 8)
        j2 = O.join_tuples(keys, 8, fs, 64, 16)
        limbs = j2.view(np.uint64)
        gkey = limbs[:, 1]                              # (pk2 << 8 | q): bits 64..103
        amt = limbs[:, 0].astype(np.int64)
        k, sums = O.reduce_sum_i64(gkey, amt)
        _, counts = O.reduce_count(gkey)
        for i, q in enumerate(group):
            sel = (k & np.uint64(0xFF)) == np.uint64(i)
            ek, es, ec = serving_query_oracle(d1, d2, fs, q.segment, q.date_lo, q.date_hi, lists.get(q.qid))
            assert np.array_equal((k[sel] >> np.uint64(8)).astype(np.uint32), ek), q
            assert np.array_equal(sums[sel], es) and np.array_equal(counts[sel].astype(np.uint32), ec), q
