"""Admission logic of the serving loop on a virtual clock (no GPU): FIFO order, slot and
byte-budget limits, oversize queries running alone, and the effect of concurrency on
latency under Poisson arrivals."""
import math

from redfox_b200 import serving as S


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
