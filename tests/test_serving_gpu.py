"""The serving loop on the GPU: every query's result is the same served in the mix (packed
into batched rounds with other queries, rounds overlapping on two streams) as run alone,
and matches the oracle; a small memory budget limits how many run at once without changing
any result."""
import numpy as np
import pytest

from redfox_b200 import serving as S

from helpers import serving_query_oracle, to_np

pytestmark = pytest.mark.gpu

SCALE = 100


@pytest.fixture(scope="module")
def resident(cuda):
    from redfox_b200 import plans as PL
    return S.Resident(PL.C2_D1_ROWS // SCALE, PL.C2_D2_ROWS // SCALE, PL.C2_F_ROWS // SCALE)


def _requests(res, n, seed):
    return S.gen_requests(n, rate=1e6, seed=seed, n2=res.n2)   # all arrive within microseconds


def test_round_equals_alone(resident):
    """One batched round of 40 mixed queries (with and without key lists, every segment)
    gives each query exactly its plain result."""
    reqs = _requests(resident, 40, seed=23)
    assert any(q.list_size for q in reqs) and any(not q.list_size for q in reqs)
    outs = S.run_round_host(resident, reqs, "cuda")
    for q, got in zip(reqs, outs):
        alone = S.run_alone(resident, q)
        assert np.array_equal(got[0], alone[0].numpy().view(np.uint32)), q
        assert np.array_equal(got[1], alone[1].numpy()), q
        assert np.array_equal(got[2], alone[2].numpy().view(np.uint32)), q


def test_served_results_equal_alone_and_oracle(resident):
    reqs = _requests(resident, 16, seed=21)
    srv = S.Server(resident, slots=2)
    sch = srv.serve(reqs, keep_results=True)
    assert sch.peak_queries > 1                          # they really overlapped
    assert max(srv.rounds) > 1                           # and were packed into rounds
    d1, d2, f = to_np(resident.d1), to_np(resident.d2), to_np(resident.f_sorted)
    for i, q in enumerate(reqs):
        alone = S.run_alone(resident, q)
        assert np.array_equal(q.result[0], alone[0].numpy().view(np.uint32)), q
        assert np.array_equal(q.result[1], alone[1].numpy()), q
        assert np.array_equal(q.result[2], alone[2].numpy().view(np.uint32)), q
        if i < 4:
            lst = S.query_list(q, resident.n2, "cuda")
            lst = None if lst is None else to_np(lst).view(np.uint32)
            ek, es, ec = serving_query_oracle(d1, d2, f, q.segment, q.date_lo, q.date_hi, lst)
            assert np.array_equal(alone[0].numpy().view(np.uint32), ek)
            assert np.array_equal(alone[1].numpy(), es)
            assert np.array_equal(alone[2].numpy().view(np.uint32), ec)
    summ = S.latency_summary(reqs)
    assert summ["latency_ms_p99"] >= summ["latency_ms_p50"] > 0


def test_small_budget_limits_concurrency(resident):
    reqs = _requests(resident, 10, seed=22)
    budget = 2 * max(q.est_bytes for q in reqs)
    sch = S.Server(resident, slots=2, budget_bytes=budget).serve(reqs, keep_results=True)
    assert sch.peak_bytes <= budget
    for q in reqs[:3]:
        alone = S.run_alone(resident, q)
        assert np.array_equal(q.result[0], alone[0].numpy().view(np.uint32))
        assert np.array_equal(q.result[1], alone[1].numpy())
        assert np.array_equal(q.result[2], alone[2].numpy().view(np.uint32))


def test_plain_server_is_one_query_at_a_time(resident):
    reqs = _requests(resident, 6, seed=24)
    srv = S.Server(resident, slots=1, plain=True)
    sch = srv.serve(reqs, keep_results=True)
    assert sch.peak_queries == 1 and max(srv.rounds) == 1
    q = reqs[0]
    alone = S.run_alone(resident, q)
    assert np.array_equal(q.result[0], alone[0].numpy().view(np.uint32))
    assert np.array_equal(q.result[1], alone[1].numpy())
    assert np.array_equal(q.result[2], alone[2].numpy().view(np.uint32))


def test_single_query_round_on_a_side_stream(resident):
    """A round of one query runs the plain plan on the round's stream; the batched plan
    given the same single query agrees with it."""
    import torch
    reqs = _requests(resident, 3, seed=25)
    st = torch.cuda.Stream()
    for q in reqs:
        got = S.run_round_host(resident, [q], "cuda", stream=st, stage=S.PinnedStage(1 << 20))[0]
        alone = S.run_alone(resident, q)
        lst = S.query_list(q, resident.n2, "cuda")
        gk, gs, gc = S.run_round(resident, [q], None if lst is None else [lst])
        bk, bs, bc = S.split_round(gk, gs, gc, 1)[0]
        for a, b in ((got[0], alone[0].numpy().view(np.uint32)), (got[1], alone[1].numpy()),
                     (got[2], alone[2].numpy().view(np.uint32)), (bk, got[0]), (bs, got[1]), (bc, got[2])):
            assert np.array_equal(a, b), q


def test_small_round_runs_plain_plans(cuda, resident):
    """A round of fewer queries than the batching threshold runs them one after another with
    the plain plan, results staged at separate offsets of the page-locked buffer: each equals
    the query run alone, also with views (copy=False) that must not overlap."""
    import torch
    reqs = _requests(resident, 3, seed=26)
    st = torch.cuda.Stream()
    outs = S.run_round_host(resident, reqs, "cuda", stream=st, stage=S.PinnedStage(1 << 20), copy=False)
    for q, got in zip(reqs, outs):
        alone = S.run_alone(resident, q)
        assert np.array_equal(got[0], alone[0].numpy().view(np.uint32)), q
        assert np.array_equal(got[1], alone[1].numpy()), q
        assert np.array_equal(got[2], alone[2].numpy().view(np.uint32)), q
