"""The serving loop on the GPU: every query's result is the same served in the mix (several
in flight on different streams) as run alone, and matches the oracle; a small memory budget
limits how many run at once without changing any result."""
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


def test_served_results_equal_alone_and_oracle(resident):
    reqs = _requests(resident, 16, seed=21)
    srv = S.Server(resident, slots=4)
    sch = srv.serve(reqs, keep_results=True)
    assert sch.peak_queries > 1                          # they really overlapped
    d1, d2, f = to_np(resident.d1), to_np(resident.d2), to_np(resident.f_sorted)
    for i, q in enumerate(reqs):
        alone = S.run_alone(resident, q)
        for a, b in zip(q.result, alone):
            assert np.array_equal(a.numpy(), b.numpy()), q
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
    sch = S.Server(resident, slots=8, budget_bytes=budget).serve(reqs, keep_results=True)
    assert sch.peak_queries <= 8
    assert sch.peak_bytes <= budget
    for q in reqs[:3]:
        alone = S.run_alone(resident, q)
        for a, b in zip(q.result, alone):
            assert np.array_equal(a.numpy(), b.numpy())
