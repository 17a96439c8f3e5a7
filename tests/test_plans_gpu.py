"""The benchmark plans end to end on the GPU against the oracle's restatement of the same
plans (bit-exact), at reduced sizes, plus size-independent checks at full size."""
import numpy as np
import pytest

from redfox_b200 import plans as PL

from helpers import (join_aggregate_oracle, join_aggregate_oracle_data, three_relation_oracle,
                     three_relation_oracle_data, to_np)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nr,ns,dom", [(1, 1, 1), (1000, 4000, 256), (50000, 200000, 12500)])
def test_join_aggregate_matches_oracle(cuda, nr, ns, dom):
    r, s = PL.gen_join_aggregate(nr, ns, key_domain=dom)
    er, es = join_aggregate_oracle_data(nr, ns, dom)
    assert np.array_equal(to_np(r), er) and np.array_equal(to_np(s), es)
    keys, sums, counts, total = PL.join_aggregate(r, s)
    ek, esum, ecnt, etot = join_aggregate_oracle(er, es)
    assert total == etot
    assert np.array_equal(to_np(keys).view(np.uint32), ek)
    assert np.array_equal(to_np(sums), esum)
    assert np.array_equal(to_np(counts).view(np.uint32), ecnt)


def test_join_aggregate_full_size_properties(cuda):
    """1M x 4M: ~19.3M join rows, ~2.6e5 groups; totals cross-checked with torch."""
    import torch
    r, s = PL.gen_join_aggregate()
    keys, sums, counts, total = PL.join_aggregate(r, s)
    assert int(counts.to(torch.int64).sum()) == total
    assert 15_000_000 < total < 25_000_000 and 200_000 < keys.shape[0] < 300_000
    assert bool((keys[1:] > keys[:-1]).all())
    # per key: sum = (R rows with the key) x (sum of S amounts with the key)
    rk = (r.view(torch.int64).view(-1) >> 32) & 0xFFFFFFFF
    s64 = s.view(torch.int64).view(-1, 2)
    nR = torch.bincount(rk, minlength=PL.C0_KEY_DOMAIN)
    sS = torch.zeros(PL.C0_KEY_DOMAIN, dtype=torch.int64, device=r.device).index_add_(0, s64[:, 1], s64[:, 0])
    k = keys.to(torch.int64)
    assert torch.equal(sums, nR[k] * sS[k])


@pytest.mark.parametrize("scale", [1000, 100])
def test_three_relation_matches_oracle(cuda, scale):
    n1, n2, n3 = PL.C2_D1_ROWS // scale, PL.C2_D2_ROWS // scale, PL.C2_F_ROWS // scale
    l5, l2 = PL.C2_L5 // scale, PL.C2_L2 // scale
    d1, d2, f, li, lo = PL.gen_three_relation(n1, n2, n3, l5, l2)
    ed1, ed2, ef, eli, elo = three_relation_oracle_data(n1, n2, n3, l5, l2)
    assert np.array_equal(to_np(d1), ed1) and np.array_equal(to_np(d2), ed2) and np.array_equal(to_np(f), ef)
    assert np.array_equal(to_np(li).view(np.uint32), eli) and np.array_equal(to_np(lo).view(np.uint32), elo)
    keys, sums, counts = PL.three_relation(d1, d2, f, li, lo)
    ek, es, ec = three_relation_oracle(ed1, ed2, ef, eli, elo)
    assert np.array_equal(to_np(keys).view(np.uint32), ek)
    assert np.array_equal(to_np(sums), es)
    assert np.array_equal(to_np(counts).view(np.uint32), ec)
