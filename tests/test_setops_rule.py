"""The keep rule the set filters' kernels apply, restated in numpy and checked against the
oracle's set_intersection / set_difference (STL multiset semantics): an element of A of
rank r within its run of equal values is matched when B's element r places after the
value's lower bound in B equals it.  The warp-segment kernel decides exactly this with its
window of B (heads, run starts and lower bounds found per tile and warp); the GPU tests
compare the kernels themselves with the oracle."""
import numpy as np
import pytest

import oracle as O


def _matched(a, b):
    i = np.arange(len(a))
    rank = i - np.searchsorted(a, a, side="left")
    lb = np.searchsorted(b, a, side="left")
    at = lb + rank
    ok = at < len(b)
    hit = np.zeros(len(a), dtype=bool)
    hit[ok] = b[at[ok]] == a[ok]
    return hit


@pytest.mark.parametrize("seed", range(6))
def test_rank_rule_matches_oracle(seed):
    rng = np.random.default_rng(seed)
    for na, nb, hi in ((0, 10, 5), (10, 0, 5), (1000, 300, 3), (5000, 5000, 100), (3000, 700, 1 << 30)):
        a = np.sort(rng.integers(0, hi, na)).astype(np.uint32)
        b = np.sort(rng.integers(0, hi, nb)).astype(np.uint32)
        m = _matched(a, b)
        assert np.array_equal(a[m], O.set_intersection(a, b))
        assert np.array_equal(a[~m], O.set_difference(a, b))
