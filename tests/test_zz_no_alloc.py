"""rfx_filter_aggregate_noalloc: the filter-aggregate for callers that cannot allocate
device memory at call time (its scratch is a fixed array inside the library).

It must give exactly the groups, sums and counts of rfx_filter_aggregate (integer
results: no tolerance), on two calls in a row -- the second call reuses the array the
first one left behind.  This file is collected last so that a failure here comes after
every other test has run; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from redfox_b200 import rfx as R
from redfox_b200 import workloads as WL

pytestmark = pytest.mark.gpu

R.LIB.rfx_filter_aggregate_noalloc.restype = C.c_int
R.LIB.rfx_filter_aggregate_noalloc.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_uint32,
                                               C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32,
                                               C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                               C.c_void_p, C.c_void_p, C.c_void_p]


def _noalloc(fa, rows, n):
    """One call of the no-allocation entry with fa's descriptors; returns host results."""
    import torch
    dev = rows.device
    keys = torch.full((fa.G,), -1, dtype=torch.int64, device=dev)
    sums = torch.full((fa.G, max(1, fa.nsum)), -1, dtype=torch.int64, device=dev)
    counts = torch.full((fa.G,), -1, dtype=torch.int64, device=dev)
    groups = torch.full((1,), -1, dtype=torch.int64, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    st = R.LIB.rfx_filter_aggregate_noalloc(
        rows.data_ptr(), n, C.addressof(fa.t), C.addressof(fa.cmps), fa.ncmp, C.addressof(fa.ariths), fa.narith,
        C.addressof(fa.gf), C.addressof(fa.gd), fa.ngroup, C.addressof(fa.sf), fa.nsum, keys.data_ptr(),
        sums.data_ptr(), counts.data_ptr(), groups.data_ptr(), err.data_ptr(),
        torch.cuda.current_stream().cuda_stream)
    assert st == R.OK, st
    torch.cuda.synchronize()
    g = int(groups.item())
    assert int(err.item()) == 0
    return keys[:g].cpu().numpy(), sums[:g, :fa.nsum].cpu().numpy(), counts[:g].cpu().numpy()


def _compare(fa, rows, n):
    fa.launch(rows, n=n)
    ek, es, ec = fa.result()
    assert R.device_status() == R.OK
    for _ in range(2):  # two calls in a row share (and must reset) the fixed scratch
        k, s, c = _noalloc(fa, rows, n)
        assert np.array_equal(k.astype(np.uint64), ek)
        assert np.array_equal(s, es)
        assert np.array_equal(c.astype(np.uint64), ec)


def test_noalloc_fact_plan_matches_workspace_entry(cuda):
    n = 2_000_003
    rows = WL.gen_fact(n)
    _compare(WL.fact_plan(n), rows, n)


def test_noalloc_larger_group_table_matches(cuda):
    """1024 groups with two sums: the shared-table kernel path."""
    import torch
    n = 500_000
    widths = [8, 8, 32, 32]
    rows = R.gen_uniform_rows(n, widths, 1234, [0, 0, 0, 0], [32, 32, 1000, 2**32])
    fa = R.FilterAggregate(n, widths, [(R.LT, (R.OPND_VAR, 2), (R.OPND_CONST, 900), R.I32)], [], [0, 1], [32, 32],
                           [2, 3], device=rows.device)
    _compare(fa, rows, n)
    torch.cuda.synchronize()


def test_noalloc_rejects_oversized_plan(cuda):
    import torch
    n = 1000
    rows = R.gen_uniform_rows(n, [16, 16], 7, [0, 0], [64, 64])
    # 128 x 64 = 8192 groups x (3 sums + a count) = 32768 accumulators > the 20480-word array
    fa = R.FilterAggregate(n, [16, 16], [], [], [0, 1], [128, 64], [0], device=rows.device)
    out = torch.zeros(8192 * 2, dtype=torch.int64, device=rows.device)
    st = R.LIB.rfx_filter_aggregate_noalloc(
        rows.data_ptr(), n, C.addressof(fa.t), None, 0, None, 0, C.addressof(fa.gf), C.addressof(fa.gd), 2,
        C.addressof(fa.sf), 3, out.data_ptr(), out.data_ptr(), out.data_ptr(), out.data_ptr(), None,
        torch.cuda.current_stream().cuda_stream)
    assert st == R.ERR_CAPACITY
