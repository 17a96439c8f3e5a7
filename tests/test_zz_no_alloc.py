"""rfx_filter_aggregate_noalloc: the filter-aggregate for callers that cannot allocate
device memory at call time (its scratch is a fixed array inside the library).

It must give exactly the groups, sums and counts of rfx_filter_aggregate and of the
oracle (integer results: no tolerance), on two calls in a row -- the second call reuses
the array the first one left behind -- and allocate no device memory.  This file is
collected last so that a failure here comes after every other test has run; it also
passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from redfox_b200 import rfx as R
from redfox_b200 import workloads as WL

from helpers import fact_oracle, oracle_cmps

pytestmark = pytest.mark.gpu

R.LIB.rfx_filter_aggregate_noalloc.restype = C.c_int
R.LIB.rfx_filter_aggregate_noalloc.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_uint32,
                                               C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32,
                                               C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                               C.c_void_p, C.c_void_p, C.c_void_p]


_warm = set()   # devices whose first call (address lookup, lazy module load) has run


def _free_bytes():
    import torch
    return torch.cuda.mem_get_info()[0]


def _noalloc(fa, rows, n, expect_error=0):
    """One call of the no-allocation entry with fa's descriptors; returns host results.
    After the first call on a device (which looks the array's address up and loads every
    kernel the entry can launch), a call must not change the device's free memory."""
    import torch
    dev = rows.device
    keys = torch.full((fa.G,), -1, dtype=torch.int64, device=dev)
    sums = torch.full((fa.G, max(1, fa.nsum)), -1, dtype=torch.int64, device=dev)
    counts = torch.full((fa.G,), -1, dtype=torch.int64, device=dev)
    groups = torch.full((1,), -1, dtype=torch.int64, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    free0, torch0 = _free_bytes(), torch.cuda.memory_allocated(dev)
    st = R.LIB.rfx_filter_aggregate_noalloc(
        rows.data_ptr(), n, C.addressof(fa.t), C.addressof(fa.cmps), fa.ncmp, C.addressof(fa.ariths), fa.narith,
        C.addressof(fa.gf), C.addressof(fa.gd), fa.ngroup, C.addressof(fa.sf), fa.nsum, keys.data_ptr(),
        sums.data_ptr(), counts.data_ptr(), groups.data_ptr(), err.data_ptr(),
        torch.cuda.current_stream().cuda_stream)
    assert st == R.OK, st
    torch.cuda.synchronize()
    if dev.index in _warm:
        assert _free_bytes() == free0 and torch.cuda.memory_allocated(dev) == torch0
    _warm.add(dev.index)
    g = int(groups.item())
    assert int(err.item()) == expect_error
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
    fa = WL.fact_plan(n)
    _compare(fa, rows, n)
    # and the oracle over the same rows, directly
    ek, es, ec = fact_oracle(rows.cpu().numpy())
    k, s, c = _noalloc(fa, rows, n)
    assert np.array_equal(k.astype(np.uint64), ek) and np.array_equal(s, es) and np.array_equal(c.astype(np.uint64), ec)


def test_noalloc_domain_violation_reported_in_d_error(cuda):
    """Rows whose group field lies outside the declared domain are skipped and reported as
    RFX_ERR_CAPACITY in the caller's error word; the other rows' groups are exact."""
    n = 300_001
    widths = [8, 32]
    rows = R.gen_uniform_rows(n, widths, 99, [0, 0], [16, 1 << 20])
    fa = R.FilterAggregate(n, widths, [], [], [0], [4], [1], device=rows.device)
    host = rows.cpu().numpy()
    for _ in range(2):
        k, s, c = _noalloc(fa, rows, n, expect_error=R.ERR_CAPACITY)
        inside = host[O.unpack(widths, host)[0] < 4]
        ek, es, ec = O.filter_aggregate(inside, widths, oracle_cmps([]), [], [0], [1])
        assert np.array_equal(k.astype(np.uint64), ek) and np.array_equal(s, es)
        assert np.array_equal(c.astype(np.uint64), ec)


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


def test_noalloc_rejects_oversized_plan_like_the_workspace_entry(cuda):
    """8192 groups is beyond the aggregate's 4096-group limit: both entries refuse the plan
    with the same status before launching anything."""
    import torch
    n = 1000
    rows = R.gen_uniform_rows(n, [16, 16], 7, [0, 0], [64, 64])
    fa = R.FilterAggregate(n, [16, 16], [], [], [0, 1], [64, 64], [0], device=rows.device)
    gd = (C.c_uint32 * 2)(128, 64)
    out = torch.zeros(8192 * 2, dtype=torch.int64, device=rows.device)
    stream = torch.cuda.current_stream().cuda_stream
    st = R.LIB.rfx_filter_aggregate_noalloc(
        rows.data_ptr(), n, C.addressof(fa.t), None, 0, None, 0, C.addressof(fa.gf), C.addressof(gd), 2,
        C.addressof(fa.sf), 3, out.data_ptr(), out.data_ptr(), out.data_ptr(), out.data_ptr(), None, stream)
    ws = torch.zeros(1 << 20, dtype=torch.uint8, device=rows.device)
    st_ws = R.LIB.rfx_filter_aggregate(
        rows.data_ptr(), n, C.addressof(fa.t), None, 0, None, 0, C.addressof(fa.gf), C.addressof(gd), 2,
        C.addressof(fa.sf), 3, out.data_ptr(), out.data_ptr(), out.data_ptr(), out.data_ptr(), ws.data_ptr(),
        ws.numel(), stream)
    assert st == st_ws == R.ERR_UNSUPPORTED


def test_noalloc_second_device_after_first(cuda):
    """A 1024-group plan (the shared-table kernel, more than 48 KB of dynamic shared memory)
    on device 0, then on device 1: the shared-memory opt-in is made per device, so the second
    device's launch succeeds and matches.  Needs two GPUs."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    n = 200_000
    widths = [8, 8, 32, 32]
    for d in (0, 1):
        with torch.cuda.device(d):
            dev = torch.device("cuda:%d" % d)
            rows = R.gen_uniform_rows(n, widths, 4321, [0, 0, 0, 0], [32, 32, 1000, 2**32], device=dev)
            fa = R.FilterAggregate(n, widths, [(R.LT, (R.OPND_VAR, 2), (R.OPND_CONST, 900), R.I32)], [], [0, 1],
                                   [32, 32], [2, 3], device=dev)
            _compare(fa, rows, n)
            torch.cuda.synchronize()
