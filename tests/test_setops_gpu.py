"""Set operations and unique against the oracle and the reference's golden vectors."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle as O
from redfox_b200 import rfx as R

from helpers import to_np

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def _cases():
    g = np.load(os.path.join(GOLD, "setops.npz"))
    return g, sorted({k.rsplit("_", 1)[0] for k in g.files if k.endswith("_a")})


def test_set_ops_match_reference_golden(cuda):
    g, keys = _cases()
    for key in keys:
        a, b = g[key + "_a"], g[key + "_b"]
        da, db = _dev(a, cuda), _dev(b, cuda)
        assert np.array_equal(to_np(R.set_op(R.SET_UNION, da, db)), g[key + "_union"]), key
        assert np.array_equal(to_np(R.set_op(R.SET_DIFFERENCE, da, db)), g[key + "_difference"]), key
        if key + "_intersection" in g.files:
            assert np.array_equal(to_np(R.set_op(R.SET_INTERSECTION, da, db)), g[key + "_intersection"]), key
        if key + "_unique" in g.files:
            assert np.array_equal(to_np(R.unique(_dev(a, cuda))), g[key + "_unique"]), key


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16, np.uint32, np.uint64])
@pytest.mark.parametrize("na,nb,hi", [(0, 0, 10), (0, 100, 10), (100, 0, 10), (1, 1, 2), (1023, 1025, 50),
                                      (100003, 70001, 3000), (200000, 200000, 2**31)])
def test_set_ops_random(cuda, dtype, na, nb, hi):
    rng = np.random.default_rng(na + nb)
    hi = min(hi, np.iinfo(dtype).max)
    a = np.sort(rng.integers(0, hi, na)).astype(dtype)
    b = np.sort(rng.integers(0, hi, nb)).astype(dtype)
    da, db = _dev(a, cuda), _dev(b, cuda)
    for op, ref in ((R.SET_UNION, O.set_union), (R.SET_DIFFERENCE, O.set_difference),
                    (R.SET_INTERSECTION, O.set_intersection)):
        assert np.array_equal(to_np(R.set_op(op, da, db)), ref(a, b)), op
    assert np.array_equal(to_np(R.unique(_dev(a, cuda))), O.unique(a))
    assert R.device_status() == R.OK


def test_set_ops_128bit(cuda):
    rng = np.random.default_rng(8)
    def mk(n):
        k = np.sort(rng.integers(0, 2000, n)).astype(np.uint64)
        a = np.zeros((n, 16), np.uint8)
        a.view(np.uint64)[:, 1] = k // 5
        a.view(np.uint64)[:, 0] = k % 5
        return a
    a, b = mk(40000), mk(30000)
    da, db = _dev(a, cuda), _dev(b, cuda)
    assert np.array_equal(to_np(R.set_op(R.SET_UNION, da, db)), O.set_union(a, b))
    assert np.array_equal(to_np(R.set_op(R.SET_DIFFERENCE, da, db)), O.set_difference(a, b))
    assert np.array_equal(to_np(R.set_op(R.SET_INTERSECTION, da, db)), O.set_intersection(a, b))
    assert np.array_equal(to_np(R.unique(_dev(a, cuda))), O.unique(a))


def test_unique_all_equal_and_all_distinct(cuda):
    import torch
    n = 1_000_003
    x = torch.full((n,), 5, dtype=torch.int32, device=cuda)
    assert R.unique(x).shape[0] == 1
    y = torch.arange(n, dtype=torch.int64, device=cuda)
    assert torch.equal(R.unique(y), torch.arange(n, dtype=torch.int64, device=cuda))


def test_reference_compatible_set_entries(cuda):
    import torch
    g, keys = _cases()
    a, b = g["e4_c1_a"], g["e4_c1_b"]
    da, db = _dev(a, cuda), _dev(b, cuda)
    out = torch.zeros(len(a) + len(b), dtype=torch.int32, device=cuda)
    size = torch.zeros(1, dtype=torch.int64, device=cuda)
    P = C.c_void_p
    torch.cuda.synchronize()
    assert R.LIB.rfx_set_union_compat(P(out.data_ptr()), P(size.data_ptr()), P(da.data_ptr()),
                                      P(da.data_ptr() + 4 * len(a)), P(db.data_ptr()), P(db.data_ptr() + 4 * len(b)),
                                      R.I32) == R.OK
    k = int(size.item()) // 4
    assert np.array_equal(to_np(out)[:k].view(np.uint32), g["e4_c1_union"])
    assert R.LIB.rfx_difference_compat(P(out.data_ptr()), P(size.data_ptr()), P(da.data_ptr()),
                                       P(da.data_ptr() + 4 * len(a)), P(db.data_ptr()), P(db.data_ptr() + 4 * len(b)),
                                       R.I32) == R.OK
    k = int(size.item()) // 4
    assert np.array_equal(to_np(out)[:k].view(np.uint32), g["e4_c1_difference"])
    u = _dev(a, cuda)
    size = torch.tensor([4 * len(a)], dtype=torch.int64, device=cuda)
    torch.cuda.synchronize()
    assert R.LIB.rfx_unique_compat(P(u.data_ptr()), P(size.data_ptr()), R.I32) == R.OK
    k = int(size.item()) // 4
    assert np.array_equal(to_np(u)[:k], g["e4_c1_unique"])
    assert R.LIB.rfx_set_union_compat(P(out.data_ptr()), P(size.data_ptr()), P(da.data_ptr()), P(da.data_ptr()),
                                      P(db.data_ptr()), P(db.data_ptr()), 99) == R.ERR_UNSUPPORTED


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("dtype", [np.uint32, np.uint64])
def test_set_filter_variants(cuda, variant, dtype):
    """Every variant pinned through the tuner -- the warp-segment form (0 and 5: 16 and 8
    items per thread, fewer where a tile's window would not fit), the one-pass form (1, 2,
    3) and the two-pass form (4 and 6: 16 and 8) -- gives the STL results, across tile
    boundaries of every variant (1024 / 2048 / 4096 elements) and with runs of equal values
    that cross warp segments and tiles."""
    try:
        R.tune_force(2, variant)
        rng = np.random.default_rng(variant * 10 + np.dtype(dtype).itemsize)
        for na, nb, hi in ((4095, 4097, 900), (4096, 1000, 50), (300_001, 120_007, 100_000), (8193, 8191, 3)):
            a = np.sort(rng.integers(0, hi, na)).astype(dtype)
            b = np.sort(rng.integers(0, hi, nb)).astype(dtype)
            da, db = _dev(a, cuda), _dev(b, cuda)
            for op, ref in ((R.SET_UNION, O.set_union), (R.SET_DIFFERENCE, O.set_difference),
                            (R.SET_INTERSECTION, O.set_intersection)):
                assert np.array_equal(to_np(R.set_op(op, da, db)), ref(a, b)), (op, na, nb)
        assert R.device_status() == R.OK
    finally:
        R.tune_force(2, -1)


@pytest.mark.parametrize("variant", [0, 5])
def test_set_filter_segments_edges(cuda, variant):
    """The warp-segment form on its edge cases: a run in B far longer than a tile's window
    capacity (that tile's items search B in global memory), runs of one value across whole
    tiles of A, many duplicates on both sides, inputs not 16-byte aligned (the two-pass form
    takes those) and an empty B, with B shorter and longer than A; every result is the STL
    one."""
    try:
        R.tune_force(2, variant)
        rng = np.random.default_rng(50 + variant)
        a = np.sort(np.concatenate([rng.integers(0, 1 << 20, 200_000), np.full(30_000, 777_777)])).astype(np.uint32)
        b = np.sort(np.concatenate([rng.integers(0, 1 << 20, 50_000), np.full(60_000, 777_777),
                                    np.full(9_000, 5)])).astype(np.uint32)
        a2 = np.sort(np.concatenate([rng.integers(0, 1 << 20, 500_000), np.full(30_000, 777_777)])).astype(np.uint32)
        b2 = np.sort(np.concatenate([rng.integers(0, 1 << 20, 20_000), np.full(60_000, 777_777),
                                     np.full(9_000, 5)])).astype(np.uint32)
        a3 = np.sort(rng.integers(0, 300, 100_000)).astype(np.uint32)
        b3 = np.sort(rng.integers(0, 300, 20_000)).astype(np.uint32)
        cases = [(a, b), (a[3:], b[1:]), (a, b[:0]), (np.full(20_000, 9, np.uint32), np.full(7_001, 9, np.uint32)),
                 (a2, b2), (a3, b3), (a3.astype(np.uint64), b3.astype(np.uint64)), (b2, a2)]
        for x, y in cases:
            dx, dy = _dev(x, cuda), _dev(y, cuda)
            for op, ref in ((R.SET_UNION, O.set_union), (R.SET_DIFFERENCE, O.set_difference),
                            (R.SET_INTERSECTION, O.set_intersection)):
                assert np.array_equal(to_np(R.set_op(op, dx, dy)), ref(x, y)), (op, len(x), len(y))
        # misaligned views of the same arrays
        da, db = _dev(a, cuda), _dev(b, cuda)
        for op, ref in ((R.SET_DIFFERENCE, O.set_difference), (R.SET_INTERSECTION, O.set_intersection)):
            assert np.array_equal(to_np(R.set_op(op, da[1:], db[3:])), ref(a[1:], b[3:]))
        assert R.device_status() == R.OK
    finally:
        R.tune_force(2, -1)


@pytest.mark.parametrize("op", ["intersection", "difference"])
def test_set_filter_in_place(cuda, op):
    """Intersection and difference written over A itself (the output overlaps the input)
    take the one-pass form, whose writes never pass inputs not yet read: the result is the
    oracle's, across many tiles."""
    import torch
    rng = np.random.default_rng(7)
    na, nb, hi = 300_001, 120_007, 90_000
    a = np.sort(rng.integers(0, hi, na)).astype(np.uint32)
    b = np.sort(rng.integers(0, hi, nb)).astype(np.uint32)
    da, db = _dev(a, cuda), _dev(b, cuda)
    cnt = torch.zeros(1, dtype=torch.int64, device=cuda)
    code = R.SET_INTERSECTION if op == "intersection" else R.SET_DIFFERENCE
    wsb = R.LIB.rfx_set_op_workspace(code, na, nb, 4)
    ws = torch.empty(wsb, dtype=torch.uint8, device=cuda)
    R.check("set", R.LIB.rfx_set_op(code, R._ptr(da), R._ptr(cnt), R._ptr(da), na, R._ptr(db), nb, 4, R._ptr(ws),
                                    wsb, R._stream()))
    exp = getattr(O, "set_" + op)(a, b)
    assert int(cnt.item()) == len(exp)
    assert np.array_equal(to_np(da)[:len(exp)], exp)
