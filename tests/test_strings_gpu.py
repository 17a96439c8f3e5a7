"""String-keyed operators on the GPU against the oracle: dictionary codes, sort_string_key /
sort_string_pair, find_bounds_string, count_string (columns of device pointers to
NUL-terminated strings, compared as signed chars, a proper prefix first)."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from redfox_b200 import rfx as R
from redfox_b200 import workloads as WL

from helpers import to_np

pytestmark = pytest.mark.gpu


def _offsets(ptrs, dpool):
    return (to_np(ptrs) - dpool.data_ptr()).astype(np.uint64)


def _special(name):
    """Columns that stress one property of the order."""
    if name == "empty":
        return O.str_pool([b""] * 300)
    if name == "identical_long":
        return O.str_pool([b"x" * 300] * 257)
    if name == "prefix_chain":
        s = [b"a" * k for k in range(0, 100)] + [b"a" * k + b"b" for k in range(0, 100, 7)]
        return O.str_pool(s[::-1])
    if name == "all_bytes":
        return O.str_pool([bytes([b]) for b in range(255, 0, -1)] + [bytes([b, b]) for b in range(1, 256, 3)])
    if name == "late_difference":
        rng = np.random.default_rng(1)
        return O.str_pool([b"k" * 60 + bytes([int(c)]) + b"z" * int(t) for c, t in
                           zip(rng.integers(1, 256, 2000), rng.integers(0, 3, 2000))])
    raise KeyError(name)


COLUMNS = ["gen_1", "gen_7", "gen_1000", "gen_200000", "empty", "identical_long", "prefix_chain", "all_bytes",
           "late_difference"]


def _column(name):
    if name.startswith("gen_"):
        n = int(name[4:])
        return WL.gen_strings(n, seed=n)
    return _special(name)


@pytest.mark.parametrize("name", COLUMNS)
def test_string_codes(cuda, name):
    pool, offs = _column(name)
    dpool, ptrs = R.string_column(pool, offs, cuda)
    codes, perm, d = R.string_codes(ptrs)
    ecodes, ed = O.str_codes(pool, offs)
    assert d == ed
    assert np.array_equal(to_np(codes).view(np.uint32), ecodes)
    assert np.array_equal(offs[to_np(perm)], O.str_sort(pool, offs))
    assert R.device_status() == R.OK


@pytest.mark.parametrize("name", ["gen_1000", "gen_200000", "prefix_chain", "all_bytes", "late_difference"])
def test_sort_string_key(cuda, name):
    pool, offs = _column(name)
    dpool, ptrs = R.string_column(pool, offs, cuda)
    R.sort_strings(ptrs)
    assert np.array_equal(_offsets(ptrs, dpool), O.str_sort(pool, offs))


@pytest.mark.parametrize("vtype,vbytes", [(R.I8, 1), (R.I16, 2), (R.I32, 4), (R.I64, 8), (R.I128, 16),
                                          (R.I256, 32), (R.I512, 64)])
def test_sort_string_pair(cuda, vtype, vbytes):
    import torch
    pool, offs = WL.gen_strings(30000, seed=vbytes)
    rng = np.random.default_rng(vbytes)
    vals = rng.integers(0, 256, (offs.shape[0], vbytes), dtype=np.uint8)
    dpool, ptrs = R.string_column(pool, offs, cuda)
    dvals = torch.from_numpy(vals.copy()).to(cuda)
    R.sort_strings(ptrs, dvals, vtype)
    eo, ev = O.str_sort(pool, offs, vals)
    assert np.array_equal(_offsets(ptrs, dpool), eo)
    assert np.array_equal(to_np(dvals), ev)


@pytest.mark.parametrize("nl,nr", [(0, 100), (100, 0), (5000, 8000), (60000, 40000)])
def test_find_bounds_string(cuda, nl, nr):
    lp, lo = WL.gen_strings(nl, seed=11, distinct=max(1, nl // 3))
    rp, ro = WL.gen_strings(nr, seed=12, distinct=max(1, nr // 3))
    # one pool: the left strings, then the right strings
    pool = np.concatenate([lp, rp])
    lo = O.str_sort(pool, lo)
    ro = O.str_sort(pool, ro + np.uint64(lp.shape[0]))
    dpool, _ = R.string_column(pool, np.zeros(0, np.uint64), cuda)
    import torch
    base = dpool.data_ptr()
    left = torch.from_numpy(lo.view(np.int64)).to(cuda) + base
    right = torch.from_numpy(ro.view(np.int64)).to(cuda) + base
    lb, sc, tot = R.find_bounds_string(left, right)
    elb, esc, etot = O.str_find_bounds(pool, lo, ro)
    assert tot == etot
    assert np.array_equal(to_np(lb), elb) and np.array_equal(to_np(sc), esc)


@pytest.mark.parametrize("name,sort", [("gen_1", False), ("gen_1000", True), ("gen_200000", True),
                                       ("gen_200000", False), ("empty", False), ("prefix_chain", True),
                                       ("late_difference", False)])
def test_count_string(cuda, name, sort):
    import torch
    pool, offs = _column(name)
    if sort:
        offs = O.str_sort(pool, offs)
    rng = np.random.default_rng(5)
    vals = rng.integers(0, 2**32, offs.shape[0], dtype=np.uint64).astype(np.uint32)
    dpool, ptrs = R.string_column(pool, offs, cuda)
    dv = torch.from_numpy(vals.view(np.int32)).to(cuda)
    ok, ov = R.count_string(ptrs, dv)
    eo, es = O.str_count(pool, offs, vals)
    assert np.array_equal(_offsets(ok, dpool), eo)
    assert np.array_equal(to_np(ov).view(np.uint32), es)


def test_count_string_empty_column(cuda):
    import torch
    ptrs = torch.zeros(0, dtype=torch.int64, device=cuda)
    vals = torch.zeros(0, dtype=torch.int32, device=cuda)
    ok, ov = R.count_string(ptrs, vals)
    assert ok.numel() == 0 and ov.numel() == 0


def test_string_shims(cuda):
    """The redfox:: string entries of the shim libraries forward to the same kernels."""
    import torch
    from test_shim import _fn, P, U
    pool, offs = WL.gen_strings(20000, seed=3, distinct=4000)
    dpool, ptrs = R.string_column(pool, offs, cuda)
    vals = torch.arange(20000, dtype=torch.int32, device=cuda)
    torch.cuda.synchronize()
    _fn("mgpu", "redfox::sort_string_pair(void*, void*, unsigned long long, unsigned long long, "
                "unsigned long long)", [P, P, U, U, U])(ptrs.data_ptr(), vals.data_ptr(), 20000, 0, R.I32)
    eo, ev = O.str_sort(pool, offs, np.arange(20000, dtype=np.int32))
    assert np.array_equal(_offsets(ptrs, dpool), eo) and np.array_equal(to_np(vals), ev)
    lb = torch.empty(20000, dtype=torch.int32, device=cuda)
    lc = torch.empty(20000, dtype=torch.int32, device=cuda)
    rs = torch.zeros(1, dtype=torch.int64, device=cuda)
    _fn("ra", "redfox::find_bounds_string(void*, void*, unsigned long long*, void*, unsigned long long, void*, "
              "unsigned long long)", [P, P, P, P, U, P, U])(lb.data_ptr(), lc.data_ptr(), rs.data_ptr(),
                                                             ptrs.data_ptr(), 20000, ptrs.data_ptr(), 20000)
    elb, esc, etot = O.str_find_bounds(pool, eo, eo)
    assert int(rs.item()) == etot and np.array_equal(to_np(lb), elb) and np.array_equal(to_np(lc), esc)
    ok = torch.empty(20000, dtype=torch.int64, device=cuda)
    ov = torch.empty(20000, dtype=torch.int32, device=cuda)
    ks = torch.tensor([8 * 20000], dtype=torch.int64, device=cuda)
    vs = torch.tensor([4 * 20000], dtype=torch.int64, device=cuda)
    ones = torch.ones(20000, dtype=torch.int32, device=cuda)
    torch.cuda.synchronize()
    _fn("ra", "redfox::count_string(void const*, void const*, void*, void*, unsigned long long*, "
              "unsigned long long*)", [P, P, P, P, P, P])(ptrs.data_ptr(), ones.data_ptr(), ok.data_ptr(),
                                                          ov.data_ptr(), ks.data_ptr(), vs.data_ptr())
    g = int(ks.item()) // 8
    eko, eks = O.str_count(pool, eo, np.ones(20000, np.uint32))
    assert g == len(eko) and int(vs.item()) // 4 == g
    assert np.array_equal(_offsets(ok[:g], dpool), eko) and np.array_equal(to_np(ov[:g]).view(np.uint32), eks)
    keys = ptrs.clone()
    _fn("ra", "redfox::sort_string(void*, void*)", [P, P])(keys.data_ptr(), keys.data_ptr() + 8 * 20000)
    assert np.array_equal(_offsets(keys, dpool), eo)   # already sorted: unchanged
    assert R.device_status() == R.OK
