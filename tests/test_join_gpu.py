"""Join (find_bounds, expansion, gather, fused tuple join) against the oracle and the
reference's known answers; bit-exact."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from redfox_b200 import rfx as R

from helpers import to_np

pytestmark = pytest.mark.gpu


def _dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def _sorted(n, hi, dtype, seed):
    return np.sort(np.random.default_rng(seed).integers(0, hi, n)).astype(dtype)


KEYS = [(np.uint8, 1, 200), (np.uint16, 2, 5000), (np.uint32, 4, 300000), (np.uint64, 8, 2**40)]


@pytest.mark.parametrize("dtype,kb,hi", KEYS)
@pytest.mark.parametrize("nl,nr", [(0, 10), (10, 0), (1, 1), (1023, 1025), (5000, 20000), (100003, 30011)])
def test_find_bounds_expand_gather(cuda, dtype, kb, hi, nl, nr):
    left = _sorted(nl, hi, dtype, seed=nl * 3 + kb)
    right = _sorted(nr, hi, dtype, seed=nr * 5 + kb)
    lb, sc, total = R.find_bounds(_dev(left, cuda), _dev(right, cuda))
    elb, esc, etot = O.find_bounds(left, right)
    assert total == etot
    assert np.array_equal(to_np(lb), elb) and np.array_equal(to_np(sc), esc)
    if total == 0:
        return
    li, ri = R.join_expand(lb, sc, total)
    eli, eri = O.join_expand(elb, esc, etot)
    assert np.array_equal(to_np(li), eli) and np.array_equal(to_np(ri), eri)
    lval = np.random.default_rng(1).integers(0, 2**31, nl).astype(np.uint32)
    rval = np.random.default_rng(2).integers(0, 2**31, nr).astype(np.uint32)
    ob = R.container_bytes(kb * 8 + 64)
    got = R.join_gather(ob, li, ri, _dev(left, cuda), _dev(lval, cuda), 32, _dev(rval, cuda), 32)
    exp = O.join_gather(ob, eli, eri, left, lval, 32, rval, 32)
    assert np.array_equal(to_np(got), exp)


def test_find_bounds_128bit_keys(cuda):
    n = 20000
    rng = np.random.default_rng(4)
    ks = np.sort(rng.integers(0, 5000, n)).astype(np.uint64)
    left = np.zeros((n, 16), np.uint8)
    left.view(np.uint64)[:, 1] = ks // 7
    left.view(np.uint64)[:, 0] = ks % 7
    ks2 = np.sort(rng.integers(0, 5000, n)).astype(np.uint64)
    right = np.zeros((n, 16), np.uint8)
    right.view(np.uint64)[:, 1] = ks2 // 7
    right.view(np.uint64)[:, 0] = ks2 % 7
    lb, sc, total = R.find_bounds(_dev(left, cuda), _dev(right, cuda))
    elb, esc, etot = O.find_bounds(left, right)
    assert total == etot and np.array_equal(to_np(lb), elb) and np.array_equal(to_np(sc), esc)


def test_testjoin_identity_self_join(cuda):
    """TestJoin.cu:107-156 known answer: 2^15 ushort keys joined with themselves."""
    n = 1 << 15
    keys = np.arange(n, dtype=np.uint16)
    d = _dev(keys, cuda)
    lb, sc, total = R.find_bounds(d, d)
    assert total == n
    li, ri = R.join_expand(lb, sc, total)
    out = to_np(R.join_gather(4, li, ri, d, None, 0, d, 16)).view(np.uint32).ravel()
    ar = np.arange(n, dtype=np.uint32)
    assert np.array_equal(out, (ar << 16) | ar)


@pytest.mark.parametrize("lw,lvb,rw,rvb,ow", [(8, 32, 16, 64, 16), (16, 64, 8, 32, 16), (8, 32, 8, 32, 8),
                                                (4, 8, 4, 16, 8), (16, 96, 16, 64, 16)])
def test_fused_tuple_join(cuda, lw, lvb, rw, rvb, ow):
    rng = np.random.default_rng(lw * 100 + rvb)
    nl, nr = 30000, 50000
    kbits_l, kbits_r = lw * 8 - lvb, rw * 8 - rvb
    kb = min(kbits_l, kbits_r, 20)
    lk = np.sort(rng.integers(0, 2**kb // 3 + 1, nl)).astype(np.uint64)
    rk = np.sort(rng.integers(0, 2**kb // 3 + 1, nr)).astype(np.uint64)
    left = O.pack([kbits_l, lvb], [lk, rng.integers(0, 2**min(lvb, 63), nl, dtype=np.uint64)])
    right = O.pack([kbits_r, rvb], [rk, rng.integers(0, 2**min(rvb, 63), nr, dtype=np.uint64)])
    got, total = R.join_tuples(_dev(left, cuda), lvb, _dev(right, cuda), rvb, ow)
    exp = O.join_tuples(left, lvb, right, rvb, ow)
    assert total == len(exp)
    assert np.array_equal(to_np(got), exp)


def test_fused_join_capacity_and_skew(cuda):
    """A Zipf-skewed key with ~1M matches; a short capacity writes a prefix and reports the total."""
    n = 200000
    left = O.pack([32, 32], [np.zeros(8, np.uint64), np.arange(8, dtype=np.uint64)])
    rk = np.sort(np.concatenate([np.zeros(n, np.uint64), np.arange(1, n, dtype=np.uint64)]))
    right = O.pack([32, 64], [rk, np.arange(len(rk), dtype=np.uint64)])
    got, total = R.join_tuples(_dev(left, cuda), 32, _dev(right, cuda), 64, 16)
    exp = O.join_tuples(left, 32, right, 64, 16)
    assert total == len(exp) == 8 * n
    assert np.array_equal(to_np(got), exp)
    part, total2 = R.join_tuples(_dev(left, cuda), 32, _dev(right, cuda), 64, 16, capacity=1000)
    assert total2 == total and np.array_equal(to_np(part), exp[:1000])


def test_reference_compatible_join_entries(cuda):
    import torch
    left = _sorted(5000, 3000, np.uint32, 1)
    right = _sorted(7000, 3000, np.uint32, 2)
    dl, dr = _dev(left, cuda), _dev(right, cuda)
    lb = torch.empty(5000, dtype=torch.int32, device=cuda)
    lc = torch.empty(5000, dtype=torch.int32, device=cuda)
    rs = torch.zeros(1, dtype=torch.int64, device=cuda)
    torch.cuda.synchronize()
    assert R.LIB.rfx_find_bounds_compat(C.c_void_p(lb.data_ptr()), C.c_void_p(lc.data_ptr()), C.c_void_p(rs.data_ptr()),
                                        C.c_void_p(dl.data_ptr()), 5000, C.c_void_p(dr.data_ptr()), 7000, 4) == R.OK
    elb, esc, etot = O.find_bounds(left, right)
    assert int(rs.item()) == etot and np.array_equal(to_np(lb), elb) and np.array_equal(to_np(lc), esc)
    li = torch.empty(etot, dtype=torch.int32, device=cuda)
    ri = torch.empty(etot, dtype=torch.int32, device=cuda)
    assert R.LIB.rfx_join_compat(C.c_void_p(li.data_ptr()), C.c_void_p(ri.data_ptr()), etot, C.c_void_p(lb.data_ptr()),
                                 C.c_void_p(lc.data_ptr()), 5000) == R.OK
    eli, eri = O.join_expand(elb, esc, etot)
    assert np.array_equal(to_np(li), eli) and np.array_equal(to_np(ri), eri)
