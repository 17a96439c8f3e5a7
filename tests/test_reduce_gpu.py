"""Reduce-by-key / count against the oracle and the reference's golden vectors."""
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


def _sorted_keys(n, kb, distinct, seed):
    rng = np.random.default_rng(seed)
    ks = np.sort(rng.integers(0, max(1, distinct), n)).astype(np.uint64)
    # the run id's bytes repeat across the container so every limb takes part in equality
    a = np.zeros((n, kb), np.uint8)
    for b in range(kb):
        a[:, b] = (ks >> np.uint64(8 * (b % 8))) & np.uint64(0xff)
    return a


@pytest.mark.parametrize("kb", [1, 2, 4, 8, 16, 32])
@pytest.mark.parametrize("n,distinct", [(0, 1), (1, 1), (2047, 100), (2048, 2048), (2049, 1), (100003, 5000),
                                        (300000, 299999)])
def test_reduce_sum_i64_and_count(cuda, kb, n, distinct):
    keys = _sorted_keys(n, kb, min(distinct, 2 ** (8 * kb)), seed=n + kb)
    vals = np.random.default_rng(n).integers(-2**62, 2**62, n).astype(np.int64)
    ok, ov, oc, g = R.reduce_by_key(_dev(keys, cuda), _dev(vals, cuda))
    ek, ev = O.reduce_sum_i64(keys, vals)
    _, ec = O.reduce_count(keys)
    assert g == len(ek)
    assert np.array_equal(to_np(ok), ek)
    assert np.array_equal(to_np(ov), ev)
    assert np.array_equal(to_np(oc).astype(np.uint32), ec)
    assert R.device_status() == R.OK


@pytest.mark.parametrize("kb", [1, 4, 16])
def test_reduce_u32_column(cuda, kb):
    n = 77777
    keys = _sorted_keys(n, kb, 300, seed=kb)
    vals = np.random.default_rng(1).integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    ok, ov, oc, g = R.reduce_by_key(_dev(keys, cuda), _dev(vals.view(np.int32), cuda), value_kind=R.VAL_U32)
    ek, ec = O.reduce_count(keys, vals)
    assert np.array_equal(to_np(ok), ek)
    assert np.array_equal(to_np(ov).view(np.uint32), ec)


def test_reduce_device_count(cuda):
    import torch
    n = 50000
    keys = _sorted_keys(n, 4, 999, seed=3)
    vals = np.arange(n, dtype=np.int64)
    dn = torch.tensor([31337], dtype=torch.int64, device=cuda)
    ok, ov, oc, g = R.reduce_by_key(_dev(keys, cuda), _dev(vals, cuda), d_n=dn)
    ek, ev = O.reduce_sum_i64(keys[:31337], vals[:31337])
    assert np.array_equal(to_np(ok), ek) and np.array_equal(to_np(ov), ev)


def test_count_compat_matches_reference_golden(cuda):
    import torch
    g = np.load(os.path.join(GOLD, "reduce.npz"))
    for e in (1, 2, 4, 16):
        keys, vals = g["count%d_keys" % e], g["count%d_vals" % e]
        n = keys.shape[0]
        dk, dv = _dev(keys, cuda), _dev(vals, cuda)
        ok = torch.zeros_like(dk)
        ov = torch.zeros_like(dv)
        ks = torch.tensor([n * e], dtype=torch.int64, device=cuda)
        vs = torch.tensor([n * 4], dtype=torch.int64, device=cuda)
        torch.cuda.synchronize()
        st = R.LIB.rfx_count_compat(C.c_void_p(dk.data_ptr()), C.c_void_p(dv.data_ptr()), C.c_void_p(ok.data_ptr()),
                                    C.c_void_p(ov.data_ptr()), C.c_void_p(ks.data_ptr()), C.c_void_p(vs.data_ptr()), e)
        assert st == R.OK
        groups = int(ks.item()) // e
        assert int(vs.item()) == groups * 4
        assert np.array_equal(to_np(ok)[:groups], g["count%d_okeys" % e])
        assert np.array_equal(to_np(ov)[:groups], g["count%d_ocounts" % e])
    keys, vals = g["total64_32_keys"], g["total64_32_vals"]
    n = len(keys)
    dk, dv = _dev(keys, cuda), _dev(vals, cuda)
    ok, ov = torch.zeros_like(dk), torch.zeros_like(dv)
    ks = torch.tensor([n * 8], dtype=torch.int64, device=cuda)
    vs = torch.tensor([n * 4], dtype=torch.int64, device=cuda)
    torch.cuda.synchronize()
    assert R.LIB.rfx_total_64_32_compat(C.c_void_p(dk.data_ptr()), C.c_void_p(dv.data_ptr()), C.c_void_p(ok.data_ptr()),
                                        C.c_void_p(ov.data_ptr()), C.c_void_p(ks.data_ptr()),
                                        C.c_void_p(vs.data_ptr())) == R.OK
    groups = int(ks.item()) // 8
    assert np.array_equal(to_np(ok)[:groups], g["total64_32_okeys"])
    assert np.array_equal(to_np(ov)[:groups], g["total64_32_osums"])


def test_large_reduce_properties(cuda):
    """8M rows: group sums add up to the total and counts to n (size-independent checks)."""
    import torch
    n = 8_000_000
    keys = torch.sort(torch.randint(0, 100000, (n,), dtype=torch.int64, device=cuda)).values.to(torch.int32)
    vals = torch.randint(-10**9, 10**9, (n,), dtype=torch.int64, device=cuda)
    ok, ov, oc, g = R.reduce_by_key(keys, vals)
    assert int(ov.sum()) == int(vals.sum())
    assert int(oc.to(torch.int64).sum()) == n
    assert torch.equal(ok, torch.unique_consecutive(keys))
