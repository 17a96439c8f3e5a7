"""Reduce-by-key over double values on the GPU: SUM against the exactly-rounded oracle (bit
for bit) and within the rounding bound of the reference's sequential sums; MIN bit for bit
against the reference's fold; the compat entries and shim symbols of Reduce.h."""
import numpy as np
import pytest

import oracle as O
from redfox_b200 import rfx as R
from redfox_b200 import workloads as WL

from helpers import to_np

pytestmark = pytest.mark.gpu


def gen_values(kind, n, seed):
    rng = np.random.default_rng(seed)
    if kind == "prices":       # decimal-like amounts
        return np.round(rng.uniform(900.0, 105000.0, n), 2) * rng.choice([1.0, -1.0], n, p=[0.9, 0.1])
    if kind == "mixed":        # 2^-40 .. 2^40, random signs and mantissas
        return rng.uniform(1.0, 2.0, n) * np.exp2(rng.integers(-40, 41, n)) * rng.choice([1.0, -1.0], n)
    if kind == "wide":         # the whole exponent range: needs the full-range accumulator
        m = rng.uniform(1.0, 2.0, n) * rng.choice([1.0, -1.0], n)
        return np.ldexp(m, rng.integers(-1070, 1000, n))
    if kind == "cancel":       # huge terms that cancel exactly around small ones
        x = rng.uniform(1.0, 2.0, n) * 1e15
        x[1::2] = -x[0::2][: n // 2]
        x[::7] = rng.uniform(-1.0, 1.0, x[::7].shape[0]) * 1e-3
        return x
    if kind == "ties":         # sums that land exactly half-way between doubles
        x = np.ones(n)
        x[::3] = 2.0 ** 53
        return x
    if kind == "subnormal":
        return rng.integers(-2**40, 2**40, n).astype(np.float64) * 5e-324
    if kind == "specials":
        x = rng.uniform(-10.0, 10.0, n)
        idx = rng.integers(0, n, max(1, n // 50))
        x[idx] = rng.choice([np.nan, np.inf, -np.inf, 0.0, -0.0], idx.shape[0])
        return x
    if kind == "zeros":
        return rng.choice([0.0, -0.0], n, p=[0.05, 0.95])
    raise KeyError(kind)


def gen_keys(kb, n, groups, seed):
    rng = np.random.default_rng(seed)
    g = np.sort(rng.integers(0, groups, n))
    if kb == 16:
        k = np.zeros((n, 2), np.uint64)
        k[:, 0] = g.astype(np.uint64) * np.uint64(0x9E3779B97F4A7C15)
        k[:, 1] = g.astype(np.uint64)
        return k.view(np.uint8).reshape(n, 16)
    dt = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[kb]
    if kb == 1:
        return (g % 256).astype(dt)
    return (g.astype(np.uint64) * np.uint64(2654435761)).astype(dt)


def _same_bits(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    both_nan = np.isnan(a) & np.isnan(b)
    return bool(np.all(both_nan | (a.view(np.uint64) == b.view(np.uint64))))


def _dev(x, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(cuda)


def _check_sum(cuda, keys, vals):
    dk = None if keys is None else _dev(keys, cuda)
    ok, ov, g = R.reduce_f64(dk, _dev(vals, cuda), R.F64_SUM)
    ek, es = O.reduce_f64_exact(keys, vals)
    assert g == es.shape[0]
    if keys is not None:
        assert np.array_equal(to_np(ok), ek)
    got = to_np(ov)
    assert _same_bits(got, es)
    # against the reference's own (sequential) order: within that order's rounding error
    _, seq = O.reduce_f64_seq(keys, vals)
    st = O.run_starts(keys, vals.shape[0])
    absum = np.add.reduceat(np.abs(np.where(np.isfinite(vals), vals, 0.0)), st) if st.size else st
    lens = np.diff(np.concatenate([st, [vals.shape[0]]]))
    fin = np.isfinite(seq) & np.isfinite(got)
    tol = lens * np.finfo(np.float64).eps * absum
    assert np.all(np.abs(got[fin] - seq[fin]) <= tol[fin])
    assert R.device_status() == R.OK


@pytest.mark.parametrize("kind", ["prices", "mixed", "wide", "cancel", "ties", "subnormal", "specials", "zeros"])
@pytest.mark.parametrize("groups", [3, 20000])
def test_sum_by_u32_key(cuda, kind, groups):
    n = 100_003
    _check_sum(cuda, gen_keys(4, n, groups, 7), gen_values(kind, n, 11))


@pytest.mark.parametrize("kb", [1, 2, 8, 16])
def test_sum_key_widths(cuda, kb):
    n = 50_000
    _check_sum(cuda, gen_keys(kb, n, 700, kb), gen_values("mixed", n, kb))


@pytest.mark.parametrize("n", [1, 5, 2047, 2048, 2049, 6145])
def test_sum_tile_edges(cuda, n):
    _check_sum(cuda, gen_keys(4, n, max(1, n // 300), n), gen_values("prices", n, n))
    _check_sum(cuda, gen_keys(4, n, n, n + 1), gen_values("mixed", n, n))


@pytest.mark.parametrize("kind", ["prices", "wide"])
def test_sum_one_run(cuda, kind):
    """No keys: the whole column is one run (total_double)."""
    n = 3_000_000 if kind == "prices" else 200_000
    _check_sum(cuda, None, gen_values(kind, n, 3))


def test_sum_few_groups_large(cuda):
    """A handful of runs spanning thousands of tiles each (the tile fix-up path)."""
    n = 8_000_000
    _check_sum(cuda, gen_keys(4, n, 4, 1), gen_values("prices", n, 2))


@pytest.mark.parametrize("kind", ["mixed", "specials", "zeros"])
@pytest.mark.parametrize("groups", [3, 20000])
def test_min_by_u32_key(cuda, kind, groups):
    n = 100_003
    keys = gen_keys(4, n, groups, 5)
    vals = gen_values(kind, n, 6)
    ok, ov, g = R.reduce_f64(_dev(keys, cuda), _dev(vals, cuda), R.F64_MIN)
    ek, ev = O.reduce_f64_seq(keys, vals, op_min=True)
    assert g == ev.shape[0] and np.array_equal(to_np(ok), ek)
    assert np.array_equal(to_np(ov).view(np.uint64), ev.view(np.uint64))   # NaN payloads too


def test_min_nan_and_zero_order(cuda):
    """The fold's order rules: a later equal zero wins, a NaN is replaced by the next value,
    a trailing NaN stays."""
    nan2 = np.frombuffer(np.uint64(0x7ff8000000000123).tobytes(), np.float64)[0]
    vals = np.array([-0.0, 0.0, 5.0, np.nan, 7.0, 3.0, 1.0, nan2, 0.0, -0.0, 2.0, nan2], np.float64)
    keys = np.array([0, 0, 0, 1, 1, 1, 2, 2, 3, 3, 4, 4], np.uint32)
    ok, ov, g = R.reduce_f64(_dev(keys, cuda), _dev(vals, cuda), R.F64_MIN)
    ek, ev = O.reduce_f64_seq(keys, vals, op_min=True)
    assert np.array_equal(to_np(ov).view(np.uint64), ev.view(np.uint64))
    assert ev.view(np.uint64)[0] == np.float64(0.0).view(np.uint64)   # +0 after -0
    assert ev[1] == 3.0 and ev.view(np.uint64)[4] == np.uint64(0x7ff8000000000123)


def test_compat_entries_and_shims(cuda):
    import torch
    from test_shim import _fn, P
    n = 40_000
    keys = gen_keys(8, n, 900, 3).view(np.int64)
    vals = gen_values("mixed", n, 4)
    dk, dv = _dev(keys, cuda), _dev(vals, cuda)
    ok = torch.empty(n, dtype=torch.int64, device=cuda)
    ov = torch.empty(n, dtype=torch.float64, device=cuda)
    ks = torch.tensor([8 * n], dtype=torch.int64, device=cuda)
    vs = torch.tensor([8 * n], dtype=torch.int64, device=cuda)
    torch.cuda.synchronize()
    _fn("ra", "redfox::total_64_double(void const*, void const*, void*, void*, unsigned long long*, "
              "unsigned long long*)", [P] * 6)(dk.data_ptr(), dv.data_ptr(), ok.data_ptr(), ov.data_ptr(),
                                               ks.data_ptr(), vs.data_ptr())
    ek, es = O.reduce_f64_exact(keys, vals)
    g = int(ks.item()) // 8
    assert g == es.shape[0] and int(vs.item()) // 8 == g
    assert np.array_equal(to_np(ok[:g]), ek) and _same_bits(to_np(ov[:g]), es)
    # min_32_double
    k32 = gen_keys(4, n, 900, 5)
    dk32 = _dev(k32, cuda)
    ok32 = torch.empty(n, dtype=torch.int32, device=cuda)
    ks.fill_(4 * n)
    vs.fill_(8 * n)
    torch.cuda.synchronize()
    _fn("ra", "redfox::min_32_double(void const*, void const*, void*, void*, unsigned long long*, "
              "unsigned long long*)", [P] * 6)(dk32.data_ptr(), dv.data_ptr(), ok32.data_ptr(), ov.data_ptr(),
                                               ks.data_ptr(), vs.data_ptr())
    ek, ev = O.reduce_f64_seq(k32, vals, op_min=True)
    g = int(ks.item()) // 4
    assert g == ev.shape[0] and np.array_equal(to_np(ok32[:g]).view(np.uint32), ek)
    assert np.array_equal(to_np(ov[:g]).view(np.uint64), ev.view(np.uint64))
    # total_double, max_double, count
    res = torch.zeros(1, dtype=torch.float64, device=cuda)
    torch.cuda.synchronize()
    _fn("ra", "redfox::total_double(void*, void const*, void const*)", [P] * 3)(
        res.data_ptr(), dv.data_ptr(), dv.data_ptr() + 8 * n)
    assert _same_bits(to_np(res), [O.exact_sum(vals)])
    mx = torch.zeros(1, dtype=torch.int64, device=cuda)
    _fn("ra", "redfox::max_double(void*, void const*, void const*)", [P] * 3)(
        mx.data_ptr(), dv.data_ptr(), dv.data_ptr() + 8 * n)
    assert to_np(mx).view(np.uint64)[0] == vals.view(np.uint64).max()
    u = np.random.default_rng(9).integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    du = _dev(u.view(np.int32), cuda)
    cnt = torch.zeros(1, dtype=torch.int32, device=cuda)
    _fn("ra", "redfox::count(void*, void const*, void const*)", [P] * 3)(
        cnt.data_ptr(), du.data_ptr(), du.data_ptr() + 4 * n)
    assert int(to_np(cnt).view(np.uint32)[0]) == int(u.astype(np.uint64).sum() % 2**32)
    assert R.device_status() == R.OK


def test_total_string_double(cuda):
    import torch
    pool, offs = WL.gen_strings(30000, seed=8, distinct=3000)
    offs = O.str_sort(pool, offs)
    vals = gen_values("prices", offs.shape[0], 8)
    dpool, ptrs = R.string_column(pool, offs, cuda)
    dv = _dev(vals, cuda)
    n = offs.shape[0]
    ok = torch.empty(n, dtype=torch.int64, device=cuda)
    ov = torch.empty(n, dtype=torch.float64, device=cuda)
    ks = torch.tensor([8 * n], dtype=torch.int64, device=cuda)
    vs = torch.tensor([8 * n], dtype=torch.int64, device=cuda)
    R.check("rfx_total_string_double_compat",
            R.LIB.rfx_total_string_double_compat(R._ptr(ptrs), R._ptr(dv), R._ptr(ok), R._ptr(ov), R._ptr(ks),
                                                 R._ptr(vs)))
    # the oracle: runs of equal strings (string codes as keys), first offset of each run
    codes, _ = O.str_codes(pool, offs)
    _, es = O.reduce_f64_exact(codes, vals)
    eo, _ = O.str_count(pool, offs, np.zeros(n, np.uint32))
    g = int(ks.item()) // 8
    assert g == es.shape[0] and int(vs.item()) // 8 == g
    assert np.array_equal((to_np(ok[:g]) - dpool.data_ptr()).astype(np.uint64), eo)
    assert _same_bits(to_np(ov[:g]), es)
