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


def test_find_bounds_window_forms(cuda):
    """The right-key window of each left tile: a window far larger than shared memory (few
    left keys against millions of right keys: global-memory searches), a tiny right side
    (the smallest window), and left keys wider than the 4-byte right keys (those above
    2^32 match nothing)."""
    rng = np.random.default_rng(31)
    for nl, nr, hi in ((3000, 2_000_000, 1000), (2_000_000, 3000, 5000)):
        left = np.sort(rng.integers(0, hi, nl)).astype(np.uint32)
        right = np.sort(rng.integers(0, hi, nr)).astype(np.uint32)
        lb, sc, total = R.find_bounds(_dev(left, cuda), _dev(right, cuda))
        elb, esc, etot = O.find_bounds(left, right)
        assert total == etot
        assert np.array_equal(to_np(lb), elb) and np.array_equal(to_np(sc), esc)
    nl, nr = 40000, 60000
    lk = np.sort(np.concatenate([rng.integers(0, 1 << 20, nl // 2), rng.integers(1 << 24, 1 << 34, nl // 4),
                                 rng.integers(1 << 38, 1 << 40, nl - nl // 2 - nl // 4)])).astype(np.uint64)
    rk = np.sort(rng.integers(0, 1 << 20, nr)).astype(np.uint64)
    left = O.pack([40, 24], [lk, rng.integers(0, 1 << 24, nl, dtype=np.uint64)])
    right = O.pack([24, 8], [rk, rng.integers(0, 256, nr, dtype=np.uint64)])
    assert left.shape[1] == 8 and right.shape[1] == 4
    got, total = R.join_tuples(_dev(left, cuda), 24, _dev(right, cuda), 8, 8)
    exp = O.join_tuples(left, 24, right, 8, 8)
    assert total == len(exp) > 0
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


def _join_agg_oracle(left, right):
    """join_tuples of R = Tuple<32,32> and S = Tuple<32,64> (output (key, payload, amount),
    key in bits 96..127), then SUM(amount) and COUNT per key, on the oracle."""
    out = O.join_tuples(left, 32, right, 64, 16)
    if len(out) == 0:
        return np.zeros(0, np.uint32), np.zeros(0, np.int64), np.zeros(0, np.uint32)
    limbs = out.view(np.uint64)
    keys = (limbs[:, 1] >> np.uint64(32)).astype(np.uint32)
    vals = limbs[:, 0].astype(np.int64)
    k, sums = O.reduce_sum_i64(keys, vals)
    _, counts = O.reduce_count(keys)
    return k, sums, counts


@pytest.mark.parametrize("nr,ns,dom,extra", [(0, 100, 10, 0), (100, 0, 10, 0), (1, 1, 1, 0), (1000, 4000, 256, 0),
                                             (50_000, 200_000, 12_500, 0), (20_000, 300_000, 40_000, 5_000),
                                             (3_000, 500_000, 2_000, 0)])
def test_join_aggregate_equals_join_then_reduce(cuda, nr, ns, dom, extra):
    """rfx_join_aggregate == rfx_join_tuples + rfx_reduce_tuples == the oracle, including
    right keys with no left match (`extra` rows with keys outside R's domain), left keys
    with no right match, heavy duplication on both sides, and empty inputs."""
    import torch
    rng = np.random.default_rng(nr + 7 * ns)
    rk = np.sort(rng.integers(0, dom, nr)).astype(np.uint64)
    r = O.pack([32, 32], [rk, rng.integers(0, 2**32, nr).astype(np.uint64)])
    sk = np.concatenate([rng.integers(0, dom, ns - extra), rng.integers(dom, 2 * dom, extra)]).astype(np.uint64)
    s = O.pack([32, 64], [np.sort(sk), rng.integers(100, 10**7, ns).astype(np.uint64)])
    rd, sd = _dev(r, cuda), _dev(s, cuda)
    keys, sums, counts = R.join_aggregate(rd, 32, sd, 64, 0, 64, 4)
    ek, es, ec = _join_agg_oracle(r, s) if nr and ns else (np.zeros(0, np.uint32),) * 3
    assert np.array_equal(to_np(keys).view(np.uint32), ek)
    assert np.array_equal(to_np(sums), np.asarray(es, np.int64))
    assert np.array_equal(to_np(counts).view(np.uint32), np.asarray(ec, np.uint32))
    if nr and ns:
        out, total = R.join_tuples_two_step(rd, 32, sd, 64, 16)
        gk, gs, gc, _ = R.reduce_tuples(out, 96, 0, 64, 4, n=total)
        assert torch.equal(gk, keys) and torch.equal(gs, sums) and torch.equal(gc, counts)


def test_join_aggregate_skewed_key(cuda):
    """One key with 300K right rows and 2K left rows: its count (6e8) and its sum wrap
    exactly like the 6e8 join rows would (checked against the closed form)."""
    nr, ns = 2_000, 300_000
    rng = np.random.default_rng(3)
    r = O.pack([32, 32], [np.full(nr, 7, np.uint64), np.arange(nr, dtype=np.uint64)])
    amounts = rng.integers(100, 10**7, ns).astype(np.uint64)
    s = O.pack([32, 64], [np.full(ns, 7, np.uint64), amounts])
    keys, sums, counts = R.join_aggregate(_dev(r, cuda), 32, _dev(s, cuda), 64, 0, 64, 4)
    assert to_np(keys).view(np.uint32).tolist() == [7]
    exp_sum = (int(amounts.astype(object).sum()) * nr) % (1 << 64)
    assert int(to_np(sums).view(np.uint64)[0]) == exp_sum
    assert int(to_np(counts).view(np.uint32)[0]) == (nr * ns) % (1 << 32)


@pytest.mark.parametrize("variant", [0, 1])
def test_join_emit_variants(cuda, variant):
    """Both emit kernels (pinned through the tuner) on the shapes that exercise the staged
    one's paths: many outputs per left row (the right window in shared memory), rows with
    one output each (more left rows per tile than the stage holds: per-output search),
    a skewed key whose right run is larger than the staged window, 4-byte rows (plain
    copies instead of bulk copies), unaligned relation bases, and a capacity cut."""
    import torch
    try:
        R.tune_force(R.TUNE_JOIN_EMIT, variant)
        rng = np.random.default_rng(11)
        cases = []
        # duplicate keys on both sides (the benchmark's shape, smaller)
        lk = np.sort(rng.integers(0, 5000, 40000)).astype(np.uint64)
        rk = np.sort(rng.integers(0, 5000, 160000)).astype(np.uint64)
        cases.append((O.pack([32, 32], [lk, rng.integers(0, 2**32, 40000, dtype=np.uint64)]), 32,
                      O.pack([32, 64], [rk, rng.integers(0, 2**40, 160000, dtype=np.uint64)]), 64, 16))
        # one match per left row, sparse keys
        ku = np.arange(0, 300000, 3, dtype=np.uint64)
        cases.append((O.pack([32, 32], [ku, ku]), 32, O.pack([32, 32], [ku, ku + 1]), 32, 8))
        # a skewed key: 3 left rows x 50000 right rows, then ordinary keys
        lk = np.concatenate([np.full(3, 5, np.uint64), np.arange(6, 3000, dtype=np.uint64)])
        rk = np.concatenate([np.full(50000, 5, np.uint64), np.repeat(np.arange(6, 3000, dtype=np.uint64), 2)])
        cases.append((O.pack([32, 32], [lk, np.arange(len(lk), dtype=np.uint64)]), 32,
                      O.pack([32, 64], [rk, np.arange(len(rk), dtype=np.uint64)]), 64, 16))
        # 4-byte rows on both sides
        lk = np.sort(rng.integers(0, 2000, 20000)).astype(np.uint64)
        rk = np.sort(rng.integers(0, 2000, 30000)).astype(np.uint64)
        cases.append((O.pack([24, 8], [lk, lk & np.uint64(0xff)]), 8, O.pack([24, 8], [rk, rk & np.uint64(0x7f)]), 8,
                      8))
        for left, lvb, right, rvb, ob in cases:
            exp = O.join_tuples(left, lvb, right, rvb, ob)
            got, total = R.join_tuples(_dev(left, cuda), lvb, _dev(right, cuda), rvb, ob)
            assert total == len(exp) and np.array_equal(to_np(got), exp)
            # bases 1 row into their allocations (not 16-byte aligned for 8- and 4-byte rows)
            dl = _dev(np.concatenate([left[:1], left]), cuda)[1:]
            dr = _dev(np.concatenate([right[:1], right]), cuda)[1:]
            got, total = R.join_tuples(dl, lvb, dr, rvb, ob)
            assert total == len(exp) and np.array_equal(to_np(got), exp)
            part, _ = R.join_tuples(_dev(left, cuda), lvb, _dev(right, cuda), rvb, ob, capacity=len(exp) // 2 + 7)
            assert np.array_equal(to_np(part), exp[:len(exp) // 2 + 7])
        torch.cuda.synchronize()
        assert R.device_status() == R.OK
    finally:
        R.tune_force(R.TUNE_JOIN_EMIT, -1)
