"""The oracle pinned against the reference: golden fixtures made by the reference's own
code (tests/golden/make_golden.py) and the reference's known-answer tests.  CPU only."""
import os

import numpy as np
import pytest

import oracle as O

from helpers import fact_oracle, fact_rows_oracle

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLD, name))


def test_tpch_fixture_A_packing():
    """TPC-H/data/A = TC.tbl rows (1,6)..(5,10) packed as Tuple<32,32> (field 0 high)."""
    raw = np.fromfile(os.path.join(GOLD, "tpch_A.bin"), dtype=np.uint8).reshape(5, 8)
    cols = [np.arange(1, 6, dtype=np.uint64), np.arange(6, 11, dtype=np.uint64)]
    assert np.array_equal(O.pack([32, 32], cols), raw)
    back = O.unpack([32, 32], raw)
    assert np.array_equal(back[0], cols[0]) and np.array_equal(back[1], cols[1])
    assert raw.view("<u8")[0, 0] == 0x0000000100000006


def test_tuple_packing_matches_reference_insert():
    g = load("tuple_pack.npz")
    names = sorted({k.rsplit("_", 1)[0] for k in g.files})
    assert len(names) >= 10
    for name in names:
        widths = [int(w) for w in g[name + "_widths"]]
        cols = list(g[name + "_cols"])
        ref = g[name + "_bytes"]
        assert np.array_equal(O.pack(widths, cols), ref), name
        for a, b in zip(O.unpack(widths, ref), cols):
            assert np.array_equal(a, b), name


def _setcases(g):
    return sorted({k.rsplit("_", 1)[0] for k in g.files if k.endswith("_a")})


def test_set_union_difference_match_reference():
    g = load("setops.npz")
    for key in _setcases(g):
        a, b = g[key + "_a"], g[key + "_b"]
        assert np.array_equal(O.set_union(a, b), g[key + "_union"]), key
        assert np.array_equal(O.set_difference(a, b), g[key + "_difference"]), key
        if key + "_intersection" in g.files:
            assert np.array_equal(O.set_intersection(a, b), g[key + "_intersection"]), key
        if key + "_unique" in g.files:
            assert np.array_equal(O.unique(a), g[key + "_unique"]), key


def test_reduce_count_match_reference():
    g = load("reduce.npz")
    for e in (1, 2, 4, 16):
        ok, oc = O.reduce_count(g["count%d_keys" % e], g["count%d_vals" % e])
        assert np.array_equal(ok, g["count%d_okeys" % e]) and np.array_equal(oc, g["count%d_ocounts" % e]), e
    # total_64_32: u64 keys, u32 sums; the oracle's int64 sums agree modulo 2^32
    ok, os_ = O.reduce_sum_i64(g["total64_32_keys"], g["total64_32_vals"].astype(np.int64))
    assert np.array_equal(ok, g["total64_32_okeys"])
    assert np.array_equal(os_.astype(np.uint64) & np.uint64(0xffffffff), g["total64_32_osums"].astype(np.uint64))
    ok, os_ = O.reduce_sum_i64(g["sum_i64_keys"], g["sum_i64_vals"])
    assert np.array_equal(ok, g["sum_i64_okeys"]) and np.array_equal(os_, g["sum_i64_osums"])


def test_sort_matches_reference():
    g = load("sort.npz")
    for e in (1, 2, 4, 8):
        assert np.array_equal(O.sort_pairs(g["e%d_in" % e]), g["e%d_out" % e]), e


def _same_bits(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return bool(np.all((np.isnan(a) & np.isnan(b)) | (a.view(np.uint64) == b.view(np.uint64))))


def test_f64_reduces_match_reference():
    """The sequential folds of the oracle reproduce redfox::total_*_double, min_32_double,
    total_double, max_double and count (Reduce.cu) bit for bit; the exact sums the GPU
    computes lie within the sequential sums' rounding error."""
    g = load("f64.npz")
    vals = g["vals"]
    for kb in (1, 2, 4, 8, 16):
        ok, ov = O.reduce_f64_seq(g["k%d" % kb], vals)
        assert np.array_equal(ok, g["k%d_okeys" % kb]) and _same_bits(ov, g["k%d_sums" % kb]), kb
        ek, es = O.reduce_f64_exact(g["k%d" % kb], vals)
        assert np.array_equal(ek, ok)
        fin = np.isfinite(ov)
        assert np.all(np.abs(es[fin] - ov[fin]) <= 1e-12 * np.maximum(np.abs(ov[fin]), 1.0))
        assert np.array_equal(np.isnan(es), np.isnan(ov))
    ok, ov = O.reduce_f64_seq(g["k4"], vals, op_min=True)
    assert np.array_equal(ok, g["k4_min_okeys"]) and np.array_equal(ov.view(np.uint64), g["k4_mins"].view(np.uint64))
    fin = vals[np.isfinite(vals)]
    _, tot = O.reduce_f64_seq(None, fin)
    assert _same_bits(tot, g["total"])
    assert vals.view(np.uint64).max() == g["max_bits"][0]
    assert int(g["u32"].astype(np.uint64).sum() % 2**32) == int(g["count"][0])


def test_exact_sum_known_answers():
    assert O.exact_sum([1e16, 1.0]) == 1e16                    # tie -> even
    assert O.exact_sum([1e16, 1.0, 1.0]) == 1e16 + 2.0
    assert O.exact_sum([1e308, 1e308, -1e308]) == 1e308        # no intermediate overflow
    assert np.signbit(O.exact_sum([-0.0, -0.0])) and not np.signbit(O.exact_sum([-0.0, 0.0]))
    assert np.isnan(O.exact_sum([np.inf, -np.inf])) and O.exact_sum([np.inf, 1.0]) == np.inf


def test_strings_match_reference():
    """redfox::sort_string (Sort.cu) and redfox::count_string (Reduce.cu) on a column with
    empty strings, proper prefixes, bytes >= 0x80 and long shared prefixes."""
    g = load("strings.npz")
    pool, offs = g["pool"], g["offs"]
    assert np.array_equal(O.str_sort(pool, offs), g["sorted"])
    for name, col in (("count_sorted", g["sorted"]), ("count_unsorted", offs)):
        ko, ks = O.str_count(pool, col, g["vals"])
        assert np.array_equal(ko, g[name + "_offs"]) and np.array_equal(ks, g[name + "_sums"]), name


def test_string_order_known_answers():
    """Signed-char order, a proper prefix first, equality by content."""
    pool, offs = O.str_pool([b"b", b"", b"ab", b"a", b"\x80", b"\x7f", b"ab\xff", b"ab"])
    order = O.str_sort(pool, offs)
    text = [bytes(pool[o:pool.tolist().index(0, int(o))]) for o in order]
    assert text == [b"", b"\x80", b"a", b"ab", b"ab", b"ab\xff", b"b", b"\x7f"]
    assert order[3] < order[4]   # equal strings keep their input order
    ko, ks = O.str_count(pool, order, np.ones(8, np.uint32))
    assert ks.tolist() == [1, 1, 1, 2, 1, 1, 1]


def test_fact_plan_matches_reference_composition():
    g = load("fact_plan.npz")
    rows = fact_rows_oracle(int(g["n"][0]))
    keys, sums, counts = fact_oracle(rows)
    assert np.array_equal(keys, g["keys"])
    assert np.array_equal(sums[:, 0], g["s1"]) and np.array_equal(sums[:, 1], g["s2"])
    assert np.array_equal(counts, g["counts"])


def test_testjoin_identity_self_join():
    """TestJoin.cu:107-156: self-join of 2^15 ushort keys 0..32767 yields (i << 16) | i."""
    n = 1 << 15
    keys = np.arange(n, dtype=np.uint16)
    lb, scan, total = O.find_bounds(keys, keys)
    assert total == n
    li, ri = O.join_expand(lb, scan, total)
    out = O.join_gather(4, li, ri, keys, None, 0, keys, 16).view(np.uint32).ravel()
    assert np.array_equal(out, (np.arange(n, dtype=np.uint32) << 16) | np.arange(n, dtype=np.uint32))


def _cpujoin(a, b):
    """moderngpu CPUJoin (tests/benchmarkjoin.cu:40-128), inner join, as a literal loop."""
    a_lb = np.searchsorted(b, a, side="left")
    a_ub = np.searchsorted(b, a, side="right")
    counts = a_ub - a_lb
    scan = np.concatenate([[0], np.cumsum(counts)[:-1]]) if len(a) else np.zeros(0, np.int64)
    total = int(counts.sum())
    ai, bi = np.zeros(total, np.int32), np.zeros(total, np.int32)
    a_index = b_index = 0
    while a_index < total:
        p = True if b_index >= len(a) else a_index < scan[b_index]
        if not p:
            b_index += 1
            continue
        src = b_index - 1
        ai[a_index] = src
        bi[a_index] = a_lb[src] + (a_index - scan[src])
        a_index += 1
    return ai, bi


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_join_order_matches_cpujoin(seed):
    rng = np.random.default_rng(seed)
    a = np.sort(rng.integers(0, 300, 500)).astype(np.uint32)
    b = np.sort(rng.integers(0, 300, 400)).astype(np.uint32)
    lb, scan, total = O.find_bounds(a, b)
    li, ri = O.join_expand(lb, scan, total)
    ai, bi = _cpujoin(a, b)
    assert np.array_equal(li, ai) and np.array_equal(ri, bi)


def test_generators_are_counter_based():
    a = O.uniform(1000, 7, 3, 10, 20)
    b = O.uniform(2000, 7, 3, 10, 20)
    assert np.array_equal(a, b[:1000]) and a.min() >= 10 and a.max() < 20


@pytest.mark.skipif(O.ref_lib() is None, reason="reference code not built here")
def test_oracle_against_reference_code_random():
    """Fresh random cases straight through the reference's compiled entry files."""
    import ctypes as C
    ref = O.ref_lib()
    ref.ref_set_union.restype = C.c_uint64
    ref.ref_difference.restype = C.c_uint64
    rng = np.random.default_rng(99)
    for _ in range(20):
        a = np.sort(rng.integers(0, 1000, rng.integers(0, 3000))).astype(np.uint64)
        b = np.sort(rng.integers(0, 1000, rng.integers(0, 3000))).astype(np.uint64)
        out = np.zeros(len(a) + len(b) + 1, np.uint64)
        k = ref.ref_set_union(out.ctypes.data_as(C.c_void_p), a.ctypes.data_as(C.c_void_p), C.c_size_t(len(a)),
                              b.ctypes.data_as(C.c_void_p), C.c_size_t(len(b)), 8, 4)
        assert np.array_equal(O.set_union(a, b), out[:k])
        k = ref.ref_difference(out.ctypes.data_as(C.c_void_p), a.ctypes.data_as(C.c_void_p), C.c_size_t(len(a)),
                               b.ctypes.data_as(C.c_void_p), C.c_size_t(len(b)), 8, 4)
        assert np.array_equal(O.set_difference(a, b), out[:k])
