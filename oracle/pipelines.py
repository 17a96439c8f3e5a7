"""The benchmark plans restated on the CPU with the oracle's operators -- TEST
INFRASTRUCTURE ONLY (the checker for the GPU plans, and the CPU legs of bench.py).

Both follow the reference's query plans as the RA operators run them: sort both sides on
their keys (b40cSort.cu / ModernGPUSort.cu), join (ModernGPUJoin.cu: find_bounds, expansion,
gather), and reduce-by-key SUM + COUNT (Reduce.cu); the three-relation plan adds selects
(Select.h), projects (Project.h) and the set operations (Union.cu / Difference.cu, and the
STL intersection).  `threads` goes to the sorts (the oracle's only multi-threaded step).
"""
import numpy as np

from . import binding as O


def join_aggregate_plan(r, s, threads=1):
    """R = Tuple<32 key, 32 payload> rows, S = Tuple<32 key, 64 amount> rows: join on the
    key, SUM(amount) and COUNT per key.  Returns (keys u32, sums i64, counts, join rows)."""
    rs = O.sort_pairs(r, begin_bit=32, end_bit=64, threads=threads)
    ss = O.sort_pairs(s, begin_bit=64, end_bit=96, threads=threads)
    out = O.join_tuples(rs, 32, ss, 64, 16)
    limbs = out.view(np.uint64)
    key = (limbs[:, 1] >> np.uint64(32)).astype(np.uint32)
    amt = limbs[:, 0].astype(np.int64)
    k, sums = O.reduce_sum_i64(key, amt)
    _, counts = O.reduce_count(key)
    return k, sums, counts, len(out)


def three_relation_plan(d1, d2, f, list_in, list_out, segment, date_lo, date_hi, threads=1):
    """D1 = (pk, segment), D2 = (pk, fk, date), F = (fk, amount): D1 on the segment, D2 on
    the date range, D2's (fk, pk) sorted on fk, joined to D1; the D2 keys sorted, kept in
    list_in and not in list_out; F sorted on its fk and joined; SUM(amount) and COUNT per
    D2 key.  Returns (keys u32, sums i64, counts)."""
    def cmp(op, field, const, vtype):
        return {"op": op, "a": (O.OPND_VAR, field), "b": (O.OPND_CONST, const), "type": vtype}
    d1s = O.select(d1, [32, 8], [cmp(O.EQ, 1, segment, O.I8)])
    d2f = O.select(d2, [32, 32, 32], [cmp(O.GE, 2, date_lo, O.I32), cmp(O.LT, 2, date_hi, O.I32)])
    d2s = O.project(d2f, [32, 32, 32], [32, 32], [1, 0])
    d2s = O.sort_pairs(d2s, begin_bit=32, end_bit=64, threads=threads)
    j1 = O.join_tuples(d1s, 8, d2s, 32, 16)
    keys = O.project(j1, [32, 8, 32], [32], [2]).view(np.uint32).ravel()
    keys = O.sort_pairs(keys, threads=threads)
    keys = O.set_difference(O.set_intersection(keys, list_in), list_out)
    fs = O.sort_pairs(f, begin_bit=64, end_bit=96, threads=threads)
    j2 = O.join_tuples(keys.view(np.uint8).reshape(-1, 4), 0, fs, 64, 16)
    limbs = j2.view(np.uint64)
    key = limbs[:, 1].astype(np.uint32)
    amt = limbs[:, 0].astype(np.int64)
    k, sums = O.reduce_sum_i64(key, amt)
    _, counts = O.reduce_count(key)
    return k, sums, counts
