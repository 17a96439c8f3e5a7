"""Shared test helpers: the oracle form of the workloads and small utilities."""
import os

import numpy as np

import oracle as O
from redfox_b200 import workloads as WL


def fact_rows_oracle(n):
    cols = [O.uniform(n, WL.FACT_SEED, f, WL.FACT_LO[f], WL.FACT_HI[f]) for f in range(7)]
    return O.pack(WL.FACT_WIDTHS, cols)


def oracle_cmps(cmps):
    """rfx-style (op, (kind, v), (kind, v), type) -> oracle dicts."""
    return [{"op": op, "a": a, "b": b, "type": vt} for (op, a, b, vt) in cmps]


def oracle_arith(expr):
    nodes = [(expr.nodes[i].kind, expr.nodes[i].op, expr.nodes[i].type, expr.nodes[i].left,
              expr.nodes[i].right, expr.nodes[i].value) for i in range(expr.nnodes)]
    return O.make_arith(nodes, expr.root, expr.dest_type, expr.dest_bits)


def fact_oracle(rows):
    return O.filter_aggregate(rows, WL.FACT_WIDTHS, oracle_cmps(WL.fact_predicate()),
                              [oracle_arith(a) for a in WL.fact_ariths()], WL.FACT_GROUP_FIELDS,
                              WL.FACT_SUM_FIELDS)


# host threads for the oracle's parallel sort (its order does not depend on the count)
THREADS = os.cpu_count() or 1


def to_np(t):
    return t.detach().cpu().numpy()


# ---------------------------------------------------------------- plan restatements (oracle)
def join_aggregate_oracle_data(nr, ns, key_domain):
    from redfox_b200 import plans as PL
    key = O.uniform(nr, PL.C0_SEED, 0, 0, key_domain)
    pay = O.uniform(nr, PL.C0_SEED, 1, 0, 1 << 32)
    idx = O.uniform(ns, PL.C0_S_SEED, 0, 0, nr)
    amt = O.uniform(ns, PL.C0_S_SEED, 1, 100, 10_000_000)
    return O.pack([32, 32], [key, pay]), O.pack([32, 64], [key[idx.astype(np.int64)], amt])


def join_aggregate_oracle(r, s):
    from oracle import pipelines as OP
    return OP.join_aggregate_plan(r, s, threads=THREADS)


def three_relation_oracle_data(n1, n2, n3, l5, l2):
    from redfox_b200 import plans as PL
    seg = O.uniform(n1, PL.C2_SEED, 0, 0, 5)
    d1 = O.pack([32, 8], [np.arange(n1, dtype=np.uint64), seg])
    fk = O.zipf(n2, PL.C2_SEED + 1, 0, n1)
    date = O.uniform(n2, PL.C2_SEED + 5, 0, 0, 2526)
    d2 = O.pack([32, 32, 32], [np.arange(n2, dtype=np.uint64), fk, date])
    fcols = [O.uniform(n3, PL.C2_SEED + 2, 0, 0, n2), O.uniform(n3, PL.C2_SEED + 2, 1, 100, 10_000_000)]
    f = O.pack([32, 64], fcols)
    lists = []
    for cnt, seed in ((l5, PL.C2_SEED + 3), (l2, PL.C2_SEED + 4)):
        raw = O.uniform(cnt, seed, 0, 0, n2).astype(np.uint32)
        lists.append(O.unique(O.sort_pairs(raw, threads=THREADS)))
    return d1, d2, f, lists[0], lists[1]


def three_relation_oracle(d1, d2, f, list_in, list_out):
    from oracle import pipelines as OP
    from redfox_b200 import plans as PL
    return OP.three_relation_plan(d1, d2, f, list_in, list_out, PL.C2_SEGMENT, PL.C2_DATE_LO, PL.C2_DATE_HI,
                                  threads=THREADS)


def serving_query_oracle(d1, d2, f, segment, date_lo, date_hi, keys_list=None):
    """The parameterised select-join-(intersect)-join-aggregate query on the oracle."""
    d1s = O.select(d1, [32, 8], oracle_cmps([(O.EQ, (O.OPND_VAR, 1), (O.OPND_CONST, segment), O.I8)]))
    d2f = O.select(d2, [32, 32, 32], oracle_cmps([(O.GE, (O.OPND_VAR, 2), (O.OPND_CONST, date_lo), O.I32),
                                                  (O.LT, (O.OPND_VAR, 2), (O.OPND_CONST, date_hi), O.I32)]))
    d2s = O.project(d2f, [32, 32, 32], [32, 32], [1, 0])
    d2s = O.sort_pairs(d2s, begin_bit=32, end_bit=64, threads=THREADS)
    j1 = O.join_tuples(d1s, 8, d2s, 32, 16)
    keys = O.project(j1, [32, 8, 32], [32], [2]).view(np.uint32).ravel()
    keys = O.sort_pairs(keys, threads=THREADS)
    if keys_list is not None:
        keys = O.set_intersection(keys, keys_list)
    fs = O.sort_pairs(f, begin_bit=64, end_bit=96, threads=THREADS)
    j2 = O.join_tuples(keys.view(np.uint8).reshape(-1, 4), 0, fs, 64, 16)
    limbs = j2.view(np.uint64)
    key = limbs[:, 1].astype(np.uint32)
    amt = limbs[:, 0].astype(np.int64)
    k, sums = O.reduce_sum_i64(key, amt)
    _, counts = O.reduce_count(key)
    return k, sums, counts
