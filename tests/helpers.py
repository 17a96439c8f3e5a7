"""Shared test helpers: the oracle form of the workloads and small utilities."""
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


def to_np(t):
    return t.detach().cpu().numpy()
