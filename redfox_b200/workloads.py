"""Workload shapes of the benchmarks: relations, their packed tuple types, value ranges
and the RA plans run over them.  Inputs are seeded synthetic data of the named shapes
(SplitMix64 streams, one per column; seed 0x5EED0000 + workload index).
"""
from . import rfx as R

SEED_BASE = 0x5EED0000

# ---------------------------------------------------------------- filter-project-aggregate
# A fact table of Tuple<32,64,64,64,64,8,8> = (date, quantity, price, discount, tax,
# flag1, flag2) in a 64-byte container; price in fixed-point cents, discount and tax in
# hundredths.
FACT_WIDTHS = [32, 64, 64, 64, 64, 8, 8]
FACT_LO = [0, 1, 90000, 0, 0, 0, 0]
FACT_HI = [2526, 51, 10500001, 11, 9, 3, 2]
FACT_ROWS = 60_000_000
FACT_CUTOFF = 2475          # date <= cutoff keeps ~98% of the rows
FACT_SEED = SEED_BASE + 1
F_DATE, F_QTY, F_PRICE, F_DISC, F_TAX, F_FLAG1, F_FLAG2 = range(7)


def fact_predicate():
    """date <= cutoff (a field-vs-constant select, compared as unsigned int)."""
    return [(R.LE, (R.OPND_VAR, F_DATE), (R.OPND_CONST, FACT_CUTOFF), R.I32)]


def fact_ariths():
    """p1 = price * (100 - discount); p2 = price * (100 - discount) * (100 + tax), both
    appended as 64-bit fields (exact int64 fixed-point products)."""
    # nodes: (kind, op, type, left, right, value)
    p1 = R.make_arith([
        (R.NODE_OP, R.MUL, R.I64, 1, 2, 0),
        (R.NODE_INDEX, 0, R.I64, -1, -1, F_PRICE),
        (R.NODE_OP, R.SUB, R.I64, 3, 4, 0),
        (R.NODE_CONST, 0, R.I64, -1, -1, 100),
        (R.NODE_INDEX, 0, R.I64, -1, -1, F_DISC),
    ], 0, R.I64, 64)
    p2 = R.make_arith([
        (R.NODE_OP, R.MUL, R.I64, 1, 6, 0),
        (R.NODE_OP, R.MUL, R.I64, 2, 3, 0),
        (R.NODE_INDEX, 0, R.I64, -1, -1, F_PRICE),
        (R.NODE_OP, R.SUB, R.I64, 4, 5, 0),
        (R.NODE_CONST, 0, R.I64, -1, -1, 100),
        (R.NODE_INDEX, 0, R.I64, -1, -1, F_DISC),
        (R.NODE_OP, R.ADD, R.I64, 7, 8, 0),
        (R.NODE_CONST, 0, R.I64, -1, -1, 100),
        (R.NODE_INDEX, 0, R.I64, -1, -1, F_TAX),
    ], 0, R.I64, 64)
    return [p1, p2]


FACT_GROUP_FIELDS = [F_FLAG1, F_FLAG2]
FACT_GROUP_DOMAIN = [3, 2]
FACT_SUM_FIELDS = [7, 8]   # the two appended products


def gen_fact(n, device="cuda", stream=None):
    return R.gen_uniform_rows(n, FACT_WIDTHS, FACT_SEED, FACT_LO, FACT_HI, device=device, stream=stream)


def fact_plan(n, device="cuda"):
    """The prepared fused select -> arith -> group-by plan over n fact rows."""
    return R.FilterAggregate(n, FACT_WIDTHS, fact_predicate(), fact_ariths(), FACT_GROUP_FIELDS,
                             FACT_GROUP_DOMAIN, FACT_SUM_FIELDS, device=device)


def fact_row_bytes():
    return R.container_bytes(sum(FACT_WIDTHS))
