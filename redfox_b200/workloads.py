"""Workload shapes of the benchmarks: relations, their packed tuple types, value ranges
and the RA plans run over them.  Inputs are seeded synthetic data of the named shapes
(SplitMix64 streams, one per column; seed 0x5EED0000 + workload index).
"""
from . import rfx as R
from .shapes import (FACT_CUTOFF, FACT_GROUP_DOMAIN, FACT_GROUP_FIELDS, FACT_HI, FACT_LO,  # noqa: F401
                     FACT_ROWS, FACT_SEED, FACT_SUM_FIELDS, FACT_WIDTHS, FACT_WORKLOAD, F_DATE, F_DISC,
                     F_FLAG1, F_FLAG2, F_PRICE, F_QTY, F_TAX, SEED_BASE)

# ---------------------------------------------------------------- filter-project-aggregate
# The fact table's shape and value ranges are in shapes.py; the plan over it is here.


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


def gen_fact(n, device="cuda", stream=None):
    return R.gen_uniform_rows(n, FACT_WIDTHS, FACT_SEED, FACT_LO, FACT_HI, device=device, stream=stream)


def fact_plan(n, device="cuda"):
    """The prepared fused select -> arith -> group-by plan over n fact rows."""
    return R.FilterAggregate(n, FACT_WIDTHS, fact_predicate(), fact_ariths(), FACT_GROUP_FIELDS,
                             FACT_GROUP_DOMAIN, FACT_SUM_FIELDS, device=device)


def fact_row_bytes():
    return R.container_bytes(sum(FACT_WIDTHS))


# ---------------------------------------------------------------- string keys
STRING_SEED = SEED_BASE + 7
# Name-like prefixes (shared runs longer than one 7-character refinement chunk) and bytes
# that are negative as `char`.
STRING_PREFIXES = [b"", b"Customer#0000", b"Supplier#000000000", b"Clerk#", b"\x80\xfe\x7f",
                   b"aaaaaaaaaaaaaaaaaaaaaa"]


def gen_strings(n, seed=STRING_SEED, distinct=None, max_len=40):
    """A seeded string column: (pool, offs), n NUL-terminated strings back to back in one
    uint8 array (every element its own copy, so equal strings have distinct addresses)
    and their offsets.  `distinct` base strings (default n // 4 + 1) are drawn with
    replacement; they cover the cases the string order has to get right: empty strings,
    proper prefixes of other strings, bytes >= 0x80, long shared prefixes and narrow
    alphabets ('a'/'b' only, digits only) that tie over many chunks."""
    import numpy as np
    rng = np.random.default_rng(seed)
    m = distinct or n // 4 + 1
    width = max_len + 1
    lens = rng.integers(0, max_len + 1, m)
    kind = rng.integers(0, 4, m)
    full = rng.integers(1, 256, (m, width), dtype=np.uint8)
    ab = rng.integers(ord("a"), ord("c"), (m, width), dtype=np.uint8)
    digits = rng.integers(ord("0"), ord("9") + 1, (m, width), dtype=np.uint8)
    mat = np.where((kind == 1)[:, None], ab, np.where((kind == 2)[:, None], digits, full))
    pre = rng.integers(0, len(STRING_PREFIXES), m)
    for k, p in enumerate(STRING_PREFIXES):
        if p:
            rows = np.nonzero((pre == k) & (kind == 3))[0]
            mat[rows, :len(p)] = np.frombuffer(p, np.uint8)
            lens[rows] = np.maximum(lens[rows], len(p))
    # every eighth string is a proper prefix of the one before it
    j = np.arange(7, m, 8)
    mat[j] = mat[j - 1]
    lens[j] = lens[j - 1] // 2
    lens[rng.random(m) < 0.02] = 0
    idx = rng.integers(0, m, n)
    rows = mat[idx]
    rl = lens[idx]
    cols = np.arange(width)[None, :]
    rows[cols == rl[:, None]] = 0
    pool = rows[cols <= rl[:, None]]
    offs = np.zeros(n, np.uint64)
    if n > 1:
        np.cumsum(rl[:-1] + 1, out=offs[1:])
    return (pool if n else np.zeros(1, np.uint8)), offs
