"""Shapes and seeds of the benchmark workloads as plain constants.

Nothing here loads librfx.so, so CPU-only code (the timed CPU baselines) can name the
workloads without mapping the GPU library into its process.  Inputs are seeded synthetic
data of the named shapes: SplitMix64 streams, one per column, seed 0x5EED0000 + workload
index.
"""

SEED_BASE = 0x5EED0000

# ---------------------------------------------------------------- filter-project-aggregate
# A fact table of Tuple<32,64,64,64,64,8,8> = (date, quantity, price, discount, tax,
# flag1, flag2) in a 64-byte container; price in fixed-point cents, discount and tax in
# hundredths.  Field f of row i is U[FACT_LO[f], FACT_HI[f]) from stream f.
FACT_WIDTHS = [32, 64, 64, 64, 64, 8, 8]
FACT_LO = [0, 1, 90000, 0, 0, 0, 0]
FACT_HI = [2526, 51, 10500001, 11, 9, 3, 2]
FACT_ROWS = 60_000_000
FACT_ROW_BYTES = 64
FACT_CUTOFF = 2475          # date <= cutoff keeps ~98% of the rows
FACT_SEED = SEED_BASE + 1
F_DATE, F_QTY, F_PRICE, F_DISC, F_TAX, F_FLAG1, F_FLAG2 = range(7)
FACT_GROUP_FIELDS = [F_FLAG1, F_FLAG2]
FACT_GROUP_DOMAIN = [3, 2]
FACT_SUM_FIELDS = [7, 8]   # the two appended products
FACT_WORKLOAD = ("filter-project-aggregate: 60M rows Tuple<32,64,64,64,64,8,8> (64 B), "
                 "select date<=2475 (~98%), 2 int64 products, group by (flag1,flag2) -> 6 groups SUM/COUNT")
