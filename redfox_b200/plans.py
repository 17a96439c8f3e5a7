"""RA plans of the benchmark workloads, built from the C ABI entries.

* join_aggregate (the reference's plain join + aggregate case): R(key, payload) and
  S(fk, amount) are sorted on their keys, sort-merge joined, and the join output is
  reduced to SUM(amount) and COUNT per key -- addJoin + addAgg
  (RelationalAlgebraCompiler.cpp:4466-5227, :7852-8643) with the split / merge glue
  fused away (sort and join work on packed tuples directly).
* three_relation: select D1 on segment and D2 on a date range, join D2 to D1, keep the
  D2 keys that are in one list and not in another (set intersection, set difference),
  join the fact table F to them and reduce SUM(amount) by D2's key.

Each plan runs stream-ordered on the device; like the reference, sizes of intermediate
results are read back where the next step must be sized by them.
"""
from . import rfx as R
from .workloads import SEED_BASE

# ---------------------------------------------------------------- join + aggregate
C0_R_ROWS = 1_000_000
C0_S_ROWS = 4_000_000
C0_KEY_DOMAIN = 1 << 18
C0_SEED = SEED_BASE + 0
C0_S_SEED = C0_SEED + 0x10000


def gen_join_aggregate(nr=C0_R_ROWS, ns=C0_S_ROWS, key_domain=C0_KEY_DOMAIN, device="cuda"):
    """R = Tuple<32,32>(key U[0,2^18), payload U32) in 8-byte rows; S = Tuple<32,64>(fk drawn
    uniformly from R's keys, amount U[100, 10^7)) in 16-byte rows."""
    import torch
    r = R.gen_uniform_rows(nr, [32, 32], C0_SEED, [0, 0], [key_domain, 1 << 32], device=device)
    s = R.gen_uniform_rows(ns, [32, 64], C0_S_SEED, [0, 100], [nr, 10_000_000], device=device)
    s64 = s.view(torch.int64).view(ns, 2)
    rkeys = (r.view(torch.int64).view(nr) >> 32) & 0xFFFFFFFF
    s64[:, 1] = rkeys[s64[:, 1]]   # field 0 (bits 64..95) := R.key[index]
    return r, s


def join_aggregate(r, s, stream=None):
    """sort R, sort S, join on key, SUM(amount) and COUNT by key.
    Returns (keys u32, sums int64, counts u32, join_rows)."""
    r = r.clone()
    s = s.clone()
    R.sort_pairs(r, begin_bit=32, end_bit=64, stream=stream)     # R on its key field
    R.sort_pairs(s, begin_bit=64, end_bit=96, stream=stream)     # S on its key field
    out, total = R.join_tuples_two_step(r, 32, s, 64, 16, stream=stream)   # (key, payload, amount)
    keys, sums, counts, g = R.reduce_tuples(out, 96, 0, 64, 4, n=total, stream=stream)
    return keys, sums, counts, total


def join_aggregate_fused(r, s, stream=None, r_bits=(32, 64), s_bits=(64, 96)):
    """The same plan with the join and the aggregate as one operator: sort R, sort S, then
    SUM(amount) and COUNT per key straight from the sorted relations (rfx_join_aggregate;
    the join rows are never written).  r_bits / s_bits: the bit ranges the sorts order on
    (by default the whole key fields; a narrower range where the key's other bits are known
    to be constant).  Returns (keys u32, sums int64, counts u32) -- the bytes join_aggregate
    returns."""
    r, _ = R.sorted_copy(r, begin_bit=r_bits[0], end_bit=r_bits[1], stream=stream)
    s, _ = R.sorted_copy(s, begin_bit=s_bits[0], end_bit=s_bits[1], stream=stream)
    return R.join_aggregate(r, 32, s, 64, 0, 64, 4, stream=stream)


# ---------------------------------------------------------------- three-relation pipeline
C2_D1_ROWS = 1_500_000
C2_D2_ROWS = 15_000_000
C2_F_ROWS = 60_000_000
C2_L5 = 5_000_000
C2_L2 = 2_000_000
C2_SEED = SEED_BASE + 2
C2_SEGMENT = 2
C2_DATE_LO, C2_DATE_HI = 500, 2000


def zipf_cdf(domain, device):
    """cdf[k] = sum_{j<=k} 1/(j+1), accumulated left to right in float64."""
    import numpy as np
    import torch
    return torch.from_numpy(np.cumsum(1.0 / np.arange(1, domain + 1, dtype=np.float64))).to(device)


def gen_three_relation(n1=C2_D1_ROWS, n2=C2_D2_ROWS, n3=C2_F_ROWS, l5=C2_L5, l2=C2_L2, device="cuda"):
    """D1 = Tuple<32,8>(pk, segment) 8-byte rows; D2 = Tuple<32,32,32>(pk, fk -> D1 Zipf(1),
    date) 16-byte rows; F = Tuple<32,64>(fk -> D2 uniform, amount) 16-byte rows; two sorted
    unique u32 key lists drawn from D2's keys."""
    import torch
    seg = R.gen_uniform_rows(n1, [8], C2_SEED, [0], [5], device=device).view(n1).to(torch.int64)
    d1 = ((torch.arange(n1, dtype=torch.int64, device=device) << 8) | seg).view(torch.uint8).view(n1, 8)
    # Zipf(1) by inverse CDF: the top 53 bits of the stream as a uniform in [0, 1)
    top53 = R.gen_uniform_rows(n2, [64], C2_SEED + 1, [0], [1 << 53], device=device).view(torch.int64).view(n2)
    cdf = zipf_cdf(n1, device)
    target = top53.to(torch.float64) * (2.0 ** -53) * cdf[-1]
    fk = torch.searchsorted(cdf, target, right=True).clamp_(max=n1 - 1)
    date = R.gen_uniform_rows(n2, [32], C2_SEED + 5, [0], [2526], device=device).view(torch.int32).view(n2)
    date = date.to(torch.int64)
    d2 = torch.empty((n2, 2), dtype=torch.int64, device=device)
    d2[:, 1] = torch.arange(n2, dtype=torch.int64, device=device)
    d2[:, 0] = (fk << 32) | date
    d2 = d2.view(torch.uint8).view(n2, 16)
    f = R.gen_uniform_rows(n3, [32, 64], C2_SEED + 2, [0, 100], [n2, 10_000_000], device=device)
    lists = []
    for k, (cnt, seed) in enumerate(((l5, C2_SEED + 3), (l2, C2_SEED + 4))):
        raw = R.gen_uniform_rows(cnt, [32], seed, [0], [n2], device=device).view(torch.int32).view(cnt).clone()
        R.sort_pairs(raw)
        lists.append(R.unique(raw).clone())
    return d1, d2, f, lists[0], lists[1]


def three_relation(d1, d2, f, list_in, list_out, f_sorted=None, stream=None):
    """The select / join / set-op / join / aggregate pipeline.  Returns (keys, sums, counts).
    `f_sorted`: F already sorted on fk (a resident, indexed base relation), else F is
    sorted as part of the plan."""
    import torch
    d1s, _ = R.select(d1, [32, 8], [(R.EQ, (R.OPND_VAR, 1), (R.OPND_CONST, C2_SEGMENT), R.I8)], stream=stream)
    d2s, _ = R.select_project(d2, [32, 32, 32], [(R.GE, (R.OPND_VAR, 2), (R.OPND_CONST, C2_DATE_LO), R.I32),
                                                 (R.LT, (R.OPND_VAR, 2), (R.OPND_CONST, C2_DATE_HI), R.I32)],
                              [], [32, 32], [1, 0], stream=stream)                     # (fk, pk)
    d2s = d2s.clone()
    R.sort_pairs(d2s, begin_bit=32, end_bit=64, stream=stream)                        # on fk
    j1, _ = R.join_tuples_two_step(d1s, 8, d2s, 32, 16, stream=stream)                 # (pk1, seg, pk2)
    keys = R.project(j1, [32, 8, 32], [32], [2], stream=stream).view(torch.int32).view(-1).clone()
    R.sort_pairs(keys, stream=stream)
    keys = R.set_op(R.SET_INTERSECTION, keys, list_in, stream=stream)
    keys = R.set_op(R.SET_DIFFERENCE, keys, list_out, stream=stream)
    if f_sorted is None:
        f_sorted = f.clone()
        R.sort_pairs(f_sorted, begin_bit=64, end_bit=96, stream=stream)               # on fk
    keys4 = keys.view(torch.uint8).view(-1, 4)
    j2, total = R.join_tuples_two_step(keys4, 0, f_sorted, 64, 16, stream=stream)     # (pk2, amount)
    gk, gs, gc, _ = R.reduce_tuples(j2, 64, 0, 64, 4, n=total, stream=stream)
    return gk, gs, gc
