"""Batched execution: many independent sort + join + aggregate queries in one launch per
operator, and the whole batched plan captured as a CUDA graph.

The queries are folded into one relation by putting the query id below each query's key
(key' = key << 9 | q, the per-query key domains |R|/4 being below 2^21 and q below 2^9), and
the relation holds the queries in query order.  A stable sort on the key's 21 bits alone
therefore leaves equal keys in query order, i.e. it sorts on the whole composite key in
three 8-bit digit passes (the query bits need none); the sort-merge join on the composite
joins every query with itself only, and the aggregate groups per (key, query).  The join and the aggregate on its key run
as one operator (rfx_join_aggregate: per key, the join's SUM and COUNT from the two sides'
sorted runs, no join rows written) in both forms, batched and plain.  Tiles of all queries then share the
persistent kernels' dynamic tile queues (the device work queue), so a 10^4-row query and an
8 * 10^6-row query occupy the GPU alike, and per-query launch and read-back costs vanish.

Per query (the batched-form workload): |R|, |S| log-uniform in [1e4, 8e6]; R keys uniform
over [0, |R|/4); S.fk drawn uniformly from R's keys; amounts uniform in [100, 10^7).
"""
import math

from . import plans as PL
from . import rfx as R
from .workloads import SEED_BASE

C3_QUERIES = 512
C3_MIN, C3_MAX = 10_000, 8_000_000
C3_SEED = SEED_BASE + 3
QUERY_BITS = 9                 # the query id: the low bits of the 32-bit key field
QUERY_MASK = (1 << QUERY_BITS) - 1
KEY_BITS = 21                  # the per-query key above it
R_SORT_BITS = (32 + QUERY_BITS, 32 + QUERY_BITS + KEY_BITS)   # R rows: the key field is bits 32..63
S_SORT_BITS = (64 + QUERY_BITS, 64 + QUERY_BITS + KEY_BITS)   # S rows: the foreign key is bits 64..95


def fold(key, q):
    """The key field of query q's row with key `key`."""
    return (key << QUERY_BITS) | q


def unfold(field):
    """(key, query id) of key fields (integers or tensors)."""
    return field >> QUERY_BITS, field & QUERY_MASK


def _mix64(x):
    m = (1 << 64) - 1
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & m
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & m
    return x ^ (x >> 31)


def _rand(seed, stream, idx):
    """The SplitMix64 stream every generator here uses (same as the device generator)."""
    m = (1 << 64) - 1
    base = _mix64(seed ^ ((stream * 0xD1B54A32D192ED03) & m))
    return _mix64((base + (idx + 1) * 0x9E3779B97F4A7C15) & m)


def query_sizes(nq=C3_QUERIES, lo=C3_MIN, hi=C3_MAX, seed=C3_SEED):
    """(|R|, |S|) per query, log-uniform in [lo, hi]."""
    out = []
    for q in range(nq):
        u = [(_rand(seed, s, q) >> 11) * 2.0 ** -53 for s in (0, 1)]
        out.append(tuple(int(round(math.exp(math.log(lo) + x * (math.log(hi) - math.log(lo))))) for x in u))
    return out


def gen_batch(sizes, device="cuda"):
    """Concatenated R (8-byte rows) and S (16-byte rows) of all queries, in query order, with
    the query id folded into the key field (fold()), plus per-query row offsets."""
    import torch
    nr_tot = sum(s[0] for s in sizes)
    ns_tot = sum(s[1] for s in sizes)
    r_all = torch.empty((nr_tot, 8), dtype=torch.uint8, device=device)
    s_all = torch.empty((ns_tot, 16), dtype=torch.uint8, device=device)
    r_off, s_off = [0], [0]
    for q, (nr, ns) in enumerate(sizes):
        dom = max(1, nr // 4)
        rq = R.gen_uniform_rows(nr, [32, 32], C3_SEED + 16 + 2 * q, [0, 0], [dom, 1 << 32], device=device)
        sq = R.gen_uniform_rows(ns, [32, 64], C3_SEED + 17 + 2 * q, [0, 100], [nr, 10_000_000], device=device)
        r64 = rq.view(torch.int64).view(nr)
        keys = (r64 >> 32) & 0xFFFFFFFF
        s64 = sq.view(torch.int64).view(ns, 2)
        s64[:, 1] = fold(keys[s64[:, 1]], q)
        r64.copy_((fold(keys, q) << 32) | (r64 & 0xFFFFFFFF))
        r_all[r_off[-1]:r_off[-1] + nr] = rq
        s_all[s_off[-1]:s_off[-1] + ns] = sq
        r_off.append(r_off[-1] + nr)
        s_off.append(s_off[-1] + ns)
    return r_all, s_all, r_off, s_off


class BatchedPlan:
    """The join + aggregate plan over the folded relations, with every buffer allocated up
    front (outputs sized by |S|, every count on the device) so that the plan can be
    captured in a CUDA graph and replayed."""

    def __init__(self, r_all, s_all):
        import torch
        dev = r_all.device
        self.r_in, self.s_in = r_all, s_all
        self.nr, self.ns = r_all.shape[0], s_all.shape[0]
        self.r = torch.empty_like(r_all)
        self.s = torch.empty_like(s_all)
        self.rsort = R.Sorter(self.nr, 8, 0, *R_SORT_BITS, device=dev)
        self.ssort = R.Sorter(self.ns, 16, 0, *S_SORT_BITS, device=dev)
        self.ja = R.JoinAggregate(self.ns, 4, device=dev)
        self.graph = None

    @property
    def keys(self):
        return self.ja.keys

    @property
    def sums(self):
        return self.ja.sums

    @property
    def counts(self):
        return self.ja.counts

    def nbytes(self):
        return sum(t.numel() * t.element_size() for t in (self.r, self.s, self.ja.keys, self.ja.sums,
                                                          self.ja.counts, self.ja.ws, self.rsort.ws, self.ssort.ws))

    def run(self, stream=None):
        """Enqueue the whole plan (no host synchronisation).  The sorts read the inputs and
        write the plan's own buffers, so the inputs stay as they are for the next replay."""
        self.rsort(self.r, stream=stream, src_keys=self.r_in)
        self.ssort(self.s, stream=stream, src_keys=self.s_in)
        self.ja(self.r, 32, self.s, 64, 0, 64, stream=stream)

    def capture(self):
        """Capture run() in a CUDA graph (after one eager run has warmed every kernel up)."""
        import torch
        self.run()
        torch.cuda.synchronize()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=s):
            self.run(stream=s)
        torch.cuda.synchronize()

    def replay(self):
        self.graph.replay()

    def result(self):
        """(keys, sums, counts, join rows): the join's row count is the sum of the counts."""
        import torch
        keys, sums, counts = self.ja.result()
        return keys, sums, counts, int(counts.to(torch.int64).sum())


def split_by_query(keys, sums, counts, nq):
    """Batched groups (ordered by key, then query) -> per-query (keys, sums, counts) for
    queries 0 .. nq - 1, keys without the query bits, in key order."""
    import torch
    k64 = keys.to(torch.int64) & 0xFFFFFFFF
    key, q = unfold(k64)
    out = []
    for i in range(nq):
        m = q == i
        out.append((key[m].to(keys.dtype), sums[m], counts[m]))
    return out


def plain_query(r_all, s_all, r_off, s_off, q, stream=None):
    """Query q alone through the plain plan (one launch sequence, the group count read
    back): the same sorts on the key's bits, the same join-aggregate.  Returns (keys with
    the query bits, sums, counts, join rows)."""
    import torch
    keys, sums, counts = PL.join_aggregate_fused(r_all[r_off[q]:r_off[q + 1]], s_all[s_off[q]:s_off[q + 1]],
                                                 stream=stream, r_bits=R_SORT_BITS, s_bits=S_SORT_BITS)
    return keys, sums, counts, int(counts.to(torch.int64).sum())
