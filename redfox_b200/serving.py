"""Serving form: resident base relations, a request loop that admits queued queries
against a device-memory budget for their intermediates, and continuous batching: the
queries admitted since the last round started are packed into one batched plan (the query
id folded into the low 8 bits of every key, as the batched form folds it into the high
bits), so one scan of D1 and D2, one sort, one join, one intersection, one join with F and
one reduce serve all of them.  Up to `slots` rounds are in flight at once on their own
CUDA streams, so a round admitted while another runs overlaps it on the device (every
operator is a persistent kernel that claims its tiles dynamically).

The query (the three-relation pipeline with parameters): select D1 on a segment, select
D2 on a date range [lo, lo + width), join D2 to D1, optionally intersect the D2 keys with
a key list, join the fact table F (resident, sorted on its foreign key) and reduce
SUM(amount), COUNT by D2's key.  Parameters per query: width uniform in [30, 2500] days,
lo uniform over the remaining days, segment uniform in 0..4, and with probability 1/2 a
sorted list of log-uniform [1e3, 1e6] distinct keys drawn from D2's keys.

`Scheduler` is the admission logic alone (no GPU): FIFO, at most `slots` queries in
flight, and the sum of the in-flight queries' estimated intermediate bytes within the
budget (a query larger than the whole budget runs alone).  `simulate` drives it with a
given service time per query on a virtual clock.  `Server` runs it for real: batched
rounds (`run_round`), or one plain query at a time (`run_query`) as the serial baseline.
"""
import collections
import math
import threading
import time
from dataclasses import dataclass, field
from typing import Optional

from . import plans as PL
from .batch import _rand

DATE_DAYS = 2526
WIDTH_MIN, WIDTH_MAX = 30, 2500
LIST_MIN, LIST_MAX = 1_000, 1_000_000
BUDGET_BYTES = 40 * 10**9
SERVING_SEED = PL.SEED_BASE + 4


@dataclass
class Query:
    qid: int
    arrival: float                 # seconds after the start of the trace
    segment: int
    date_lo: int
    date_hi: int
    list_size: int                 # 0: no intersection
    list_seed: int = 0
    est_bytes: int = 0
    result: object = field(default=None, repr=False)
    start: float = math.nan
    done: float = math.nan

    @property
    def latency(self):
        return self.done - self.arrival


def _u01(seed, stream, idx):
    return (_rand(seed, stream, idx) >> 11) * 2.0 ** -53


def gen_requests(n, rate, seed=SERVING_SEED, n2=PL.C2_D2_ROWS):
    """n queries with Poisson arrivals of the given rate (queries/s) and seeded parameters."""
    out, t = [], 0.0
    for q in range(n):
        t += -math.log(1.0 - _u01(seed, 0, q)) / rate
        width = WIDTH_MIN + int(_u01(seed, 1, q) * (WIDTH_MAX - WIDTH_MIN + 1))
        lo = int(_u01(seed, 2, q) * (DATE_DAYS - width + 1))
        seg = int(_u01(seed, 3, q) * 5)
        size = 0
        if _u01(seed, 4, q) < 0.5:
            x = math.log(LIST_MIN) + _u01(seed, 5, q) * (math.log(LIST_MAX) - math.log(LIST_MIN))
            size = min(int(round(math.exp(x))), n2)
        qr = Query(q, t, seg, lo, lo + width, size, list_seed=seed + 1000 + q)
        qr.est_bytes = estimate_bytes(qr, n2)
        out.append(qr)
    return out


def estimate_bytes(q, n2=PL.C2_D2_ROWS, n1=PL.C2_D1_ROWS):
    """Upper estimate of a query's device intermediates: the date selection of D2 (8-byte
    rows, its sorted copy and the sort's buffer), the D1 selection, the first join and its
    key column, the optional list, and the F join (4 F rows per D2 key on average, with
    margin) with its reduce outputs."""
    frac = (q.date_hi - q.date_lo) / DATE_DAYS
    d2 = int(n2 * frac * 1.05) + 4096
    d1 = n1 // 5 + 4096
    j1 = d2 // 4 + 4096                       # D2 rows whose D1 row is in the segment (~1/5)
    f_rows = 6 * j1
    return 3 * 8 * d2 + 8 * d1 + 16 * j1 + 8 * j1 + 8 * q.list_size + 16 * f_rows + 16 * j1 + (16 << 20)


class Scheduler:
    """FIFO admission with `slots` concurrent queries and a byte budget."""

    def __init__(self, slots, budget_bytes=BUDGET_BYTES):
        self.slots = slots
        self.budget = budget_bytes
        self.pending = collections.deque()
        self.free = list(range(slots))[::-1]
        self.inflight = {}
        self.inflight_bytes = 0
        self.peak_bytes = 0
        self.peak_queries = 0

    def arrive(self, q):
        self.pending.append(q)

    def admissions(self):
        """Queries to start now, each with its slot (FIFO: the head waits for room)."""
        out = []
        while self.pending and self.free:
            q = self.pending[0]
            if self.inflight and self.inflight_bytes + q.est_bytes > self.budget:
                break
            self.pending.popleft()
            slot = self.free.pop()
            self.inflight[q.qid] = (q, slot)
            self.inflight_bytes += q.est_bytes
            self.peak_bytes = max(self.peak_bytes, self.inflight_bytes)
            self.peak_queries = max(self.peak_queries, len(self.inflight))
            out.append((q, slot))
        return out

    def complete(self, q):
        _, slot = self.inflight.pop(q.qid)
        self.inflight_bytes -= q.est_bytes
        self.free.append(slot)

    def idle(self):
        return not self.pending and not self.inflight


def simulate(requests, service_time, slots, budget_bytes=BUDGET_BYTES):
    """Discrete-event run of the scheduler on a virtual clock; service_time(q, concurrent)
    gives a query's run time.  Sets start / done on the queries and returns the scheduler."""
    import heapq
    sch = Scheduler(slots, budget_bytes)
    events = []                                     # (time, kind, seq, query); kind 0 = done
    for q in requests:
        heapq.heappush(events, (q.arrival, 1, q.qid, q))
    seq = len(requests)
    while events:
        now, kind, _, q = heapq.heappop(events)
        if kind == 0:
            sch.complete(q)
        else:
            sch.arrive(q)
        for a, _slot in sch.admissions():
            a.start = now
            a.done = now + service_time(a, len(sch.inflight))
            seq += 1
            heapq.heappush(events, (a.done, 0, seq, a))
    return sch


# ------------------------------------------------------------------ device side
class Resident:
    """The base relations resident in HBM: D1, D2 and F sorted on its foreign key."""

    def __init__(self, n1=PL.C2_D1_ROWS, n2=PL.C2_D2_ROWS, n3=PL.C2_F_ROWS, device="cuda"):
        import torch

        from . import rfx as R
        self.n1, self.n2, self.n3 = n1, n2, n3
        self.d1, self.d2, f, _, _ = PL.gen_three_relation(n1, n2, n3, 1, 1, device=device)
        self.f_sorted = f.clone()
        R.sort_pairs(self.f_sorted, begin_bit=64, end_bit=96)
        del f
        torch.cuda.synchronize()

    def nbytes(self):
        return sum(t.numel() * t.element_size() for t in (self.d1, self.d2, self.f_sorted))


def query_list(q, n2, device):
    """The query's sorted distinct u32 keys (or None), drawn with its own seed."""
    if q.list_size == 0:
        return None
    import torch

    from . import rfx as R
    raw = R.gen_uniform_rows(q.list_size, [32], q.list_seed, [0], [n2], device=device)
    raw = raw.view(torch.int32).view(q.list_size).clone()
    R.sort_pairs(raw)
    return R.unique(raw).clone()


def run_query(res, q, keys_list=None):
    """The parameterised pipeline on the current stream; returns (keys, sums, counts) on
    the device."""
    import torch

    from . import rfx as R
    d1s, _ = R.select(res.d1, [32, 8], [(R.EQ, (R.OPND_VAR, 1), (R.OPND_CONST, q.segment), R.I8)])
    d2s, _ = R.select_project(res.d2, [32, 32, 32], [(R.GE, (R.OPND_VAR, 2), (R.OPND_CONST, q.date_lo), R.I32),
                                                     (R.LT, (R.OPND_VAR, 2), (R.OPND_CONST, q.date_hi), R.I32)],
                              [], [32, 32], [1, 0])                               # (fk, pk)
    d2s = d2s.clone()
    R.sort_pairs(d2s, begin_bit=32, end_bit=64)
    j1, _ = R.join_tuples_two_step(d1s, 8, d2s, 32, 16)                            # (pk1, seg, pk2)
    keys = R.project(j1, [32, 8, 32], [32], [2]).view(torch.int32).view(-1).clone()
    R.sort_pairs(keys)
    if keys_list is not None:
        keys = R.set_op(R.SET_INTERSECTION, keys, keys_list)
    keys4 = keys.view(torch.uint8).view(-1, 4)
    j2, total = R.join_tuples_two_step(keys4, 0, res.f_sorted, 64, 16)             # (pk2, amount)
    gk, gs, gc, _ = R.reduce_tuples(j2, 64, 0, 64, 4, n=total)
    return gk, gs, gc


def run_alone(res, q, device="cuda"):
    """One query by itself on the default stream; host copies of its result."""
    import torch
    lst = query_list(q, res.n2, device)
    out = run_query(res, q, lst)
    torch.cuda.synchronize()
    return tuple(t.cpu() for t in out)


def _fold_lists(lists, stream=None):
    """Per-query sorted distinct u32 key lists -> one sorted list of (key << 8 | q) in
    8-byte elements (int64)."""
    import torch

    from . import rfx as R
    parts = [(lst.to(torch.int64) & 0xFFFFFFFF) << 8 | q for q, lst in enumerate(lists)]
    folded = torch.cat(parts) if parts else torch.zeros(0, dtype=torch.int64)
    R.sort_pairs(folded, begin_bit=0, end_bit=40, stream=stream)
    return folded


def run_round(res, queries, lists=None, stream=None):
    """The queries of one admission round as one batched plan.  Every key carries the
    query id q (index in `queries`, < 256) in its low 8 bits, so each operator serves all
    queries at once and never mixes them:

      D1 scan    rows (pk << 8 | q, seg)        for each q with seg == segment_q
      D2 scan    rows (fk << 8 | q, pk)         for each q with date in [lo_q, hi_q)
      sort       D2 rows on (fk, q)
      join       on (pk, q) = (fk, q)           -> (pk1, q, seg, pk2)
      project    (pk2, q), sort, and with lists: intersect with the folded lists
      join F     on pk2 (the query bits sit below the key)  -> (pk2, q, amount)
      reduce     SUM(amount), COUNT by (pk2, q)

    `lists`: None, or one sorted distinct u32 key list per query (every query of the
    round then has one).  Returns the reduce's (keys = pk2 << 8 | q as int64, sums,
    counts) on the device; `split_round` separates the queries."""
    import torch

    from . import rfx as R
    assert 0 < len(queries) <= 256
    d1m, _ = R.multi_select(res.d1, (0, 8), [(q.segment, q.segment + 1) for q in queries], (8, 32), (0, 8),
                            stream=stream)                                         # Tuple<32,8,8>
    d2m, _ = R.multi_select(res.d2, (0, 32), [(q.date_lo, q.date_hi) for q in queries], (32, 24), (64, 32),
                            stream=stream)                                         # Tuple<24,8,32>
    d1r = d1m.view(torch.uint8).view(-1, 8)
    d2r = d2m.view(torch.uint8).view(-1, 8)
    R.sort_pairs(d2r, begin_bit=32, end_bit=64, stream=stream)                      # on (fk, q)
    j1, _ = R.join_tuples_two_step(d1r, 8, d2r, 32, 16, stream=stream)               # (pk1, q, seg, pk2)
    keys = R.project(j1, [32, 8, 8, 32], [32, 8], [3, 1], stream=stream).clone()    # (pk2, q)
    R.sort_pairs(keys, begin_bit=0, end_bit=40, stream=stream)
    if lists is not None:
        keys = R.set_op(R.SET_INTERSECTION, keys, _fold_lists(lists, stream).view(torch.uint8).view(-1, 8),
                        stream=stream)
    j2, total = R.join_tuples_two_step(keys, 8, res.f_sorted, 64, 16, stream=stream)  # (pk2, q, amount)
    gk, gs, gc, _ = R.reduce_tuples(j2, 64, 0, 64, 8, n=total, stream=stream)
    return gk, gs, gc


class PinnedStage:
    """A page-locked host buffer that results are copied into (device-to-host copies from
    pageable memory run at a fraction of the link's speed); grown geometrically, reused."""

    def __init__(self, nbytes=0):
        import torch
        # pinning memory takes long (hundreds of MB per ~0.1 s): done up front, not per round
        self.buf = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True) if nbytes else None

    def take(self, nbytes):
        import torch
        if self.buf is None or self.buf.numel() < nbytes:
            cap = max(nbytes, 2 * (self.buf.numel() if self.buf is not None else 0), 1 << 20)
            self.buf = torch.empty(cap, dtype=torch.uint8, pin_memory=True)
        return self.buf


def to_host(tensors, stream=None, stage=None, copy=False, at=0):
    """Device tensors -> numpy arrays.  With a PinnedStage the copies go through its
    page-locked buffer from byte `at` on (the arrays are views of it unless copy=True)."""
    import torch
    if stage is None:
        return [t.cpu().numpy() for t in tensors]
    sizes = [t.numel() * t.element_size() for t in tensors]
    buf = stage.take(at + sum((b + 255) // 256 * 256 for b in sizes))
    views, off = [], at
    for t, b in zip(tensors, sizes):
        v = buf[off:off + b].view(t.dtype).view(t.shape)
        v.copy_(t, non_blocking=True)
        views.append(v)
        off += (b + 255) // 256 * 256
    (stream or torch.cuda.current_stream()).synchronize()
    return [v.numpy().copy() if copy else v.numpy() for v in views]


def split_round(gk, gs, gc, nq, stream=None, stage=None, copy=True):
    """A round's groups -> per query (keys u32, sums int64, counts u32) on the host, in key
    order.  The groups are ordered by (pk2, q); a stable one-pass radix sort on the query
    byte (on the device) makes each query's groups contiguous and keeps them in key order,
    then one copy per column (16 bytes per group) and the per-query group counts bring them
    to the host (through `stage` when given)."""
    import numpy as np
    import torch

    from . import rfx as R
    g = gk.shape[0]
    q8 = (gk & 0xFF).to(torch.int32)
    perm = torch.arange(g, dtype=torch.int32, device=gk.device)
    if g > 1:
        R.sort_pairs(q8, perm, begin_bit=0, end_bit=8, stream=stream)
    p64 = perm.to(torch.int64)
    kk = (gk.index_select(0, p64) >> 8).to(torch.int32)
    per_q = torch.bincount(q8, minlength=nq)[:nq]          # groups of each query, on the device
    k, sums, counts, nper = to_host([kk, gs.index_select(0, p64), gc.index_select(0, p64), per_q], stream, stage,
                                    copy)
    k, counts = k.view(np.uint32), counts.view(np.uint32)
    bounds = np.concatenate([[0], np.cumsum(nper)])
    return [(k[bounds[i]:bounds[i + 1]], sums[bounds[i]:bounds[i + 1]], counts[bounds[i]:bounds[i + 1]])
            for i in range(nq)]


def run_round_host(res, queries, device="cuda", stream=None, stage=None, copy=True, batch_min=8, on_done=None):
    """A round end to end: lists generated, queries with and without a list run as two
    batched plans (the intersection applies to the first only), results on the host in
    the order of `queries` (copied out of `stage` unless copy=False).  A round of fewer than
    `batch_min` queries runs them one after another with the plain plan: a batched plan's
    extra passes (the query byte in every key) cost more than a few queries share; then
    on_done(i, result), if given, is called as each query's result reaches the host."""
    import contextlib

    import numpy as np
    import torch
    if len(queries) < batch_min:
        outs, at = [], 0
        for i, q in enumerate(queries):
            with torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext():
                out = run_query(res, q, query_list(q, res.n2, device))
            k, sm, c = to_host(out, stream, stage, copy, at=at)
            outs.append((k.view(np.uint32), sm, c.view(np.uint32)))
            if on_done is not None:
                on_done(i, outs[-1])
            at += sum((t.numel() * t.element_size() + 255) // 256 * 256 for t in out)
        return outs
    res_by_q = [None] * len(queries)
    with_list = [i for i, q in enumerate(queries) if q.list_size > 0]
    without = [i for i, q in enumerate(queries) if q.list_size == 0]
    for idx, has in ((with_list, True), (without, False)):
        if not idx:
            continue
        qs = [queries[i] for i in idx]
        lists = [query_list(q, res.n2, device) for q in qs] if has else None
        gk, gs, gc = run_round(res, qs, lists, stream=stream)
        for i, r in zip(idx, split_round(gk, gs, gc, len(qs), stream=stream, stage=stage, copy=copy)):
            res_by_q[i] = r
    return res_by_q


class Server:
    """Request loop over resident relations.  A dispatcher admits arrived queries through a
    Scheduler (FIFO, budget) and packs the admitted queries into rounds of at most
    `max_batch`; up to `slots` worker threads each run a round on their own CUDA stream
    (`run_round`) and complete its queries when its results are on the host.  A round
    starts beside one already running only when at least `concurrent_min` queries are
    ready: two small rounds at once share the GPU and the host thread that launches them,
    and both finish later than they would one after the other.  With plain=True every
    round is one query run by `run_query` (the serial plain baseline when slots = 1).
    Latency = host time from arrival to the result on the host."""

    # result bytes staged per query: (key, sum, count, query byte) for each of its groups,
    # at most one per D2 row and in practice below 3M
    STAGE_GROUPS_PER_QUERY = 3_000_000

    def __init__(self, res, slots=2, budget_bytes=BUDGET_BYTES, device="cuda", max_batch=64, plain=False,
                 concurrent_min=8):
        import torch
        self.res = res
        self.slots = slots
        self.concurrent_min = concurrent_min
        self.budget = budget_bytes
        self.plain = plain
        self.max_batch = 1 if plain else max(1, min(256, max_batch))
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(slots)]
        # results reach the host through these page-locked buffers, sized for a full round
        per_query = 20 * min(self.STAGE_GROUPS_PER_QUERY, res.n2)
        self.stages = [PinnedStage(self.max_batch * per_query) for _ in range(slots)]

    def _run(self, i, rnd, keep_results, on_done=None):
        import numpy as np
        if self.plain:
            q = rnd[0]
            lst = query_list(q, self.res.n2, self.device)
            k, sm, c = to_host(run_query(self.res, q, lst), self.streams[i], self.stages[i], copy=keep_results)
            return [(k.view(np.uint32), sm, c.view(np.uint32))]
        return run_round_host(self.res, rnd, self.device, stream=self.streams[i], stage=self.stages[i],
                              copy=keep_results, on_done=on_done)

    def serve(self, requests, keep_results=False):
        import torch
        sch = Scheduler(self.slots * self.max_batch, self.budget)
        cv = threading.Condition()
        ready = collections.deque()        # admitted, not yet in a round
        work = [None] * self.slots          # the round each worker runs
        busy = [False] * self.slots
        stop = [False]
        errors = []
        self.rounds = []                    # queries per round, in start order
        self.round_log = []                 # (queries, start s, end s) per round, in end order
        t0 = time.perf_counter()

        def worker(i):
            torch.cuda.set_device(self.device)
            with torch.cuda.stream(self.streams[i]):
                while True:
                    with cv:
                        while work[i] is None and not stop[0]:
                            cv.wait()
                        if work[i] is None:
                            return
                        rnd = work[i]
                    # a query of a small round (plain plans one after another) is done when
                    # its own result is on the host; the others when the round's are
                    early = {}

                    def on_done(j, host, rnd=rnd, early=early):
                        early[j] = time.perf_counter() - t0
                        rnd[j].result = host if keep_results else (int(host[0].shape[0]),)

                    try:
                        outs = self._run(i, rnd, keep_results, on_done)
                        for q, host in zip(rnd, outs):
                            q.result = host if keep_results else (int(host[0].shape[0]),)
                    except Exception as e:  # reported after the run
                        errors.append(([q.qid for q in rnd], repr(e)))
                    done = time.perf_counter() - t0
                    with cv:
                        self.round_log.append((len(rnd), rnd[0].start, done))
                        for j, q in enumerate(rnd):
                            q.done = early.get(j, done)
                            sch.complete(q)
                        work[i] = None
                        busy[i] = False
                        cv.notify_all()

        threads = [threading.Thread(target=worker, args=(i,), daemon=True) for i in range(self.slots)]
        for th in threads:
            th.start()
        order = sorted(requests, key=lambda q: q.arrival)
        nxt = 0
        with cv:
            while nxt < len(order) or not sch.idle():
                now = time.perf_counter() - t0
                while nxt < len(order) and order[nxt].arrival <= now:
                    sch.arrive(order[nxt])
                    nxt += 1
                for q, _slot in sch.admissions():
                    ready.append(q)
                for i in range(self.slots):
                    if not ready or (any(busy) and len(ready) < self.concurrent_min):
                        break
                    if not busy[i]:
                        rnd = [ready.popleft() for _ in range(min(self.max_batch, len(ready)))]
                        for q in rnd:
                            q.start = now
                        self.rounds.append(len(rnd))
                        work[i] = rnd
                        busy[i] = True
                cv.notify_all()
                timeout = None
                if nxt < len(order):
                    timeout = max(0.0, order[nxt].arrival - (time.perf_counter() - t0))
                if timeout is None or timeout > 0:
                    cv.wait(timeout=timeout if timeout is not None else 0.05)
            stop[0] = True
            cv.notify_all()
        for th in threads:
            th.join()
        if errors:
            raise RuntimeError("queries failed: %s" % errors[:3])
        return sch


def latency_summary(requests, makespan=None):
    lat = sorted(q.latency for q in requests)
    if makespan is None:
        makespan = max(q.done for q in requests) - min(q.arrival for q in requests)

    def pct(p):
        return lat[min(len(lat) - 1, int(round(p / 100 * (len(lat) - 1))))]

    return {"queries": len(lat), "queries_per_s": len(lat) / makespan if makespan > 0 else None,
            "latency_ms_p50": pct(50) * 1e3, "latency_ms_p99": pct(99) * 1e3, "makespan_s": makespan}
