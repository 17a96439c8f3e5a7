"""Serving form: resident base relations, a request loop that admits queued queries
against a device-memory budget for their intermediates, and continuous batching --
queries that arrive while others run are admitted as soon as a slot and budget free up,
and their work overlaps on the device (one CUDA stream per slot; every operator is a
persistent kernel that claims its tiles dynamically, so kernels of different queries
share the SMs without waiting on one another).

The query (the three-relation pipeline with parameters): select D1 on a segment, select
D2 on a date range [lo, lo + width), join D2 to D1, optionally intersect the D2 keys with
a key list, join the fact table F (resident, sorted on its foreign key) and reduce
SUM(amount), COUNT by D2's key.  Parameters per query: width uniform in [30, 2500] days,
lo uniform over the remaining days, segment uniform in 0..4, and with probability 1/2 a
sorted list of log-uniform [1e3, 1e6] distinct keys drawn from D2's keys.

`Scheduler` is the admission logic alone (no GPU): FIFO, at most `slots` queries in
flight, and the sum of the in-flight queries' estimated intermediate bytes within the
budget (a query larger than the whole budget runs alone).  `simulate` drives it with a
given service time per query on a virtual clock.  `Server` runs it for real.
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


class Server:
    """Request loop over resident relations: a dispatcher admits arrived queries through a
    Scheduler, and one worker thread per slot runs each admitted query on the slot's CUDA
    stream and copies its result to the host.  Latency = host time from arrival to the
    result on the host."""

    def __init__(self, res, slots=8, budget_bytes=BUDGET_BYTES, device="cuda"):
        import torch
        self.res = res
        self.slots = slots
        self.budget = budget_bytes
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(slots)]

    def serve(self, requests, keep_results=False):
        import torch
        sch = Scheduler(self.slots, self.budget)
        cv = threading.Condition()
        work = [collections.deque() for _ in range(self.slots)]
        stop = [False]
        errors = []
        t0 = time.perf_counter()

        def worker(i):
            torch.cuda.set_device(self.device)
            with torch.cuda.stream(self.streams[i]):
                while True:
                    with cv:
                        while not work[i] and not stop[0]:
                            cv.wait()
                        if not work[i]:
                            return
                        q = work[i].popleft()
                    try:
                        lst = query_list(q, self.res.n2, self.device)
                        out = run_query(self.res, q, lst)
                        host = tuple(t.to("cpu", non_blocking=True) for t in out)
                        self.streams[i].synchronize()
                        q.result = host if keep_results else (int(host[0].shape[0]),)
                    except Exception as e:  # reported after the run
                        errors.append((q.qid, repr(e)))
                    q.done = time.perf_counter() - t0
                    with cv:
                        sch.complete(q)
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
                for q, slot in sch.admissions():
                    q.start = now
                    work[slot].append(q)
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
