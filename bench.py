#!/usr/bin/env python
"""Benchmark of the RA execution layer on B200.

Workload (one step): the filter-project-aggregate scan over a 60M-row fact table of
Tuple<32,64,64,64,64,8,8> (64-byte rows): select date <= 2475, append the exact int64
products price*(100-discount) and price*(100-discount)*(100+tax), group by
(flag1, flag2) into 6 groups with SUM/COUNT.  One fused kernel per step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value  = rows/s with the table resident in HBM (3.84 GB per GPU, larger than L2, so no
         flush is needed between steps), timed with CUDA events, max over ranks.
e2e    = the same through the public API with the table in pinned host memory: each
         step copies it to the device, runs the plan and reads the groups back.
N > 1  = weak scaling: every rank scans its own 60M-row partition; the 6-group partial
         results are summed with one all-reduce inside each step.
--impl reference times the reference's own code for this plan (its Tuple.h / select /
arith / project device code and thrust reduce_by_key, compiled for the host in
oracle/_ref) on the host cores, or the C oracle where that library is absent.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

ROWS = 60_000_000
METRIC = "tuples/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--rows", type=int, default=ROWS)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-operators", action="store_true")
    ap.add_argument("--batched-queries", type=int, default=512,
                    help="queries of the batched join+aggregate comparison (0: skip it)")
    ap.add_argument("--serving-queries", type=int, default=300,
                    help="queries per arrival rate of the serving comparison (0: skip it)")
    ap.add_argument("--only", default=None,
                    help="comma-separated operator groups (%s): run only those operator benchmarks on one GPU "
                         "and print their JSON (no headline step)" % ",".join(["select", "sort_c0", "join",
                                                                                "sort_large", "setops", "pipelines",
                                                                                "strings_f64"]))
    ap.add_argument("--reps", type=int, default=5, help="timed calls per operator with --only")
    ap.add_argument("--sort-rows", type=int, default=60_000_000, help="rows of the large sorts (sort_large group)")
    ap.add_argument("--section", default=None, choices=["strings_f64", "batched", "serving"],
                    help="run one secondary benchmark alone and print its JSON (used by the main run, "
                         "which gives each secondary benchmark a fresh process and allocator)")
    return ap.parse_args()


def run_section(name, args):
    """A secondary benchmark in a fresh process: its timings then do not depend on the
    allocator and memory state the earlier benchmarks left behind."""
    cmd = [sys.executable, os.path.abspath(__file__), "--section", name,
           "--batched-queries", str(args.batched_queries), "--serving-queries", str(args.serving_queries)]
    p = subprocess.run(cmd, capture_output=True, text=True)
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    if p.returncode != 0 or not lines:
        return {"error": "section %s exited %d: %s" % (name, p.returncode, p.stderr.strip().splitlines()[-1:])}
    return json.loads(lines[-1])


def main_section(args):
    import torch
    dev = torch.device("cuda:0")
    if args.section == "strings_f64":
        out = string_f64_benchmarks(dev, measured_peak_hbm()[0])
    elif args.section == "batched":
        out = batched_benchmark(dev, args.batched_queries)
    else:
        out = serving_benchmark(dev, args.serving_queries)
    print(json.dumps(out), flush=True)
    return 0


# ------------------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sms, maxes, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm, mx = float(parts[1]), float(parts[2])
            except ValueError:
                continue
            sms.append(sm)
            maxes.append(mx)
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sms) if sms else None,
                "sm_max_mhz": max(maxes) if maxes else None,
                "reasons": sorted(reasons), "samples": len(sms)}


def measured_peak_hbm():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(rows):
    """DRAM bytes per launch from the committed ncu summary, scaled to `rows`."""
    path = os.path.join(REPO, "profiles", "fact_filter_aggregate.md")
    try:
        with open(path) as f:
            for ln in f:
                if ln.startswith("dram_bytes_per_row:"):
                    return float(ln.split(":")[1]) * rows
    except OSError:
        pass
    return None


# ------------------------------------------------------------------------------ CPU legs
# The CPU legs import only the oracle package and redfox_b200.shapes (plain constants), so
# the process that times the reference's CPU code never maps librfx.so.
def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def fact_oracle_descriptors():
    """The plan's predicate and the two products as oracle descriptors:
    date <= cutoff; price*(100-discount); price*(100-discount)*(100+tax)."""
    import oracle as O
    from redfox_b200 import shapes as SH
    cmps = [{"op": O.LE, "a": (O.OPND_VAR, SH.F_DATE), "b": (O.OPND_CONST, SH.FACT_CUTOFF), "type": O.I32}]
    p1 = O.make_arith([(O.NODE_OP, O.MUL, O.I64, 1, 2, 0), (O.NODE_INDEX, 0, O.I64, -1, -1, SH.F_PRICE),
                       (O.NODE_OP, O.SUB, O.I64, 3, 4, 0), (O.NODE_CONST, 0, O.I64, -1, -1, 100),
                       (O.NODE_INDEX, 0, O.I64, -1, -1, SH.F_DISC)], 0, O.I64, 64)
    p2 = O.make_arith([(O.NODE_OP, O.MUL, O.I64, 1, 6, 0), (O.NODE_OP, O.MUL, O.I64, 2, 3, 0),
                       (O.NODE_INDEX, 0, O.I64, -1, -1, SH.F_PRICE), (O.NODE_OP, O.SUB, O.I64, 4, 5, 0),
                       (O.NODE_CONST, 0, O.I64, -1, -1, 100), (O.NODE_INDEX, 0, O.I64, -1, -1, SH.F_DISC),
                       (O.NODE_OP, O.ADD, O.I64, 7, 8, 0), (O.NODE_CONST, 0, O.I64, -1, -1, 100),
                       (O.NODE_INDEX, 0, O.I64, -1, -1, SH.F_TAX)], 0, O.I64, 64)
    return cmps, [p1, p2]


def fact_rows_host(n):
    """The first n rows of the seeded fact table, packed on the host (same bytes as the
    device generator)."""
    import oracle as O
    from redfox_b200 import shapes as SH
    cols = [O.uniform(n, SH.FACT_SEED, f, SH.FACT_LO[f], SH.FACT_HI[f]) for f in range(7)]
    return O.pack(SH.FACT_WIDTHS, cols)


def oracle_port_fn(threads):
    """One run of the C oracle's filter-aggregate (OpenMP) over `rows` -> (keys, sums, counts)."""
    import oracle as O
    from redfox_b200 import shapes as SH
    cmps, ariths = fact_oracle_descriptors()

    def run(rows):
        return O.filter_aggregate(rows, SH.FACT_WIDTHS, cmps, ariths, SH.FACT_GROUP_FIELDS, SH.FACT_SUM_FIELDS,
                                  threads=threads)
    return run


def reference_plan_fn(threads):
    """ref_fact_plan from oracle/_ref -- the reference's Select.h / Project.h / arith device
    code and thrust reduce_by_key compiled for the host -- over `threads` row partitions
    in parallel, partial groups summed; None where oracle/_ref is not built."""
    import ctypes as C
    from concurrent.futures import ThreadPoolExecutor

    import numpy as np
    import oracle as O
    from redfox_b200 import shapes as SH
    ref = O.ref_lib()
    if ref is None:
        return None
    fn = ref.ref_fact_plan
    fn.restype = C.c_int64
    fn.argtypes = [C.c_void_p, C.c_size_t, C.c_uint, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    pool = ThreadPoolExecutor(max_workers=threads)

    def run(rows):
        n = rows.shape[0]
        cuts = [n * i // threads for i in range(threads + 1)]

        def one(i):
            sub = rows[cuts[i]:cuts[i + 1]]
            ok = np.zeros(16, np.uint64)
            s1 = np.zeros(16, np.int64)
            s2 = np.zeros(16, np.int64)
            cnt = np.zeros(16, np.uint64)
            g = fn(sub.ctypes.data_as(C.c_void_p), sub.shape[0], SH.FACT_CUTOFF, ok.ctypes.data_as(C.c_void_p),
                   s1.ctypes.data_as(C.c_void_p), s2.ctypes.data_as(C.c_void_p), cnt.ctypes.data_as(C.c_void_p))
            return ok[:g], s1[:g], s2[:g], cnt[:g]

        merged = {}
        for ok, s1, s2, cnt in pool.map(one, range(threads)):   # ctypes releases the GIL
            for k, a, b, c in zip(ok, s1, s2, cnt):
                x = merged.get(int(k), (0, 0, 0))
                merged[int(k)] = (x[0] + int(a), x[1] + int(b), x[2] + int(c))
        keys = sorted(merged)
        return (np.array(keys, np.uint64), np.array([[merged[k][0], merged[k][1]] for k in keys], np.int64),
                np.array([merged[k][2] for k in keys], np.uint64))
    return run


def time_steps(run, rows, steps, warmup):
    """`warmup` untimed runs, then `steps` timed runs; returns the per-run seconds."""
    for _ in range(warmup):
        run(rows)
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        run(rows)
        ts.append(time.perf_counter() - t0)
    return ts


def cpu_legs(rows, kind, steps=5, warmup=1, one_core=True):
    """All-host-thread and 1-thread timings of the CPU implementation of the plan over the
    whole table: median of `steps` runs after `warmup`, and one 1-thread run."""
    threads = cpu_threads()
    make = reference_plan_fn if kind == "reference" else oracle_port_fn
    run = make(threads)
    if run is None:
        return None
    ts = time_steps(run, rows, steps, warmup)
    n = rows.shape[0]
    out = {"threads": threads, "seconds": ts, "median_s": statistics.median(ts), "value": n / statistics.median(ts)}
    if one_core:
        t1 = time_steps(make(1), rows, 1, 0)[0]
        out["one_core"] = {"value": n / t1, "seconds": t1, "cores": 1}
    return out


def cpu_baseline_line(rows):
    """The oracle port (C, OpenMP) over the whole seeded table on the host: median of 5
    after 1 warm-up with all host threads, plus one 1-thread run."""
    leg = cpu_legs(rows, "port")
    return {"value": leg["value"], "unit": "tuples/s", "cores": leg["threads"], "kind": "port",
            "sample": "the whole %d-row table (host copy of the timed input), C oracle (OpenMP), median of 5 "
                      "after 1 warm-up" % rows.shape[0],
            "one_core": {"value": leg["one_core"]["value"], "unit": "tuples/s", "cores": 1,
                         "sample": "one run over the whole table"}}


def bench_config(n, world):
    from redfox_b200 import shapes as SH
    return {"workload": SH.FACT_WORKLOAD, "rows_per_gpu": n, "row_bytes": SH.FACT_ROW_BYTES,
            "l2": "inputs larger than L2 (%.2f GB per GPU), no flush" % (n * SH.FACT_ROW_BYTES / 1e9),
            "parallelism": "dp%d (row partitions, 6-group all-reduce)" % world if world > 1 else "1 GPU"}


# ------------------------------------------------------------------------------ reference arm
def main_reference(args):
    """The reference's CPU code for the plan (oracle/_ref's ref_fact_plan, or the C oracle
    where the reference did not build) over the same 60M-row table as our arm, every host
    thread; value = rows / median step time over the timed steps."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = cpu_threads()
    n = args.rows
    rows = fact_rows_host(n)
    run = reference_plan_fn(threads)
    kind = "reference" if run is not None else "port"
    if run is None:
        run = oracle_port_fn(threads)
    ts = time_steps(run, rows, args.steps, max(args.warmup, 1))
    med = statistics.median(ts)
    value = n / med
    one = time_steps((reference_plan_fn if kind == "reference" else oracle_port_fn)(1), rows, 1, 0)[0]
    what = ("the reference's Select.h / Project.h / Tuple.h device code and thrust reduce_by_key built for the "
            "host (oracle/_ref ref_fact_plan), %d row partitions in parallel" % threads) if kind == "reference" \
        else "C oracle (OpenMP)"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "tuples/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": med * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": bench_config(n, 1),
        "cpu_baseline": {"value": value, "unit": "tuples/s", "cores": threads, "kind": kind,
                         "sample": "the whole %d-row table every step; %s; median of %d steps after %d warm-up"
                                   % (n, what, args.steps, max(args.warmup, 1)),
                         "mean_ms_per_step": statistics.mean(ts) * 1e3,
                         "one_core": {"value": n / one, "unit": "tuples/s", "cores": 1,
                                      "sample": "one run over the whole table"}},
        "e2e": {"value": value, "unit": "tuples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------ per operator
def _time_ms(fn, reps, setup=None):
    """Mean device time of fn() over `reps` calls (CUDA events on the current stream)
    after one untimed call (first-call host set-up: tensor maps, launch attributes).
    Without setup the calls run back to back between one pair of events, so the host's
    time to enqueue a call overlaps the previous call on the device; with setup(), which
    runs before each call outside the timed interval, each call has its own events."""
    import torch
    stream = torch.cuda.current_stream()
    if setup is not None:
        setup()
    fn()
    torch.cuda.synchronize()
    if setup is None:
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b) / reps
    total = 0.0
    for _ in range(reps):
        if setup is not None:
            setup()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        total += a.elapsed_time(b)
    return total / reps


def _op_line(n, nbytes, ms, peak, **extra):
    gbs = nbytes / (ms / 1e3) / 1e9
    d = {"tuples": n, "ms": ms, "tuples_per_s": n / (ms / 1e3), "algorithmic_bytes": nbytes, "gb_s": gbs,
         "frac_of_measured_hbm": gbs / peak}
    d.update(extra)
    return d


class OpContext:
    """Inputs of the operator benchmarks, generated on first use and kept resident."""

    def __init__(self, dev, fact_rows):
        self.dev = dev
        self.fact_rows = fact_rows
        self._c0 = None
        self._c2 = None

    def c0(self):
        """(R, S) of the join + aggregate workload, unsorted and sorted on their keys."""
        if self._c0 is None:
            from redfox_b200 import plans as PL
            from redfox_b200 import rfx as R
            r, s = PL.gen_join_aggregate(device=self.dev)
            rs, ss = r.clone(), s.clone()
            R.sort_pairs(rs, begin_bit=32, end_bit=64)
            R.sort_pairs(ss, begin_bit=64, end_bit=96)
            self._c0 = (r, s, rs, ss)
        return self._c0

    def c2(self):
        if self._c2 is None:
            from redfox_b200 import plans as PL
            self._c2 = PL.gen_three_relation(device=self.dev)
        return self._c2


def _op_select(ctx, peak, reps):
    import torch

    from redfox_b200 import rfx as R
    from redfox_b200 import workloads as WL
    rows = ctx.fact_rows
    n = rows.shape[0]
    out = torch.empty_like(rows)
    cnt = torch.zeros(1, dtype=torch.int64, device=ctx.dev)
    t = R.Tuple.of(WL.FACT_WIDTHS)
    cm = R.make_cmps(WL.fact_predicate())
    wsb = R.LIB.rfx_select_workspace(n, R.C.byref(t))
    ws = R._empty_bytes(wsb, ctx.dev)

    def sel():
        R.check("rfx_select", R.LIB.rfx_select(R._ptr(out), R._ptr(cnt), R._ptr(rows), n, R.C.byref(t), cm, 1,
                                               R._ptr(ws), wsb, R._stream()))
    sel()
    ms = _time_ms(sel, reps)
    k = int(cnt.item())
    tag = "%dM" % (n // 1_000_000) if n % 1_000_000 == 0 else str(n)
    return {"select_fact_%s" % tag: _op_line(n, n * 64 + k * 64, ms, peak, kept=k)}


def _sort_line(src, kb, begin, end, reps, peak, flags=0, note=None, passes=None):
    """Device time of sorting a copy of `src` (n x kb bytes) on bits [begin, end); the
    copy is restored before each call outside the timed interval."""
    import torch

    from redfox_b200 import rfx as R
    n = src.shape[0]
    work = torch.empty_like(src)
    srt = R.Sorter(n, kb, 0, begin, end, device=src.device)
    ms = _time_ms(lambda: srt(work, flags=flags), reps, setup=lambda: work.copy_(src))
    p = passes if passes is not None else (end - begin + 7) // 8
    extra = {"passes": p}
    if note:
        extra["note"] = note
    return _op_line(n, n * kb + p * 2 * n * kb, ms, peak, **extra)


def _op_sort_c0(ctx, peak, reps):
    r, s, _, _ = ctx.c0()
    return {"sort_pairs_4M_u32key_u64val": _sort_line(s, 16, 64, 96, reps, peak, note="S rows (fk, amount); 64 MB, fits L2"),
            "sort_tuples_1M_8B_on_key": _sort_line(r, 8, 32, 64, reps, peak, note="R rows (key, payload); fits L2")}


SORT_ROWS = 60_000_000   # rows of the large sorts (--sort-rows: smaller for profiling)


def _op_sort_large(ctx, peak, reps):
    import torch

    from redfox_b200 import plans as PL
    from redfox_b200 import rfx as R
    n = SORT_ROWS
    tag = "%dM" % (n // 1_000_000) if n % 1_000_000 == 0 else str(n)
    # the three-relation workload's F (fk uniform over D2's keys, amount), the same generator
    f = R.gen_uniform_rows(n, [32, 64], PL.C2_SEED + 2, [0, 100], [PL.C2_D2_ROWS, 10_000_000], device=ctx.dev)
    out = {"sort_tuples_%s_16B_on_fk" % tag: _sort_line(f, 16, 64, 96, 3, peak, flags=R.SORT_SKIP_TRIVIAL, passes=3,
                                                        note="fk < 2^24: the top digit is constant and skipped")}
    R.tune_force(R.TUNE_SORT_PASS, 1)
    try:
        out["sort_tuples_%s_16B_on_fk_onesweep_pass" % tag] = _sort_line(f, 16, 64, 96, 3, peak,
                                                                         flags=R.SORT_SKIP_TRIVIAL, passes=3,
                                                                         note="the pipelined onesweep pass")
    finally:
        R.tune_force(R.TUNE_SORT_PASS, -1)
    R.tune_force(R.TUNE_SORT_PASS, 4)
    try:
        out["sort_tuples_%s_16B_on_fk_match_rank" % tag] = _sort_line(f, 16, 64, 96, 3, peak,
                                                                      flags=R.SORT_SKIP_TRIVIAL, passes=3,
                                                                      note="per-tile pass ranking with match_any")
    finally:
        R.tune_force(R.TUNE_SORT_PASS, -1)
    del f
    keys = R.gen_uniform_rows(n, [32], 0x5EED0101, [0], [1 << 32], device=ctx.dev)
    out["sort_keys_%s_u32" % tag] = _sort_line(keys.view(torch.uint8).view(n, 4), 4, 0, 32, 3, peak,
                                               note="uniform 32-bit keys, 4 passes")
    del keys
    rows8 = R.gen_uniform_rows(n, [32, 32], 0x5EED0102, [0, 0], [1 << 32, 1 << 32], device=ctx.dev)
    out["sort_tuples_%s_8B_on_key" % tag] = _sort_line(rows8, 8, 32, 64, 3, peak, note="Tuple<32,32> rows on the key")
    return out


def _op_join(ctx, peak, reps):
    import torch

    from redfox_b200 import rfx as R
    _, _, rs, ss = ctx.c0()
    ops = {}
    nl, nr = rs.shape[0], ss.shape[0]
    tj = R.TupleJoin(nl, device=ctx.dev)
    dummy = torch.empty((1, 16), dtype=torch.uint8, device=ctx.dev)
    tj(dummy, 0, rs, 32, ss, 64)
    total = int(tj.count.item())
    jout = torch.empty((total, 16), dtype=torch.uint8, device=ctx.dev)
    ms = _time_ms(lambda: tj(jout, total, rs, 32, ss, 64), reps)
    ops["join_fused_1Mx4M"] = _op_line(total, total * 16 + nl * 8 + nr * 16 + nl * 16, ms, peak, inputs=nl + nr)
    # the same with the emit that gathers rows per output (the tuner's other variant)
    R.tune_force(R.TUNE_JOIN_EMIT, 1)
    try:
        ms = _time_ms(lambda: tj(jout, total, rs, 32, ss, 64), reps)
    finally:
        R.tune_force(R.TUNE_JOIN_EMIT, -1)
    ops["join_fused_1Mx4M_gather_emit"] = _op_line(total, total * 16 + nl * 8 + nr * 16 + nl * 16, ms, peak,
                                                   inputs=nl + nr)
    # find_bounds alone on the split u32 keys
    lk = ((rs.view(torch.int64).view(-1) >> 32) & 0xFFFFFFFF).to(torch.int32)
    rk = (ss.view(torch.int64).view(-1, 2)[:, 1] & 0xFFFFFFFF).to(torch.int32)
    lb = torch.empty(nl, dtype=torch.int32, device=ctx.dev)
    sc = torch.empty(nl, dtype=torch.int32, device=ctx.dev)
    tot = torch.zeros(1, dtype=torch.int64, device=ctx.dev)
    fwsb = R.LIB.rfx_join_find_bounds_workspace(nl)
    fws = R._empty_bytes(fwsb, ctx.dev)
    ms = _time_ms(lambda: R.check("fb", R.LIB.rfx_join_find_bounds(R._ptr(lb), R._ptr(sc), R._ptr(tot), R._ptr(lk), nl,
                                                                   R._ptr(rk), nr, 4, R._ptr(fws), fwsb, R._stream())),
                  reps)
    ops["find_bounds_1Mx4M_u32"] = _op_line(nl, (nl + nr) * 4 + 8 * nl, ms, peak, note="inputs fit L2")
    # reduce-by-key over the 19.3M-row join output (16 B rows, key = high 32 bits)
    g = torch.zeros(1, dtype=torch.int64, device=ctx.dev)
    okeys = torch.empty(total, dtype=torch.int32, device=ctx.dev)
    osum = torch.empty(total, dtype=torch.int64, device=ctx.dev)
    ocnt = torch.empty(total, dtype=torch.int32, device=ctx.dev)
    rwsb = R.LIB.rfx_reduce_by_key_workspace(total)
    rws = R._empty_bytes(rwsb, ctx.dev)
    ms = _time_ms(lambda: R.check("rt", R.LIB.rfx_reduce_tuples(R._ptr(jout), total, None, 16, 96, 0, 64, R._ptr(okeys),
                                                                4, R._ptr(osum), R._ptr(ocnt), R._ptr(g), R._ptr(rws),
                                                                rwsb, R._stream())), reps)
    groups = int(g.item())
    ops["reduce_by_key_19M_rows"] = _op_line(total, total * 16 + groups * 16, ms, peak, groups=groups)
    # the same with the earlier design: a look-back per 32 KB tile (the tuner's variant 2)
    R.tune_force(1, 2)
    try:
        ms = _time_ms(lambda: R.check("rt", R.LIB.rfx_reduce_tuples(R._ptr(jout), total, None, 16, 96, 0, 64,
                                                                    R._ptr(okeys), 4, R._ptr(osum), R._ptr(ocnt),
                                                                    R._ptr(g), R._ptr(rws), rwsb, R._stream())), reps)
    finally:
        R.tune_force(1, -1)
    ops["reduce_by_key_19M_rows_tile_lookback"] = _op_line(total, total * 16 + groups * 16, ms, peak, groups=groups,
                                                           note="look-back per 256-line tile (tuner variant 2)")
    # dense groups: 60M 16-byte rows (key U[0, 6M) at bits 64..95, 64-bit value), sorted on
    # the key, about 10 rows per group (the group density of the batched plan's reduce)
    dense = R.gen_uniform_rows(60_000_000, [32, 64], 0x5EED0301, [0, 100], [6_000_000, 10_000_000], device=ctx.dev)
    R.sort_pairs(dense, begin_bit=64, end_bit=96)
    dn = dense.shape[0]
    dkeys = torch.empty(dn, dtype=torch.int32, device=ctx.dev)
    dsum = torch.empty(dn, dtype=torch.int64, device=ctx.dev)
    dcnt = torch.empty(dn, dtype=torch.int32, device=ctx.dev)
    dwsb = R.LIB.rfx_reduce_by_key_workspace(dn)
    dws = R._empty_bytes(dwsb, ctx.dev)
    ms = _time_ms(lambda: R.check("rt", R.LIB.rfx_reduce_tuples(R._ptr(dense), dn, None, 16, 64, 0, 64, R._ptr(dkeys), 4,
                                                                R._ptr(dsum), R._ptr(dcnt), R._ptr(g), R._ptr(dws), dwsb,
                                                                R._stream())), reps)
    dg = int(g.item())
    ops["reduce_by_key_60M_rows_dense_groups"] = _op_line(dn, dn * 16 + dg * 16, ms, peak, groups=dg,
                                                          note="about 10 rows per group; inputs larger than L2")
    del dense, dkeys, dsum, dcnt, dws
    # join + aggregate on the key as one operator (no join rows)
    ja = R.JoinAggregate(nr, 4, device=ctx.dev)
    ms = _time_ms(lambda: ja(rs, 32, ss, 64, 0, 64), reps)
    gj = int(ja.groups.item())
    ops["join_aggregate_1Mx4M"] = _op_line(nl + nr, nl * 8 + nr * 16 + gj * 16, ms, peak, groups=gj,
                                           note="S reduced to its groups, then matched against R; inputs fit L2")
    return ops


def _op_setops(ctx, peak, reps):
    import torch

    from redfox_b200 import rfx as R
    _, _, _, l5, l2 = ctx.c2()
    ops = {}
    lists = [("5M_2M_u32", l5, l2, "inputs fit L2")]
    big_a = R.gen_uniform_rows(60_000_000, [32], 0x5EED0201, [0], [1 << 30], device=ctx.dev).view(torch.int32).view(-1)
    big_b = R.gen_uniform_rows(15_000_000, [32], 0x5EED0202, [0], [1 << 30], device=ctx.dev).view(torch.int32).view(-1)
    R.sort_pairs(big_a)
    R.sort_pairs(big_b)
    lists.append(("60M_15M_u32", big_a, big_b, "sorted u32 lists with duplicates, larger than L2"))
    for tag, a, b, note in lists:
        for name, op in (("intersect", R.SET_INTERSECTION), ("difference", R.SET_DIFFERENCE), ("union", R.SET_UNION)):
            outp = torch.empty(a.shape[0] + b.shape[0], dtype=torch.int32, device=ctx.dev)
            c = torch.zeros(1, dtype=torch.int64, device=ctx.dev)
            swsb = R.LIB.rfx_set_op_workspace(op, a.shape[0], b.shape[0], 4)
            sws = R._empty_bytes(swsb, ctx.dev)

            def run(op=op, a=a, b=b, outp=outp, c=c, sws=sws, swsb=swsb):
                R.check("set", R.LIB.rfx_set_op(op, R._ptr(outp), R._ptr(c), R._ptr(a), a.shape[0], R._ptr(b),
                                                b.shape[0], 4, R._ptr(sws), swsb, R._stream()))
            ms = _time_ms(run, reps)
            no = int(c.item())
            ops["%s_%s" % (name, tag)] = _op_line(a.shape[0] + b.shape[0], (a.shape[0] + b.shape[0] + no) * 4, ms,
                                                  peak, out=no, note=note)
            # the tuner's other variants beside the default (the warp-segment form, 16 items per
            # thread): the warp-segment form with 8 (5) and the two-pass form (6) for every
            # operator, the two-pass form with 16 items per thread (4) and the one-pass form (1, 3)
            # for the intersection
            variants = ((5, "warp_segment_8_per_thread"), (6, "two_pass"))
            if name == "intersect":
                variants += ((4, "two_pass_16_per_thread"), (1, "one_pass"), (3, "one_pass_16_per_thread"))
            for v, suffix in variants:
                R.tune_force(2, v)
                try:
                    ms = _time_ms(run, reps)
                finally:
                    R.tune_force(2, -1)
                ops["%s_%s_%s" % (name, tag, suffix)] = _op_line(a.shape[0] + b.shape[0],
                                                                 (a.shape[0] + b.shape[0] + no) * 4, ms, peak,
                                                                 out=no, note=note)
    return ops


PIPELINE_CPU_LEGS = True   # --no-cpu-baseline turns the pipelines' CPU legs off


def _pipeline_cpu_leg(fn, args, nin, steps=5, warmup=1):
    """The oracle's restatement of a plan (oracle/pipelines.py) on the host copies of the
    same inputs: all host threads (median of `steps` after `warmup`; the sorts use the
    threads, the other steps one), then one 1-thread run; also returns the result."""
    threads = cpu_threads()
    ts, res = [], None
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        res = fn(*args, threads=threads)
        if i >= warmup:
            ts.append(time.perf_counter() - t0)
    t0 = time.perf_counter()
    fn(*args, threads=1)
    t1 = time.perf_counter() - t0
    med = statistics.median(ts)
    return {"value": nin / med, "unit": "tuples/s", "cores": threads, "kind": "port", "median_s": med,
            "sample": "the whole workload, C oracle (sorts on every host thread), median of %d after %d warm-up"
                      % (steps, warmup),
            "one_core": {"value": nin / t1, "unit": "tuples/s", "cores": 1, "seconds": t1}}, res


def _op_pipelines(ctx, peak, reps):
    """The plans end to end (host reads sizes back between steps, as the reference): one
    untimed run first compiles the plan-specialised kernels, then the median of 5 timed
    runs (wall clock).  With PIPELINE_CPU_LEGS each plan also runs on the host through the
    oracle's restatement, timed and compared with the GPU result."""
    import numpy as np
    import torch

    from redfox_b200 import plans as PL
    r, s, _, _ = ctx.c0()
    d1, d2, f, l5, l2 = ctx.c2()
    ops = {}
    nin0 = r.shape[0] + s.shape[0]
    nin2 = d1.shape[0] + d2.shape[0] + f.shape[0]
    results = {}
    for name, fn, nin, note in (
            ("pipeline_join_aggregate_1Mx4M", lambda: PL.join_aggregate(r, s), nin0,
             "sort R, sort S, join (19.3M rows written), reduce; wall clock incl. size reads"),
            ("pipeline_join_aggregate_fused_1Mx4M", lambda: PL.join_aggregate_fused(r, s), nin0,
             "sort R, sort S, join-aggregate on the key (no join rows); wall clock incl. the group count read"),
            ("pipeline_three_relation_76M", lambda: PL.three_relation(d1, d2, f, l5, l2), nin2,
             "selects, sort, 2 joins, set ops, sort of F, reduce; wall clock")):
        results[name] = fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(5):
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            ts.append((time.perf_counter() - t0) * 1e3)
        ms = statistics.median(ts)
        ops[name] = {"tuples": nin, "ms": ms, "tuples_per_s": nin / (ms / 1e3), "note": note + ", median of 5"}
    if PIPELINE_CPU_LEGS:
        from oracle import pipelines as OP

        def host(t):
            return t.cpu().numpy()
        leg, (ek, es, ec, _) = _pipeline_cpu_leg(OP.join_aggregate_plan, (host(r), host(s)), nin0)
        gk, gs, gc = (host(x) for x in results["pipeline_join_aggregate_fused_1Mx4M"][:3])
        leg["parity"] = "ok" if (np.array_equal(gk.view(np.uint32), ek) and np.array_equal(gs, es) and
                                 np.array_equal(gc.view(np.uint32), ec.astype(np.uint32))) else "MISMATCH"
        ops["pipeline_join_aggregate_1Mx4M"]["cpu"] = leg
        leg, (ek, es, ec) = _pipeline_cpu_leg(
            OP.three_relation_plan, (host(d1), host(d2), host(f), host(l5), host(l2), PL.C2_SEGMENT, PL.C2_DATE_LO,
                                     PL.C2_DATE_HI), nin2)
        gk, gs, gc = (host(x) for x in results["pipeline_three_relation_76M"])
        leg["parity"] = "ok" if (np.array_equal(gk.view(np.uint32), ek) and np.array_equal(gs, es) and
                                 np.array_equal(gc.view(np.uint32), ec.astype(np.uint32))) else "MISMATCH"
        ops["pipeline_three_relation_76M"]["cpu"] = leg
    return ops


OPERATORS = {"select": _op_select, "sort_c0": _op_sort_c0, "join": _op_join, "sort_large": _op_sort_large,
             "setops": _op_setops, "pipelines": _op_pipelines}


def operator_benchmarks(dev, fact_rows, peak, reps=5, only=None):
    """tuples/s and fraction of the measured HBM bandwidth per operator, on the workload
    shapes (data resident in HBM; inputs larger than L2 except where noted).  `only`: a
    list of OPERATORS keys to run (all when None)."""
    ctx = OpContext(dev, fact_rows)
    ops = {}
    for name, fn in OPERATORS.items():
        if only is None or name in only:
            ops.update(fn(ctx, peak, reps))
    return ops


def string_f64_benchmarks(dev, peak, reps=5):
    """The string-keyed and double-valued operators (data resident in HBM)."""
    import numpy as np
    import torch

    from redfox_b200 import rfx as R
    from redfox_b200 import workloads as WL

    ops = {}
    # double SUM / MIN by u32 key: 19.3M rows, 256K groups (the join-output reduce shape)
    n, groups = 19_300_000, 256_000
    rng = np.random.default_rng(17)
    keys = torch.from_numpy(np.sort(rng.integers(0, groups, n)).astype(np.int32)).to(dev)
    vals = torch.from_numpy(np.round(rng.uniform(900.0, 105000.0, n), 2)).to(dev)
    ok = torch.empty_like(keys)
    ov = torch.empty(n, dtype=torch.float64, device=dev)
    g = torch.zeros(1, dtype=torch.int64, device=dev)
    wsb = R.LIB.rfx_reduce_f64_workspace(n)
    ws = R._empty_bytes(wsb, dev)
    for name, op in (("reduce_f64_sum_19M_u32key", R.F64_SUM), ("reduce_f64_min_19M_u32key", R.F64_MIN)):
        def run(op=op):
            R.check("f64", R.LIB.rfx_reduce_f64(R._ptr(keys), n, 4, R._ptr(vals), op, R._ptr(ok), R._ptr(ov),
                                                R._ptr(g), R._ptr(ws), wsb, R._stream()))
        ms = _time_ms(run, reps)
        k = int(g.item())
        pre = n * 8 if op == R.F64_SUM else 0   # the exponent pre-pass reads the values once more
        ops[name] = _op_line(n, n * 12 + k * 12, ms, peak, groups=k, traffic_floor_bytes=n * 12 + k * 12 + pre)
    # one run over 60M doubles (total_double)
    n1 = 60_000_000
    v1 = torch.from_numpy(np.round(rng.uniform(900.0, 105000.0, n1), 2)).to(dev)
    res = torch.zeros(1, dtype=torch.float64, device=dev)
    ms = _time_ms(lambda: R.check("sum", R.LIB.rfx_sum_double_compat(R._ptr(res), R._ptr(v1),
                                                                    R.C.c_void_p(v1.data_ptr() + 8 * n1))), reps)
    ops["sum_double_60M"] = _op_line(n1, n1 * 8, ms, peak, note="compat entry: allocates, synchronises")
    del v1, keys, vals, ok, ov, ws
    # strings: 2M names (about 21 characters on average, many shared prefixes)
    ns = 2_000_000
    pool, offs = WL.gen_strings(ns, distinct=500_000)
    dpool, ptrs = R.string_column(pool, offs, dev)
    sbytes = ns * 8 + int(pool.shape[0])
    work = ptrs.clone()
    codes = torch.empty(ns, dtype=torch.int32, device=dev)
    perm = torch.empty(ns, dtype=torch.int32, device=dev)
    nd = R.C.c_uint64(0)
    ms = _time_ms(lambda: R.check("codes", R.LIB.rfx_string_codes(R._ptr(ptrs), ns, R._ptr(codes), R._ptr(perm),
                                                                  R.C.byref(nd), R._stream())), 3)
    ops["string_codes_2M"] = _op_line(ns, sbytes, ms, peak, distinct=nd.value,
                                      note="rounds of 7 characters through the radix sort; wall-clock bound")
    ms = _time_ms(lambda: R.sort_strings(work), 3, setup=lambda: work.copy_(ptrs))
    ops["sort_string_key_2M"] = _op_line(ns, sbytes, ms, peak)
    R.sort_strings(work)
    cv = torch.ones(ns, dtype=torch.int32, device=dev)
    ms = _time_ms(lambda: R.count_string(work, cv), 3)
    ops["count_string_2M_sorted"] = _op_line(ns, sbytes + ns * 4, ms, peak)
    return ops


def tuning_benchmark(dev, fact_rows, reps=5):
    """Default variant vs the autotuner's choice per size class for the tuned operators:
    select (plan-specialised compaction, rows per thread), the staged reduce (256- or
    128-line tiles) and the set filters (8 or 4 items per thread), each at a large and a
    small size.  Device time per call (CUDA events), same inputs both ways."""
    import torch

    from redfox_b200 import plans as PL
    from redfox_b200 import rfx as R
    from redfox_b200 import workloads as WL

    cases = []
    small_rows = fact_rows[:600_000]
    for name, rows in (("select_fact_60M", fact_rows), ("select_fact_600K", small_rows)):
        out = torch.empty_like(rows)
        cnt = torch.zeros(1, dtype=torch.int64, device=dev)
        t = R.Tuple.of(WL.FACT_WIDTHS)
        cm = R.make_cmps(WL.fact_predicate())
        wsb = R.LIB.rfx_select_workspace(rows.shape[0], R.C.byref(t))
        ws = R._empty_bytes(wsb, dev)

        def f(rows=rows, out=out, cnt=cnt, t=t, cm=cm, ws=ws, wsb=wsb):
            R.check("sel", R.LIB.rfx_select(R._ptr(out), R._ptr(cnt), R._ptr(rows), rows.shape[0], R.C.byref(t), cm,
                                            1, R._ptr(ws), wsb, R._stream()))
        cases.append((name, f, (out, ws)))
    for name, (nr, ns, dom) in (("reduce_join_19M", (1_000_000, 4_000_000, 1 << 18)),
                                ("reduce_join_190K", (10_000, 40_000, 1 << 11))):
        r, s_ = PL.gen_join_aggregate(nr, ns, key_domain=dom, device=dev)
        R.sort_pairs(r, begin_bit=32, end_bit=64)
        R.sort_pairs(s_, begin_bit=64, end_bit=96)
        jout, total = R.join_tuples_two_step(r, 32, s_, 64, 16)
        g = torch.zeros(1, dtype=torch.int64, device=dev)
        ok = torch.empty(total, dtype=torch.int32, device=dev)
        osum = torch.empty(total, dtype=torch.int64, device=dev)
        ocnt = torch.empty(total, dtype=torch.int32, device=dev)
        wsb = R.LIB.rfx_reduce_by_key_workspace(total)
        ws = R._empty_bytes(wsb, dev)

        def f(jout=jout, total=total, g=g, ok=ok, osum=osum, ocnt=ocnt, ws=ws, wsb=wsb):
            R.check("rt", R.LIB.rfx_reduce_tuples(R._ptr(jout), total, None, 16, 96, 0, 64, R._ptr(ok), 4,
                                                  R._ptr(osum), R._ptr(ocnt), R._ptr(g), R._ptr(ws), wsb,
                                                  R._stream()))
        cases.append((name, f, (jout, ok, osum, ocnt, ws)))
    for name, (na, nb) in (("intersect_5M_2M", (5_000_000, 2_000_000)), ("intersect_50K_20K", (50_000, 20_000))):
        a = R.gen_uniform_rows(na, [32], 31, [0], [15_000_000], device=dev).view(torch.int32).view(-1).clone()
        b = R.gen_uniform_rows(nb, [32], 32, [0], [15_000_000], device=dev).view(torch.int32).view(-1).clone()
        R.sort_pairs(a)
        R.sort_pairs(b)
        a = R.unique(a).clone()
        b = R.unique(b).clone()
        out = torch.empty(a.shape[0] + b.shape[0], dtype=torch.int32, device=dev)
        c = torch.zeros(1, dtype=torch.int64, device=dev)
        wsb = R.LIB.rfx_set_op_workspace(R.SET_INTERSECTION, a.shape[0], b.shape[0], 4)
        ws = R._empty_bytes(wsb, dev)

        def f(a=a, b=b, out=out, c=c, ws=ws, wsb=wsb):
            R.check("set", R.LIB.rfx_set_op(R.SET_INTERSECTION, R._ptr(out), R._ptr(c), R._ptr(a), a.shape[0],
                                            R._ptr(b), b.shape[0], 4, R._ptr(ws), wsb, R._stream()))
        cases.append((name, f, (a, b, out, ws)))
    res = {}
    R.tune(0)
    R.tune_reset()
    for name, f, _ in cases:
        res[name] = {"default_ms": _time_ms(f, reps)}
    R.tune(1)
    for name, f, _ in cases:
        f()                      # the tuning call of this class
        torch.cuda.synchronize()
        res[name]["tuned_ms"] = _time_ms(f, reps)
    table = R.tune_table()
    R.tune(0)
    R.tune_reset()
    return {"cases": res, "table": table}


def batched_benchmark(dev, nq, reps=3):
    """512 (nq) independent sort + join + aggregate queries, |R|, |S| log-uniform in
    [1e4, 8e6]: one plain launch sequence per query, back to back, against the batched plan
    (all queries folded into one relation by query id, each operator one persistent launch)
    replayed as one CUDA graph.  All queries are submitted at once, so a query's latency is
    the time from the start of the batch to its own completion."""
    import torch

    from redfox_b200 import batch as B

    sizes = B.query_sizes(nq)
    r_all, s_all, r_off, s_off = B.gen_batch(sizes, device=dev)
    rows = int(r_all.shape[0] + s_all.shape[0])
    for q in range(min(nq, 4)):                         # warm-up (allocator, kernels)
        B.plain_query(r_all, s_all, r_off, s_off, q)
    torch.cuda.synchronize()
    done = [torch.cuda.Event(enable_timing=True) for _ in range(nq)]
    ev0 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    plain = []
    for q in range(nq):
        res = B.plain_query(r_all, s_all, r_off, s_off, q)
        done[q].record()
        if q < 8:
            plain.append(tuple(x.clone() if torch.is_tensor(x) else x for x in res))
    torch.cuda.synchronize()
    plain_done = [ev0.elapsed_time(e) for e in done]
    plain_ms = plain_done[-1]
    service = [plain_done[0]] + [b - a for a, b in zip(plain_done, plain_done[1:])]
    torch.cuda.empty_cache()

    plan = B.BatchedPlan(r_all, s_all)
    plan.capture()
    plan.replay()
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        plan.replay()
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    batch_ms = statistics.median(ms)
    keys, sums, counts, total = plan.result()
    per = B.split_by_query(keys, sums, counts, min(nq, 8))
    ok = all(torch.equal(per[q][0], B.unfold(plain[q][0])[0]) and torch.equal(per[q][1], plain[q][1])
             and torch.equal(per[q][2], plain[q][2]) for q in range(len(plain)))
    nbytes = plan.nbytes()
    del plan
    torch.cuda.empty_cache()

    def pct(v, p):
        v = sorted(v)
        return v[min(len(v) - 1, int(round(p / 100 * (len(v) - 1))))]

    return {
        "queries": nq, "rows": rows, "join_rows": total,
        "plain": {"ms": plain_ms, "queries_per_s": nq / (plain_ms / 1e3),
                  "latency_ms_p50": pct(plain_done, 50), "latency_ms_p99": pct(plain_done, 99),
                  "service_ms_p50": pct(service, 50), "service_ms_p99": pct(service, 99)},
        "batched_graph": {"ms": batch_ms, "queries_per_s": nq / (batch_ms / 1e3),
                          "latency_ms_p50": batch_ms, "latency_ms_p99": batch_ms, "replays": ms,
                          "plan_buffers_gb": nbytes / 1e9},
        "speedup_queries_per_s": plain_ms / batch_ms,
        "parity_first_8_queries": "ok" if ok else "MISMATCH",
        "note": "same kernels both ways (sort R, sort S, join-aggregate on the key); plain runs one launch "
                "sequence per query and reads its group count back, batched sorts and aggregates all queries "
                "folded by query id in one captured plan",
    }


def serving_benchmark(dev, nq, rates=(100.0, 300.0, 1000.0, 3000.0, 5000.0), slots=2):
    """Parameterised select-join-aggregate queries over the resident three-relation data
    (D1 1.5M, D2 15M, F 60M sorted on fk), Poisson arrivals at each rate: the serving loop
    (admission against a 40 GB intermediate budget; the queries admitted since the last
    round started packed into one batched plan; `slots` rounds in flight on their own
    streams) against serial plain execution of the same trace (one query at a time,
    FIFO).  Latency = host time from a query's arrival to its result on the host."""
    import torch

    from redfox_b200 import serving as S

    res = S.Resident(device=dev)
    warm = S.gen_requests(6, 1e6, seed=S.SERVING_SEED + 99)
    for q in warm:                                              # untimed warm-up
        S.run_alone(res, q, device=dev)
    S.run_round_host(res, warm, dev)
    out = {"resident_gb": res.nbytes() / 1e9, "slots": slots, "budget_gb": S.BUDGET_BYTES / 1e9,
           "queries_per_rate": nq, "rates": {}}
    servers = (("serial", S.Server(res, slots=1, device=dev, plain=True)),
               ("serving", S.Server(res, slots=slots, device=dev)))   # pinned result buffers made once
    for _, srv in servers:
        # untimed, the same for both servers: a burst that fills the largest rounds on every
        # slot, and a few spaced queries (rounds of one), so each server's streams have their
        # memory pools and kernels before the timed runs
        srv.serve(S.gen_requests(2 * 64 * slots, 1e6, seed=S.SERVING_SEED + 98))
        srv.serve(S.gen_requests(2 * slots, 200.0, seed=S.SERVING_SEED + 97))
    for rate in rates:
        line = {}
        for name, srv in servers:
            reqs = S.gen_requests(nq, rate)
            torch.cuda.synchronize()
            torch.cuda.reset_peak_memory_stats(dev)
            base = torch.cuda.memory_allocated(dev)
            sch = srv.serve(reqs)
            line[name] = S.latency_summary(reqs)
            line[name]["peak_in_flight"] = sch.peak_queries
            line[name]["rounds"] = len(srv.rounds)
            line[name]["mean_round"] = sum(srv.rounds) / max(1, len(srv.rounds))
            line[name]["max_round_ms"] = 1e3 * max((e - b for _, b, e in srv.round_log), default=0.0)
            line[name]["peak_intermediate_gb"] = (torch.cuda.max_memory_allocated(dev) - base) / 1e9
        line["speedup_queries_per_s"] = line["serving"]["queries_per_s"] / line["serial"]["queries_per_s"]
        out["rates"][str(int(rate))] = line
    del res
    torch.cuda.empty_cache()
    return out


# ------------------------------------------------------------------------------ our arm
def main_ours(args):
    import torch
    import torch.distributed as dist

    from redfox_b200 import rfx as R
    from redfox_b200 import workloads as WL
    from redfox_b200.partition import merge_group_tables, partition_seed

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    n = args.rows
    stream = torch.cuda.current_stream()

    # each rank's partition: rows [rank*n, (rank+1)*n) of the seeded table, made on device
    rows = R.gen_uniform_rows(n, WL.FACT_WIDTHS, partition_seed(WL.FACT_SEED, rank), WL.FACT_LO, WL.FACT_HI, device=dev)
    plan = WL.fact_plan(n, device=dev)
    nacc = plan.G * (plan.nsum + 1)
    gacc = plan.ws[: nacc * 8].view(torch.int64)
    torch.cuda.synchronize()

    def step():
        plan.launch(rows)
        if world > 1:
            merge_group_tables(gacc)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    assert R.device_status() == R.OK
    # correctness spot check against the oracle on the first rows (not timed)
    check_n = 1_000_000
    chk = WL.fact_plan(check_n, device=dev)
    chk.launch(rows)
    keys, sums, counts = chk.result()

    if world > 1:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    k_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.synchronize()
    ev0.record(stream)
    for i in range(args.steps):
        k_ev[i][0].record(stream)
        plan.launch(rows)
        k_ev[i][1].record(stream)
        if world > 1:
            merge_group_tables(gacc)
    ev1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    ms_total = ev0.elapsed_time(ev1)
    kernel_ms = [a.elapsed_time(b) for a, b in k_ev]
    t = torch.tensor([ms_total, statistics.mean(kernel_ms)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_total, kms = float(t[0]), float(t[1])
    ms_step = ms_total / args.steps
    value = world * n / (ms_step / 1e3)

    # ---- end to end: host table -> device -> plan -> groups back to host
    host = torch.empty((n, WL.fact_row_bytes()), dtype=torch.uint8, pin_memory=True)
    host.copy_(rows)
    dev_in = torch.empty_like(rows)
    out_k = torch.empty(plan.G, dtype=torch.int64, pin_memory=True)
    out_s = torch.empty((plan.G, plan.nsum), dtype=torch.int64, pin_memory=True)
    out_c = torch.empty(plan.G, dtype=torch.int64, pin_memory=True)
    out_g = torch.empty(1, dtype=torch.int64, pin_memory=True)

    def e2e_step():
        dev_in.copy_(host, non_blocking=True)
        plan.launch(dev_in)
        if world > 1:
            merge_group_tables(gacc)
        out_k.copy_(plan.keys, non_blocking=True)
        out_s.copy_(plan.sums[:, :plan.nsum], non_blocking=True)
        out_c.copy_(plan.counts, non_blocking=True)
        out_g.copy_(plan.ngroups, non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.e2e_steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    te = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_ms = float(te[0]) / args.e2e_steps
    d2h = (plan.G * (2 + plan.nsum) + 1) * 8
    del host
    dev_in_keep = dev_in

    ok = R.device_status() == R.OK
    result = None
    if rank == 0:
        peak, peak_kind = measured_peak_hbm()
        bytes_alg = n * WL.fact_row_bytes()
        achieved = bytes_alg / (kms / 1e3) / 1e9
        traffic = profiled_traffic(n)
        cpu = None
        parity_rows = 0
        import numpy as np
        import oracle as O
        cmps, ariths = fact_oracle_descriptors()
        sub = rows[:check_n].cpu().numpy()
        ek, es, ec = O.filter_aggregate(sub, WL.FACT_WIDTHS, cmps, ariths, WL.FACT_GROUP_FIELDS, WL.FACT_SUM_FIELDS)
        ok = ok and np.array_equal(keys, ek) and np.array_equal(sums, es) and np.array_equal(counts, ec)
        parity_rows = check_n
        if not args.no_cpu_baseline and world == 1:
            try:
                host_rows = rows.cpu().numpy()
                cpu = cpu_baseline_line(host_rows)
                # whole-table parity: the plan's last result (the e2e steps ran it over a copy
                # of this table) against the oracle over the same 60M rows
                fk, fs, fc = plan.result()
                ek, es, ec = oracle_port_fn(cpu_threads())(host_rows)
                ok = ok and np.array_equal(fk, ek) and np.array_equal(fs, es) and np.array_equal(fc, ec)
                parity_rows = n
                del host_rows
            except Exception as e:  # the baseline is reported, never required
                cpu = {"value": None, "unit": "tuples/s", "cores": cpu_threads(), "kind": "port",
                       "sample": "failed: %s" % e}
        result = {
            "metric": METRIC, "value": value, "unit": "tuples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": bench_config(n, world),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "rfx_plan_aggregate (plan-specialised scan_aggregate_kernel<64>)", "kernel_ms": kms,
                         "algorithmic_bytes_per_launch": bytes_alg},
            "cpu_baseline": cpu,
            "e2e": {"value": world * n / (e2e_ms / 1e3), "unit": "tuples/s", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": n * WL.fact_row_bytes(), "d2h_bytes_per_step": d2h},
            "gpu_launches": args.steps,
            "clocks": clocks,
            "parity": ("ok" if ok else "MISMATCH"),
            "parity_rows": parity_rows,
        }
        if world == 1 and not args.no_operators:
            del dev_in_keep
            global PIPELINE_CPU_LEGS
            PIPELINE_CPU_LEGS = not args.no_cpu_baseline
            result["operators"] = operator_benchmarks(dev, rows, peak)
            result["tuning"] = tuning_benchmark(dev, rows)
        if world == 1:
            del rows
            torch.cuda.empty_cache()
            if not args.no_operators:
                result["operators"].update(run_section("strings_f64", args))
            if args.batched_queries > 0:
                result["batched"] = run_section("batched", args)
            if args.serving_queries > 0:
                result["serving"] = run_section("serving", args)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if result is not None:
        print(json.dumps(result), flush=True)
    return 0 if ok else 1


def main_only(args):
    """Selected operator benchmarks alone (profiling and quick measurements)."""
    import torch

    from redfox_b200 import rfx as R
    from redfox_b200 import workloads as WL
    global SORT_ROWS, PIPELINE_CPU_LEGS
    SORT_ROWS = args.sort_rows
    PIPELINE_CPU_LEGS = not args.no_cpu_baseline
    dev = torch.device("cuda:0")
    peak = measured_peak_hbm()[0]
    only = [x for x in args.only.split(",") if x]
    rows = WL.gen_fact(args.rows, device=dev) if "select" in only else None
    out = operator_benchmarks(dev, rows, peak, reps=args.reps, only=only)
    if "strings_f64" in only:
        out.update(string_f64_benchmarks(dev, peak, reps=args.reps))
    torch.cuda.synchronize()
    out["device_status"] = R.device_status()
    print(json.dumps(out), flush=True)
    return 0 if out["device_status"] == R.OK else 1


def main():
    args = parse()
    if args.impl == "reference":
        return main_reference(args)
    if args.section:
        return main_section(args)
    if args.only:
        return main_only(args)
    return main_ours(args)


if __name__ == "__main__":
    sys.exit(main())
