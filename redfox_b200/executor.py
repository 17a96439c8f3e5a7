"""Python face of the native plan executor (rfx_exec_* in librfx.so): JSON plans of RA
operators over named variables, run with liveness-based allocation under a byte budget.
`join_aggregate_plan` and `three_relation_plan` state the benchmark plans in that form."""
import ctypes as C
import json

from . import rfx as R


def _declare():
    L, P, u64, st = R.LIB, C.c_void_p, C.c_uint64, C.c_int
    L.rfx_exec_create.restype = st
    L.rfx_exec_create.argtypes = [C.POINTER(P), C.c_char_p, u64, C.c_char_p, C.c_size_t]
    L.rfx_exec_destroy.restype = None
    L.rfx_exec_destroy.argtypes = [P]
    L.rfx_exec_bind.restype = st
    L.rfx_exec_bind.argtypes = [P, C.c_char_p, P, u64]
    L.rfx_exec_load.restype = st
    L.rfx_exec_load.argtypes = [P, C.c_char_p, C.c_char_p, P]
    L.rfx_exec_run.restype = st
    L.rfx_exec_run.argtypes = [P, P]
    L.rfx_exec_output.restype = st
    L.rfx_exec_output.argtypes = [P, C.c_char_p, C.POINTER(P), C.POINTER(u64), C.POINTER(C.c_uint32)]
    L.rfx_exec_stats.restype = st
    L.rfx_exec_stats.argtypes = [P, C.POINTER(u64), C.POINTER(u64), C.POINTER(u64), C.c_char_p, C.c_size_t]
    L.rfx_exec_copy_out.restype = st
    L.rfx_exec_copy_out.argtypes = [P, C.c_char_p, P, u64, P]
    L.rfx_exec_capture.restype = st
    L.rfx_exec_capture.argtypes = [P, P]
    L.rfx_exec_replay.restype = st
    L.rfx_exec_replay.argtypes = [P, P]


_declare()


class PlanError(RuntimeError):
    pass


class Executor:
    def __init__(self, plan, budget_bytes=0):
        self.plan = plan if isinstance(plan, str) else json.dumps(plan)
        h = C.c_void_p()
        err = C.create_string_buffer(512)
        st = R.LIB.rfx_exec_create(C.byref(h), self.plan.encode(), int(budget_bytes), err, 512)
        if st != R.OK:
            raise PlanError("rfx_exec_create: %d: %s" % (st, err.value.decode()))
        self.h = h
        self._keep = {}

    def close(self):
        if self.h:
            R.LIB.rfx_exec_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, fn, st):
        if st != R.OK:
            raise PlanError("%s: %d: %s" % (fn, st, self.stats()["error"]))

    def bind(self, name, tensor):
        self._keep[name] = tensor
        self._check("rfx_exec_bind", R.LIB.rfx_exec_bind(self.h, name.encode(), R._ptr(tensor),
                                                         tensor.numel() * tensor.element_size()))

    def load(self, name, path, stream=None):
        self._check("rfx_exec_load", R.LIB.rfx_exec_load(self.h, name.encode(), str(path).encode(), R._stream(stream)))

    def run(self, stream=None):
        self._check("rfx_exec_run", R.LIB.rfx_exec_run(self.h, R._stream(stream)))

    def capture(self, stream):
        """Capture the plan as a CUDA graph on `stream` (a torch.cuda.Stream, not the
        default stream); runs it once eagerly first."""
        self._check("rfx_exec_capture", R.LIB.rfx_exec_capture(self.h, R._stream(stream)))

    def replay(self, stream):
        """Launch the captured graph; raises when an intermediate size differs from the
        captured one (RFX_ERR_CAPACITY: run eagerly or capture again)."""
        self._check("rfx_exec_replay", R.LIB.rfx_exec_replay(self.h, R._stream(stream)))

    def output(self, name, stream=None):
        """A copy of the variable's rows as a (rows, row_bytes) uint8 tensor."""
        import torch
        ptr, rows, rb = C.c_void_p(), C.c_uint64(), C.c_uint32()
        self._check("rfx_exec_output", R.LIB.rfx_exec_output(self.h, name.encode(), C.byref(ptr), C.byref(rows),
                                                             C.byref(rb)))
        out = torch.empty((rows.value, rb.value), dtype=torch.uint8, device="cuda")
        self._check("rfx_exec_copy_out", R.LIB.rfx_exec_copy_out(self.h, name.encode(), R._ptr(out),
                                                                 out.numel(), R._stream(stream)))
        return out

    def stats(self):
        a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        err = C.create_string_buffer(512)
        R.LIB.rfx_exec_stats(self.h, C.byref(a), C.byref(b), C.byref(c), err, 512)
        return {"in_use": a.value, "peak": b.value, "ops": c.value, "error": err.value.decode()}


def join_aggregate_plan():
    """plans.join_aggregate as a plan: sort R and S on their keys, join, SUM/COUNT by key."""
    return {
        "variables": {"R": {"row_bytes": 8}, "S": {"row_bytes": 16}, "J": {"row_bytes": 16},
                      "keys": {"row_bytes": 4}, "sums": {"row_bytes": 8}, "counts": {"row_bytes": 4}},
        "outputs": ["keys", "sums", "counts"],
        "ops": [
            {"op": "sort", "rel": "R", "begin_bit": 32, "end_bit": 64},
            {"op": "sort", "rel": "S", "begin_bit": 64, "end_bit": 96},
            {"op": "join", "left": "R", "right": "S", "out": "J", "left_value_bits": 32, "right_value_bits": 64},
            {"op": "reduce", "in": "J", "key_shift": 96, "value_shift": 0, "value_bits": 64,
             "keys": "keys", "sums": "sums", "counts": "counts"},
        ],
    }


def three_relation_plan(segment, date_lo, date_hi, with_lists=True):
    """plans.three_relation as a plan (F sorted inside the plan)."""
    ops = [
        {"op": "select", "in": "D1", "out": "D1s", "widths": [32, 8],
         "cmps": [{"op": "eq", "a": {"field": 1}, "b": {"const": segment}, "type": "i8"}]},
        {"op": "select_project", "in": "D2", "out": "D2s", "widths": [32, 32, 32],
         "cmps": [{"op": "ge", "a": {"field": 2}, "b": {"const": date_lo}, "type": "i32"},
                  {"op": "lt", "a": {"field": 2}, "b": {"const": date_hi}, "type": "i32"}],
         "out_widths": [32, 32], "map": [1, 0]},
        {"op": "sort", "rel": "D2s", "begin_bit": 32, "end_bit": 64},
        {"op": "join", "left": "D1s", "right": "D2s", "out": "J1", "left_value_bits": 8, "right_value_bits": 32},
        {"op": "project", "in": "J1", "out": "K", "widths": [32, 8, 32], "out_widths": [32], "map": [2]},
        {"op": "sort", "rel": "K"},
    ]
    if with_lists:
        ops += [{"op": "set", "kind": "intersection", "a": "K", "b": "Lin", "out": "K2"},
                {"op": "set", "kind": "difference", "a": "K2", "b": "Lout", "out": "K3"}]
    kf = "K3" if with_lists else "K"
    ops += [{"op": "sort", "rel": "F", "begin_bit": 64, "end_bit": 96},
            {"op": "join", "left": kf, "right": "F", "out": "J2", "left_value_bits": 0, "right_value_bits": 64},
            {"op": "reduce", "in": "J2", "key_shift": 64, "value_shift": 0, "value_bits": 64,
             "keys": "keys", "sums": "sums", "counts": "counts"}]
    var = {"D1": 8, "D2": 16, "F": 16, "Lin": 4, "Lout": 4, "D1s": 8, "D2s": 8, "J1": 16, "K": 4, "K2": 4, "K3": 4,
           "J2": 16, "keys": 4, "sums": 8, "counts": 4}
    if not with_lists:
        for k in ("Lin", "Lout", "K2", "K3"):
            var.pop(k)
    return {"variables": {k: {"row_bytes": v} for k, v in var.items()}, "outputs": ["keys", "sums", "counts"],
            "ops": ops}
