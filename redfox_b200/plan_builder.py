"""Python face of the native plan builder (rfx_plan_* in librfx.so): relational-algebra
operators over named relations lowered to an executor plan, as the reference's
RelationalAlgebraCompiler lowers them to kernel sequences.  `join_aggregate_ra` and
`three_relation_ra` state the two benchmark queries as RA."""
import ctypes as C
import json

from . import rfx as R

AGG_COUNT, AGG_TOTAL = 0, 1


def _declare():
    L, P, u32, st = R.LIB, C.c_void_p, C.c_uint32, C.c_int
    cs = C.c_char_p
    U32P = C.POINTER(u32)
    sig = {
        "rfx_plan_create": (st, [C.POINTER(P)]),
        "rfx_plan_destroy": (None, [P]),
        "rfx_plan_error": (cs, [P]),
        "rfx_plan_relation": (st, [P, cs, U32P, u32, u32]),
        "rfx_plan_select": (st, [P, cs, cs, P, u32]),
        "rfx_plan_project": (st, [P, cs, cs, U32P, u32]),
        "rfx_plan_join": (st, [P, cs, cs, cs, u32]),
        "rfx_plan_agg": (st, [P, cs, cs, U32P, u32, u32, u32]),
        "rfx_plan_set": (st, [P, cs, cs, cs, u32]),
        "rfx_plan_unique": (st, [P, cs]),
        "rfx_plan_output": (st, [P, cs]),
        "rfx_plan_json": (C.c_size_t, [P, C.c_char_p, C.c_size_t]),
        "rfx_plan_schema": (st, [P, cs, U32P, U32P, U32P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


_declare()


class PlanBuildError(ValueError):
    pass


def _u32s(v):
    v = list(v)
    return (C.c_uint32 * max(1, len(v)))(*v), len(v)


class PlanBuilder:
    def __init__(self):
        h = C.c_void_p()
        R.check("rfx_plan_create", R.LIB.rfx_plan_create(C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            R.LIB.rfx_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ok(self, fn, st):
        if st != R.OK:
            raise PlanBuildError("%s: %d: %s" % (fn, st, R.LIB.rfx_plan_error(self.h).decode()))
        return self

    def relation(self, name, widths, sorted_fields=0):
        a, n = _u32s(widths)
        return self._ok("relation", R.LIB.rfx_plan_relation(self.h, name.encode(), a, n, sorted_fields))

    def select(self, dest, src, cmps):
        """cmps: [(op, (kind, field_or_const), (kind, field_or_const), value_type)] (ANDed)."""
        arr = R.make_cmps(cmps)
        return self._ok("select", R.LIB.rfx_plan_select(self.h, dest.encode(), src.encode(), C.cast(arr, C.c_void_p),
                                                        len(cmps)))

    def project(self, dest, src, fields):
        a, n = _u32s(fields)
        return self._ok("project", R.LIB.rfx_plan_project(self.h, dest.encode(), src.encode(), a, n))

    def join(self, dest, a, b, keycount=1):
        return self._ok("join", R.LIB.rfx_plan_join(self.h, dest.encode(), a.encode(), b.encode(), keycount))

    def agg(self, dest, src, domains, tag, field=0):
        a, n = _u32s(domains)
        return self._ok("agg", R.LIB.rfx_plan_agg(self.h, dest.encode(), src.encode(), a, n, tag, field))

    def set_op(self, dest, a, b, kind):
        return self._ok("set", R.LIB.rfx_plan_set(self.h, dest.encode(), a.encode(), b.encode(), kind))

    def unique(self, name):
        return self._ok("unique", R.LIB.rfx_plan_unique(self.h, name.encode()))

    def output(self, *names):
        for name in names:
            self._ok("output", R.LIB.rfx_plan_output(self.h, name.encode()))
        return self

    def json(self):
        need = R.LIB.rfx_plan_json(self.h, None, 0)
        buf = C.create_string_buffer(need)
        R.LIB.rfx_plan_json(self.h, buf, need)
        return buf.value.decode()

    def plan(self):
        return json.loads(self.json())

    def schema(self, name):
        w = (C.c_uint32 * 16)()
        n, s = C.c_uint32(), C.c_uint32()
        self._ok("schema", R.LIB.rfx_plan_schema(self.h, name.encode(), w, C.byref(n), C.byref(s)))
        return list(w[:n.value]), s.value


def join_aggregate_ra():
    """R(key, payload) join S(key, amount) on key, then SUM(amount) and COUNT(*) by key."""
    b = PlanBuilder()
    b.relation("R", [32, 32]).relation("S", [32, 64])
    b.join("J", "R", "S", 1)                      # J = (key, payload, amount)
    b.agg("T", "J", [0], AGG_TOTAL, 2)             # T = (key, SUM(amount))
    b.agg("C", "J", [0], AGG_COUNT)                # C = (key, COUNT), shares T's reduce
    return b.output("T", "C")


def three_relation_ra(segment, date_lo, date_hi, with_lists=True):
    """D1(id, seg) with seg = segment, D2(id, fk, date) with date in [lo, hi), joined on
    D1.id = D2.fk; the D2 ids (intersected with Lin, minus Lout) join F(fk, amount);
    SUM(amount) and COUNT by fk."""
    b = PlanBuilder()
    b.relation("D1", [32, 8], sorted_fields=1).relation("D2", [32, 32, 32], sorted_fields=1)
    b.relation("F", [32, 64])
    b.select("D1s", "D1", [(R.EQ, (R.OPND_VAR, 1), (R.OPND_CONST, segment), R.I8)])
    b.select("D2f", "D2", [(R.GE, (R.OPND_VAR, 2), (R.OPND_CONST, date_lo), R.I32),
                           (R.LT, (R.OPND_VAR, 2), (R.OPND_CONST, date_hi), R.I32)])
    b.project("D2s", "D2f", [1, 0])               # (fk, id)
    b.join("J1", "D1s", "D2s", 1)                 # (id, seg, d2 id)
    b.project("K", "J1", [2])
    key = "K"
    if with_lists:
        b.relation("Lin", [32], sorted_fields=1).relation("Lout", [32], sorted_fields=1)
        b.set_op("K2", "K", "Lin", R.SET_INTERSECTION)
        b.set_op("K3", "K2", "Lout", R.SET_DIFFERENCE)
        key = "K3"
    b.join("J2", key, "F", 1)                     # (fk, amount)
    b.agg("T", "J2", [0], AGG_TOTAL, 1)
    b.agg("C", "J2", [0], AGG_COUNT)
    return b.output("T", "C")
