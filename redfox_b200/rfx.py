"""ctypes binding of librfx.so, the redfox_b200 C ABI (include/rfx/rfx.h).

Device buffers are torch tensors (plumbing only: memory and streams); every computation
runs in the CUDA kernels of librfx.so.  There is no CPU fallback: if the library is
missing, importing this module raises.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "librfx.so")

OK, ERR_INVALID, ERR_UNSUPPORTED, ERR_CAPACITY, ERR_TIMEOUT, ERR_CUDA, ERR_WORKSPACE = range(7)
STATUS_NAMES = {0: "OK", 1: "INVALID", 2: "UNSUPPORTED", 3: "CAPACITY", 4: "TIMEOUT", 5: "CUDA", 6: "WORKSPACE"}
I8, I16, I32, I64, I128, I256, I512 = range(1, 8)
EQ, NE, SLT, LT, SLE, LE, SGT, GT, SGE, GE = range(1, 11)
OPND_CONST, OPND_VAR = 0, 2
ADD, MUL, SUB, DIV, MOD = range(5)
NODE_OP, NODE_CONST, NODE_INDEX = 0, 1, 2


class RfxError(RuntimeError):
    def __init__(self, fn, code):
        super().__init__("%s failed: RFX_ERR_%s (%d)" % (fn, STATUS_NAMES.get(code, "?"), code))
        self.code = code


class Tuple(C.Structure):
    _fields_ = [("nfields", C.c_uint32), ("widths", C.c_uint32 * 16)]

    @classmethod
    def of(cls, widths):
        t = cls()
        t.nfields = len(widths)
        for i, w in enumerate(widths):
            t.widths[i] = w
        return t


class Cmp(C.Structure):
    _fields_ = [("op", C.c_uint32), ("a_kind", C.c_uint32), ("b_kind", C.c_uint32),
                ("a_field", C.c_uint32), ("b_field", C.c_uint32), ("value_type", C.c_uint32),
                ("a_const", C.c_uint64), ("b_const", C.c_uint64)]


class ArithNode(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("op", C.c_uint32), ("type", C.c_uint32),
                ("left", C.c_int32), ("right", C.c_int32), ("pad", C.c_uint32),
                ("value", C.c_uint64)]


class ArithExpr(C.Structure):
    _fields_ = [("nodes", C.POINTER(ArithNode)), ("nnodes", C.c_uint32), ("root", C.c_uint32),
                ("dest_type", C.c_uint32), ("dest_bits", C.c_uint32)]


def container_bytes(bits):
    for c in (8, 16, 32, 64, 128, 256, 512):
        if bits <= c:
            return c // 8
    raise ValueError("tuples wider than 512 bits are not supported")


def _load():
    if not os.path.exists(_LIB_PATH):
        raise ImportError("redfox_b200/librfx.so is not built; run __graft_entry__.build()")
    lib = C.CDLL(_LIB_PATH)
    P, u32, u64, sz, st = C.c_void_p, C.c_uint32, C.c_uint64, C.c_size_t, C.c_int
    sig = {
        "rfx_device_status": (st, [P]),
        "rfx_version": (C.c_char_p, []),
        "rfx_select_workspace": (sz, [u64, P]),
        "rfx_select": (st, [P, P, P, u64, P, P, u32, P, sz, P]),
        "rfx_arith": (st, [P, P, u64, P, P, P]),
        "rfx_project": (st, [P, P, u64, P, P, P, P]),
        "rfx_select_project": (st, [P, P, P, u64, P, P, u32, P, u32, P, P, P, sz, P]),
        "rfx_filter_aggregate_workspace": (sz, [u64, P, P, u32, u32]),
        "rfx_filter_aggregate": (st, [P, u64, P, P, u32, P, u32, P, P, u32, P, u32, P, P, P, P, P, sz, P]),
        "rfx_gen_uniform_rows": (st, [P, u64, P, u64, P, P, P]),
        "rfx_sort_workspace": (sz, [u64, u32, u32, u32, u32]),
        "rfx_sort_pairs": (st, [P, P, u64, u32, u32, u32, u32, u32, P, sz, P]),
        "rfx_sort_pairs_from": (st, [P, P, P, P, u64, u32, u32, u32, u32, u32, P, sz, P]),
        "rfx_b40c_sort_pair": (st, [P, P, u64, u64, u64]),
        "rfx_b40c_sort_key": (st, [P, u64, u64]),
        "rfx_mgpu_sort_pair": (st, [P, P, u64, u64, u64]),
        "rfx_mgpu_sort_key": (st, [P, u64, u64]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


LIB = _load()


def check(fn, code):
    if code != OK:
        raise RfxError(fn, code)


def declared_symbols():
    """Entry points declared in include/rfx/*.h (parsed from the headers)."""
    import re
    inc = os.path.join(os.path.dirname(_HERE), "include", "rfx")
    names = []
    for h in sorted(os.listdir(inc)):
        if h.endswith(".h"):
            text = open(os.path.join(inc, h)).read()
            names += re.findall(r"^\s*(?:rfx_status|size_t|const char\*|void|uint64_t)\s+(rfx_\w+)\s*\(", text, re.M)
    return names


# ---------------------------------------------------------------------------- helpers
def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def device_status(stream=None):
    """Synchronise the stream and return (and clear) the device error word."""
    return LIB.rfx_device_status(_stream(stream))


def make_cmps(cmps):
    """cmps: list of (op, (kind, field_or_const), (kind, field_or_const), value_type)."""
    arr = (Cmp * max(1, len(cmps)))()
    for i, (op, a, b, vt) in enumerate(cmps):
        arr[i].op, arr[i].value_type = op, vt
        for side, (kind, val) in (("a", a), ("b", b)):
            setattr(arr[i], side + "_kind", kind)
            setattr(arr[i], side + ("_field" if kind == OPND_VAR else "_const"), val)
    return arr


def make_arith(nodes, root, dest_type, dest_bits):
    """nodes: list of (kind, op, type, left, right, value)."""
    arr = (ArithNode * len(nodes))()
    for i, (kind, op, typ, left, right, value) in enumerate(nodes):
        arr[i].kind, arr[i].op, arr[i].type = kind, op, typ
        arr[i].left, arr[i].right, arr[i].value = left, right, value
    e = ArithExpr()
    e.nodes = arr
    e.nnodes, e.root, e.dest_type, e.dest_bits = len(nodes), root, dest_type, dest_bits
    e._keep = arr
    return e


def _arith_array(ariths):
    arr = (ArithExpr * max(1, len(ariths)))()
    for i, a in enumerate(ariths):
        arr[i] = a
    arr._keep = [a._keep for a in ariths]
    return arr


def _empty_bytes(nbytes, device):
    import torch
    return torch.empty(max(1, nbytes), dtype=torch.uint8, device=device)


# ---------------------------------------------------------------------------- entries
def gen_uniform_rows(n, widths, seed, lo, hi, device="cuda", stream=None):
    import torch
    W = container_bytes(sum(widths))
    out = torch.empty((n, W), dtype=torch.uint8, device=device)
    lo_a = (C.c_uint64 * len(widths))(*lo)
    hi_a = (C.c_uint64 * len(widths))(*hi)
    check("rfx_gen_uniform_rows", LIB.rfx_gen_uniform_rows(_ptr(out), n, C.byref(Tuple.of(widths)), seed,
                                                           lo_a, hi_a, _stream(stream)))
    return out


def select(rows, widths, cmps, stream=None):
    """Order-preserving filter; returns (selected rows view, count)."""
    import torch
    n = rows.shape[0]
    t = Tuple.of(widths)
    out = torch.empty_like(rows)
    cnt = torch.zeros(1, dtype=torch.int64, device=rows.device)
    wsb = LIB.rfx_select_workspace(n, C.byref(t))
    ws = _empty_bytes(wsb, rows.device)
    carr = make_cmps(cmps)
    check("rfx_select", LIB.rfx_select(_ptr(out), _ptr(cnt), _ptr(rows), n, C.byref(t), carr, len(cmps),
                                       _ptr(ws), wsb, _stream(stream)))
    k = int(cnt.item())
    return out[:k], k


def arith(rows, widths, expr, stream=None):
    import torch
    n = rows.shape[0]
    W = container_bytes(sum(widths) + expr.dest_bits)
    out = torch.empty((n, W), dtype=torch.uint8, device=rows.device)
    check("rfx_arith", LIB.rfx_arith(_ptr(out), _ptr(rows), n, C.byref(Tuple.of(widths)), C.byref(expr),
                                     _stream(stream)))
    return out


def project(rows, in_widths, out_widths, fmap, stream=None):
    import torch
    n = rows.shape[0]
    W = container_bytes(sum(out_widths))
    out = torch.empty((n, W), dtype=torch.uint8, device=rows.device)
    m = (C.c_uint32 * 16)(*(list(fmap) + [100] * (16 - len(fmap))))
    check("rfx_project", LIB.rfx_project(_ptr(out), _ptr(rows), n, C.byref(Tuple.of(in_widths)),
                                         C.byref(Tuple.of(out_widths)), m, _stream(stream)))
    return out


def select_project(rows, widths, cmps, ariths, out_widths, fmap, stream=None):
    import torch
    n = rows.shape[0]
    t = Tuple.of(widths)
    W = container_bytes(sum(out_widths))
    out = torch.empty((n, W), dtype=torch.uint8, device=rows.device)
    cnt = torch.zeros(1, dtype=torch.int64, device=rows.device)
    wsb = LIB.rfx_select_workspace(n, C.byref(t))
    ws = _empty_bytes(wsb, rows.device)
    m = (C.c_uint32 * 16)(*(list(fmap) + [100] * (16 - len(fmap))))
    check("rfx_select_project", LIB.rfx_select_project(
        _ptr(out), _ptr(cnt), _ptr(rows), n, C.byref(t), make_cmps(cmps), len(cmps), _arith_array(ariths),
        len(ariths), C.byref(Tuple.of(out_widths)), m, _ptr(ws), wsb, _stream(stream)))
    k = int(cnt.item())
    return out[:k], k


class FilterAggregate:
    """A prepared rfx_filter_aggregate call: descriptors, outputs and workspace allocated
    once so that repeated launches (benchmarks, serving) allocate nothing."""

    def __init__(self, n, widths, cmps, ariths, group_fields, group_domain, sum_fields, device="cuda"):
        import torch
        self.n = n
        self.t = Tuple.of(widths)
        self.cmps = make_cmps(cmps)
        self.ncmp = len(cmps)
        self.ariths = _arith_array(ariths)
        self.narith = len(ariths)
        self.gf = (C.c_uint32 * 4)(*group_fields)
        self.gd = (C.c_uint32 * 4)(*group_domain)
        self.ngroup = len(group_fields)
        self.sf = (C.c_uint32 * 4)(*sum_fields)
        self.nsum = len(sum_fields)
        G = 1
        for d in group_domain:
            G *= d
        self.G = G
        self.keys = torch.zeros(G, dtype=torch.int64, device=device)
        self.sums = torch.zeros((G, max(1, self.nsum)), dtype=torch.int64, device=device)
        self.counts = torch.zeros(G, dtype=torch.int64, device=device)
        self.ngroups = torch.zeros(1, dtype=torch.int64, device=device)
        self.wsb = LIB.rfx_filter_aggregate_workspace(n, C.byref(self.t), self.gd, self.ngroup, self.nsum)
        self.ws = _empty_bytes(self.wsb, device)

    def launch(self, rows, n=None, stream=None):
        n = self.n if n is None else n
        check("rfx_filter_aggregate", LIB.rfx_filter_aggregate(
            _ptr(rows), n, C.byref(self.t), self.cmps, self.ncmp, self.ariths, self.narith, self.gf, self.gd,
            self.ngroup, self.sf, self.nsum, _ptr(self.keys), _ptr(self.sums), _ptr(self.counts),
            _ptr(self.ngroups), _ptr(self.ws), self.wsb, _stream(stream)))

    def result(self):
        g = int(self.ngroups.item())
        return (self.keys[:g].cpu().numpy().astype("uint64"), self.sums[:g, :self.nsum].cpu().numpy(),
                self.counts[:g].cpu().numpy().astype("uint64"))


def filter_aggregate(rows, widths, cmps, ariths, group_fields, group_domain, sum_fields, stream=None):
    fa = FilterAggregate(rows.shape[0], widths, cmps, ariths, group_fields, group_domain, sum_fields,
                         device=rows.device)
    fa.launch(rows, stream=stream)
    return fa.result()


# ---------------------------------------------------------------------------- sort
SORT_SKIP_TRIVIAL = 1


def _width(t):
    """Bytes per element of a 1-D (dtype) or 2-D (uint8 rows) tensor."""
    return t.element_size() if t.dim() == 1 else t.shape[1] * t.element_size()


class Sorter:
    """A prepared stable radix sort (workspace allocated once)."""

    def __init__(self, n, key_bytes, value_bytes=0, begin_bit=0, end_bit=None, device="cuda"):
        self.n, self.kb, self.vb = n, key_bytes, value_bytes
        self.begin = begin_bit
        self.end = key_bytes * 8 if end_bit is None else end_bit
        self.wsb = LIB.rfx_sort_workspace(n, key_bytes, value_bytes, self.begin, self.end)
        self.ws = _empty_bytes(self.wsb, device)

    def __call__(self, keys, values=None, flags=0, stream=None, src_keys=None, src_values=None):
        """Sort keys (and values) in place, or, with src_keys (and src_values), sort those
        into keys (and values) and leave them as they are."""
        if src_keys is not None:
            check("rfx_sort_pairs_from", LIB.rfx_sort_pairs_from(
                _ptr(src_keys), _ptr(src_values), _ptr(keys), _ptr(values), self.n, self.kb, self.vb, self.begin,
                self.end, flags, _ptr(self.ws), self.wsb, _stream(stream)))
            return
        check("rfx_sort_pairs", LIB.rfx_sort_pairs(_ptr(keys), _ptr(values), self.n, self.kb, self.vb, self.begin,
                                                   self.end, flags, _ptr(self.ws), self.wsb, _stream(stream)))


def sort_pairs(keys, values=None, begin_bit=0, end_bit=None, flags=0, stream=None):
    """Sort keys (and values) in place; returns them."""
    n = keys.shape[0]
    s = Sorter(n, _width(keys), 0 if values is None else _width(values), begin_bit, end_bit, device=keys.device)
    s(keys, values, flags, stream)
    return keys, values


def sorted_copy(keys, values=None, begin_bit=0, end_bit=None, flags=0, stream=None):
    """New tensors holding keys (and values) sorted; the inputs are left as they are."""
    import torch
    n = keys.shape[0]
    out_k = torch.empty_like(keys)
    out_v = None if values is None else torch.empty_like(values)
    s = Sorter(n, _width(keys), 0 if values is None else _width(values), begin_bit, end_bit, device=keys.device)
    s(out_k, out_v, flags, stream, src_keys=keys, src_values=values)
    return out_k, out_v


# ---------------------------------------------------------------------------- reduce
VAL_NONE, VAL_U32, VAL_I64 = 0, 1, 2


def _declare_more():
    P, u32, u64, sz, st = C.c_void_p, C.c_uint32, C.c_uint64, C.c_size_t, C.c_int
    more = {
        "rfx_reduce_by_key_workspace": (sz, [u64]),
        "rfx_reduce_by_key": (st, [P, u64, P, u32, P, u32, P, P, P, P, P, sz, P]),
        "rfx_count_compat": (st, [P, P, P, P, P, P, u32]),
        "rfx_total_64_32_compat": (st, [P, P, P, P, P, P]),
        "rfx_total_i64_compat": (st, [P, P, P, P, P, P, u32]),
    }
    for name, (res, args) in more.items():
        f = getattr(LIB, name)
        f.restype = res
        f.argtypes = args


_declare_more()


def reduce_by_key(keys, values=None, value_kind=None, counts=True, d_n=None, stream=None):
    """Runs of equal keys -> (out_keys, out_sums or None, out_counts or None, groups)."""
    import torch
    n = keys.shape[0]
    kb = _width(keys)
    if value_kind is None:
        value_kind = VAL_NONE if values is None else (VAL_I64 if values.element_size() == 8 else VAL_U32)
    out_k = torch.empty_like(keys)
    out_v = None
    if value_kind != VAL_NONE:
        out_v = torch.empty(n, dtype=torch.int64 if value_kind == VAL_I64 else torch.int32, device=keys.device)
    out_c = torch.empty(n, dtype=torch.int32, device=keys.device) if counts else None
    g = torch.zeros(1, dtype=torch.int64, device=keys.device)
    wsb = LIB.rfx_reduce_by_key_workspace(n)
    ws = _empty_bytes(wsb, keys.device)
    check("rfx_reduce_by_key", LIB.rfx_reduce_by_key(_ptr(keys), n, _ptr(d_n), kb, _ptr(values), value_kind,
                                                     _ptr(out_k), _ptr(out_v), _ptr(out_c), _ptr(g), _ptr(ws), wsb,
                                                     _stream(stream)))
    k = int(g.item())
    return out_k[:k], (out_v[:k] if out_v is not None else None), (out_c[:k] if out_c is not None else None), k


# ---------------------------------------------------------------------------- join / set ops
SET_UNION, SET_DIFFERENCE, SET_INTERSECTION = 0, 1, 2


def _declare_join():
    P, u32, u64, sz, st = C.c_void_p, C.c_uint32, C.c_uint64, C.c_size_t, C.c_int
    more = {
        "rfx_join_find_bounds_workspace": (sz, [u64]),
        "rfx_join_find_bounds": (st, [P, P, P, P, u64, P, u64, u32, P, sz, P]),
        "rfx_join_expand": (st, [P, P, u64, P, P, P, u64, P]),
        "rfx_join_gather": (st, [P, u32, u64, P, P, P, P, u32, P, u32, u32, P, u32, u32, P]),
        "rfx_join_tuples_workspace": (sz, [u64]),
        "rfx_join_tuples": (st, [P, u32, u64, P, P, u64, u32, u32, P, u64, u32, u32, P, sz, P]),
        "rfx_find_bounds_compat": (st, [P, P, P, P, u64, P, u64, u32]),
        "rfx_join_compat": (st, [P, P, u64, P, P, u64]),
        "rfx_set_op_workspace": (sz, [u32, u64, u64, u32]),
        "rfx_set_op": (st, [u32, P, P, P, u64, P, u64, u32, P, sz, P]),
        "rfx_unique_workspace": (sz, [u64, u32]),
        "rfx_unique": (st, [P, u64, P, u32, P, sz, P]),
        "rfx_set_union_compat": (st, [P, P, P, P, P, P, u32]),
        "rfx_difference_compat": (st, [P, P, P, P, P, P, u32]),
        "rfx_intersection_compat": (st, [P, P, P, P, P, P, u32]),
        "rfx_unique_compat": (st, [P, P, u64]),
    }
    for name, (res, args) in more.items():
        f = getattr(LIB, name)
        f.restype = res
        f.argtypes = args


_declare_join()


def find_bounds(left, right, stream=None):
    import torch
    nl, nr = left.shape[0], right.shape[0]
    kb = _width(left)
    lb = torch.empty(nl, dtype=torch.int32, device=left.device)
    sc = torch.empty(nl, dtype=torch.int32, device=left.device)
    tot = torch.zeros(1, dtype=torch.int64, device=left.device)
    wsb = LIB.rfx_join_find_bounds_workspace(nl)
    ws = _empty_bytes(wsb, left.device)
    check("rfx_join_find_bounds", LIB.rfx_join_find_bounds(_ptr(lb), _ptr(sc), _ptr(tot), _ptr(left), nl, _ptr(right),
                                                           nr, kb, _ptr(ws), wsb, _stream(stream)))
    return lb, sc, int(tot.item())


def join_expand(lb, scan, nout, stream=None):
    import torch
    li = torch.empty(max(1, nout), dtype=torch.int32, device=lb.device)
    ri = torch.empty(max(1, nout), dtype=torch.int32, device=lb.device)
    check("rfx_join_expand", LIB.rfx_join_expand(_ptr(li), _ptr(ri), nout, None, _ptr(lb), _ptr(scan), lb.shape[0],
                                                 _stream(stream)))
    return li[:nout], ri[:nout]


def join_gather(out_bytes, li, ri, lkey, lval, lval_bits, rval, rval_bits, stream=None):
    import torch
    n = li.shape[0]
    out = torch.empty((max(1, n), out_bytes), dtype=torch.uint8, device=li.device)
    check("rfx_join_gather", LIB.rfx_join_gather(
        _ptr(out), out_bytes, n, None, _ptr(li), _ptr(ri), _ptr(lkey), _width(lkey), _ptr(lval),
        _width(lval) if lval is not None else 0, lval_bits, _ptr(rval), _width(rval) if rval is not None else 0,
        rval_bits, _stream(stream)))
    return out[:n]


class TupleJoin:
    """A prepared fused tuple join (workspace allocated once)."""

    def __init__(self, nl, device="cuda"):
        self.wsb = LIB.rfx_join_tuples_workspace(nl)
        self.ws = _empty_bytes(self.wsb, device)
        import torch
        self.count = torch.zeros(1, dtype=torch.int64, device=device)

    def __call__(self, out, capacity, left, lvbits, right, rvbits, stream=None):
        check("rfx_join_tuples", LIB.rfx_join_tuples(_ptr(out), _width(out), capacity, _ptr(self.count), _ptr(left),
                                                     left.shape[0], _width(left), lvbits, _ptr(right), right.shape[0],
                                                     _width(right), rvbits, _ptr(self.ws), self.wsb, _stream(stream)))


def join_tuples(left, lvbits, right, rvbits, out_bytes, capacity=None, stream=None):
    """Returns (rows, total).  With capacity None the count is taken first (two calls)."""
    import torch
    tj = TupleJoin(left.shape[0], device=left.device)
    if capacity is None:
        dummy = torch.empty((1, out_bytes), dtype=torch.uint8, device=left.device)
        tj(dummy, 0, left, lvbits, right, rvbits, stream)
        capacity = int(tj.count.item())
    out = torch.empty((max(1, capacity), out_bytes), dtype=torch.uint8, device=left.device)
    tj(out, capacity, left, lvbits, right, rvbits, stream)
    total = int(tj.count.item())
    return out[:min(total, capacity)], total


def set_op(op, a, b, stream=None):
    import torch
    na, nb = a.shape[0], b.shape[0]
    e = _width(a)
    out = torch.empty((max(1, na + nb),) + tuple(a.shape[1:]), dtype=a.dtype, device=a.device)
    cnt = torch.zeros(1, dtype=torch.int64, device=a.device)
    wsb = LIB.rfx_set_op_workspace(op, na, nb, e)
    ws = _empty_bytes(wsb, a.device)
    check("rfx_set_op", LIB.rfx_set_op(op, _ptr(out), _ptr(cnt), _ptr(a), na, _ptr(b), nb, e, _ptr(ws), wsb,
                                       _stream(stream)))
    k = int(cnt.item())
    return out[:k]


def unique(data, stream=None):
    """In place; returns the kept prefix."""
    import torch
    n = data.shape[0]
    e = _width(data)
    cnt = torch.zeros(1, dtype=torch.int64, device=data.device)
    wsb = LIB.rfx_unique_workspace(n, e)
    ws = _empty_bytes(wsb, data.device)
    check("rfx_unique", LIB.rfx_unique(_ptr(data), n, _ptr(cnt), e, _ptr(ws), wsb, _stream(stream)))
    return data[:int(cnt.item())]


def _declare_tuple_ops():
    P, u32, u64, sz, st = C.c_void_p, C.c_uint32, C.c_uint64, C.c_size_t, C.c_int
    more = {
        "rfx_reduce_tuples": (st, [P, u64, P, u32, u32, u32, u32, P, u32, P, P, P, P, sz, P]),
        "rfx_join_tuples_emit": (st, [P, u32, u64, P, u64, u32, P, u64, u32, u32, P, sz, P]),
        "rfx_multi_select_workspace": (sz, [u64]),
        "rfx_multi_select": (st, [P, u64, P, P, u64, u32, u32, u32, P, P, u32, u32, u32, u32, u32, P, sz, P]),
        "rfx_join_aggregate_workspace": (sz, [u64, u32]),
        "rfx_join_aggregate": (st, [P, u64, u32, u32, P, u64, u32, u32, u32, u32, P, u32, P, P, P, P, sz, P]),
    }
    for name, (res, args) in more.items():
        f = getattr(LIB, name)
        f.restype = res
        f.argtypes = args


_declare_tuple_ops()


def reduce_tuples(rows, key_shift, value_shift, value_bits, out_key_bytes, n=None, d_n=None, stream=None):
    """Runs of equal keys (row >> key_shift) of packed rows -> (keys, sums, counts, groups)."""
    import torch
    n = rows.shape[0] if n is None else n
    kdt = {4: torch.int32, 8: torch.int64}.get(out_key_bytes)
    keys = (torch.empty(max(1, n), dtype=kdt, device=rows.device) if kdt is not None
            else torch.empty((max(1, n), 16), dtype=torch.uint8, device=rows.device))
    sums = torch.empty(max(1, n), dtype=torch.int64, device=rows.device)
    counts = torch.empty(max(1, n), dtype=torch.int32, device=rows.device)
    g = torch.zeros(1, dtype=torch.int64, device=rows.device)
    wsb = LIB.rfx_reduce_by_key_workspace(n)
    ws = _empty_bytes(wsb, rows.device)
    check("rfx_reduce_tuples", LIB.rfx_reduce_tuples(_ptr(rows), n, _ptr(d_n), _width(rows), key_shift, value_shift,
                                                     value_bits, _ptr(keys), out_key_bytes, _ptr(sums), _ptr(counts),
                                                     _ptr(g), _ptr(ws), wsb, _stream(stream)))
    k = int(g.item())
    return keys[:k], sums[:k], counts[:k], k


def join_tuples_two_step(left, lvbits, right, rvbits, out_bytes, stream=None):
    """Count, read the size back, allocate exactly, emit (the reference's shape)."""
    import torch
    tj = TupleJoin(left.shape[0], device=left.device)
    dummy = torch.empty((1, out_bytes), dtype=torch.uint8, device=left.device)
    tj(dummy, 0, left, lvbits, right, rvbits, stream)
    total = int(tj.count.item())
    out = torch.empty((max(1, total), out_bytes), dtype=torch.uint8, device=left.device)
    check("rfx_join_tuples_emit", LIB.rfx_join_tuples_emit(
        _ptr(out), out_bytes, total, _ptr(left), left.shape[0], _width(left), _ptr(right), right.shape[0],
        _width(right), rvbits, _ptr(tj.ws), tj.wsb, _stream(stream)))
    return out[:total], total


def multi_select(rows, field, bounds, key, val, capacity=None, stream=None):
    """One scan of `rows` for many range selections: bounds = [(lo, hi), ...] (at most 256
    queries); field / key / val = (shift, width) bit fields of a row.  Returns the 8-byte
    rows ((key << 8 | q) << val_width) | val in (row, query) order (int64 tensor) and
    their number.  With capacity None the count is taken first (two calls)."""
    import torch
    n = rows.shape[0]
    nq = len(bounds)
    lo = (C.c_uint32 * nq)(*[b[0] for b in bounds])
    hi = (C.c_uint32 * nq)(*[b[1] for b in bounds])
    cnt = torch.zeros(1, dtype=torch.int64, device=rows.device)
    wsb = LIB.rfx_multi_select_workspace(n)
    ws = _empty_bytes(wsb, rows.device)

    def call(out, cap):
        check("rfx_multi_select", LIB.rfx_multi_select(
            _ptr(out), cap, _ptr(cnt), _ptr(rows), n, _width(rows), field[0], field[1], lo, hi, nq, key[0], key[1],
            val[0], val[1], _ptr(ws), wsb, _stream(stream)))
    if capacity is None:
        call(None, 0)
        capacity = int(cnt.item())
    out = torch.empty(max(1, capacity), dtype=torch.int64, device=rows.device)
    call(out, capacity)
    k = int(cnt.item())
    return out[:min(k, capacity)], k


class JoinAggregate:
    """A prepared rfx_join_aggregate (join on the key + SUM(right value) and COUNT per key,
    no join rows written): outputs of capacity nr and the workspace allocated once, sizes
    stay on the device, so repeated calls allocate nothing and can be graph-captured."""

    def __init__(self, nr, out_key_bytes=4, device="cuda"):
        import torch
        self.nr = nr
        self.kb = out_key_bytes
        self.keys = torch.empty(max(1, nr), dtype={4: torch.int32, 8: torch.int64}[out_key_bytes], device=device)
        self.sums = torch.empty(max(1, nr), dtype=torch.int64, device=device)
        self.counts = torch.empty(max(1, nr), dtype=torch.int32, device=device)
        self.groups = torch.zeros(1, dtype=torch.int64, device=device)
        self.wsb = LIB.rfx_join_aggregate_workspace(nr, out_key_bytes)
        self.ws = _empty_bytes(self.wsb, device)

    def __call__(self, left, lvbits, right, rvbits, value_shift, value_bits, stream=None):
        assert right.shape[0] <= self.nr
        check("rfx_join_aggregate", LIB.rfx_join_aggregate(
            _ptr(left), left.shape[0], _width(left), lvbits, _ptr(right), right.shape[0], _width(right), rvbits,
            value_shift, value_bits, _ptr(self.keys), self.kb, _ptr(self.sums), _ptr(self.counts), _ptr(self.groups),
            _ptr(self.ws), self.wsb, _stream(stream)))

    def result(self):
        g = int(self.groups.item())
        return self.keys[:g], self.sums[:g], self.counts[:g]


def join_aggregate(left, lvbits, right, rvbits, value_shift, value_bits, out_key_bytes=4, stream=None):
    """(keys, sums, counts) of the join of left and right on their keys, aggregated on the key."""
    ja = JoinAggregate(right.shape[0], out_key_bytes, device=left.device)
    ja(left, lvbits, right, rvbits, value_shift, value_bits, stream)
    return ja.result()


# ---------------------------------------------------------------- autotuning
def _declare_tune():
    LIB.rfx_tune_set.restype = None
    LIB.rfx_tune_set.argtypes = [C.c_int]
    LIB.rfx_tune_reset.restype = None
    LIB.rfx_tune_reset.argtypes = []
    LIB.rfx_tune_force.restype = None
    LIB.rfx_tune_force.argtypes = [C.c_uint32, C.c_int]
    LIB.rfx_tune_dump.restype = C.c_size_t
    LIB.rfx_tune_dump.argtypes = [C.c_char_p, C.c_size_t]


_declare_tune()

TUNE_OPS = {1: "reduce_tuples", 2: "set_filter", 3: "select_compact", 4: "filter_aggregate", 5: "sort_pass",
            6: "join_emit"}
TUNE_JOIN_EMIT = 6   # variants: 0 operands staged in shared memory by bulk copies, 1 gathered per output
TUNE_SORT_PASS = 5   # variants: 0 per-tile pass, 1 / 2 / 3 pipelined onesweep pass (three tile sizes),
#                      4 per-tile pass ranking with match_any


def tune(mode=1):
    """1: time each operator variant on first use per (shape, size class) and keep the
    fastest; 0: run the defaults."""
    LIB.rfx_tune_set(int(mode))


def tune_force(op, variant):
    """Pin operator `op` (a TUNE_OPS key) to a variant; variant < 0 unpins it."""
    LIB.rfx_tune_force(op, variant)


def tune_reset():
    LIB.rfx_tune_reset()


def tune_table():
    """The tuning decisions: list of dicts (op, shape, size_class, variant, ms per variant)."""
    need = LIB.rfx_tune_dump(None, 0)
    buf = C.create_string_buffer(need)
    LIB.rfx_tune_dump(buf, need)
    out = []
    for line in buf.value.decode().splitlines():
        kv = dict(p.split("=", 1) for p in line.split())
        out.append({"op": TUNE_OPS.get(int(kv["op"]), kv["op"]), "shape": kv["shape"],
                    "size_class": int(kv["class"]), "variant": int(kv["variant"]),
                    "ms": [float(x) for x in kv["ms"].split(",") if x]})
    return out


# ---------------------------------------------------------------------------- string keys
def _declare_strings():
    P, u64, st = C.c_void_p, C.c_uint64, C.c_int
    more = {
        "rfx_string_codes": (st, [P, u64, P, P, P, P]),
        "rfx_sort_string_compat": (st, [P, P, u64, u64]),
        "rfx_find_bounds_string_compat": (st, [P, P, P, P, u64, P, u64]),
        "rfx_count_string_compat": (st, [P, P, P, P, P, P]),
    }
    for name, (res, args) in more.items():
        f = getattr(LIB, name)
        f.restype = res
        f.argtypes = args


_declare_strings()


def string_column(pool, offs, device="cuda"):
    """A host string column (uint8 pool of NUL-terminated strings, uint64 offsets) on the
    device: (dpool, ptrs), ptrs an int64 tensor of the strings' device addresses.  The
    column lives as long as dpool does."""
    import numpy as np
    import torch
    dpool = torch.from_numpy(np.ascontiguousarray(pool, np.uint8)).to(device)
    ptrs = torch.from_numpy(np.ascontiguousarray(offs, np.uint64).view(np.int64)).to(device) + dpool.data_ptr()
    return dpool, ptrs


def string_codes(ptrs, stream=None):
    """(codes, perm, distinct): per element the rank of its string among the distinct
    strings, the stable sorted order, and the number of distinct strings (int32 tensors
    holding u32 values)."""
    import torch
    n = ptrs.shape[0]
    codes = torch.empty(n, dtype=torch.int32, device=ptrs.device)
    perm = torch.empty(n, dtype=torch.int32, device=ptrs.device)
    d = C.c_uint64(0)
    check("rfx_string_codes", LIB.rfx_string_codes(_ptr(ptrs), n, _ptr(codes), _ptr(perm), C.byref(d),
                                                   _stream(stream)))
    return codes, perm, d.value


def sort_strings(ptrs, values=None, value_type=0):
    """sort_string_key / sort_string_pair in place (values: value_type a DataType code)."""
    check("rfx_sort_string_compat", LIB.rfx_sort_string_compat(_ptr(ptrs), _ptr(values), ptrs.shape[0],
                                                               value_type))


def find_bounds_string(left, right):
    """find_bounds_string: (lower_bound, left_count scan, total) over sorted pointer columns."""
    import torch
    nl = left.shape[0]
    lb = torch.empty(nl, dtype=torch.int32, device=left.device)
    sc = torch.empty(nl, dtype=torch.int32, device=left.device)
    tot = torch.zeros(1, dtype=torch.int64, device=left.device)
    check("rfx_find_bounds_string_compat",
          LIB.rfx_find_bounds_string_compat(_ptr(lb), _ptr(sc), _ptr(tot), _ptr(left), nl, _ptr(right),
                                            right.shape[0]))
    return lb, sc, int(tot.item())


def count_string(ptrs, values):
    """count_string: (first pointer of each run of equal strings, u32 sums as int32)."""
    import torch
    n = ptrs.shape[0]
    ok = torch.empty(max(n, 1), dtype=torch.int64, device=ptrs.device)
    ov = torch.empty(max(n, 1), dtype=torch.int32, device=ptrs.device)
    ks = torch.tensor([8 * n], dtype=torch.int64, device=ptrs.device)
    vs = torch.tensor([4 * n], dtype=torch.int64, device=ptrs.device)
    check("rfx_count_string_compat", LIB.rfx_count_string_compat(_ptr(ptrs), _ptr(values), _ptr(ok), _ptr(ov),
                                                                 _ptr(ks), _ptr(vs)))
    g = int(ks.item()) // 8
    assert int(vs.item()) // 4 == g
    return ok[:g], ov[:g]


# ---------------------------------------------------------------------------- double values
F64_SUM, F64_MIN = 0, 1


def _declare_f64():
    P, u32, u64, sz, st = C.c_void_p, C.c_uint32, C.c_uint64, C.c_size_t, C.c_int
    more = {
        "rfx_reduce_f64_workspace": (sz, [u64]),
        "rfx_reduce_f64": (st, [P, u64, u32, P, u32, P, P, P, P, sz, P]),
        "rfx_total_double_compat": (st, [P, P, P, P, P, P, u32]),
        "rfx_total_string_double_compat": (st, [P, P, P, P, P, P]),
        "rfx_min_32_double_compat": (st, [P, P, P, P, P, P]),
        "rfx_sum_double_compat": (st, [P, P, P]),
        "rfx_max_double_compat": (st, [P, P, P]),
        "rfx_count_u32_compat": (st, [P, P, P]),
    }
    for name, (res, args) in more.items():
        f = getattr(LIB, name)
        f.restype = res
        f.argtypes = args


_declare_f64()


def reduce_f64(keys, values, op=F64_SUM, stream=None):
    """Runs of equal keys (None: one run) over float64 values -> (out_keys or None,
    out_values, groups).  SUM is the exact sum rounded once; MIN the reference's fold."""
    import torch
    n = values.shape[0]
    kb = 0 if keys is None else _width(keys)
    out_k = None if keys is None else torch.empty_like(keys)
    out_v = torch.empty(max(n, 1), dtype=torch.float64, device=values.device)
    g = torch.zeros(1, dtype=torch.int64, device=values.device)
    wsb = LIB.rfx_reduce_f64_workspace(n)
    ws = _empty_bytes(wsb, values.device)
    check("rfx_reduce_f64", LIB.rfx_reduce_f64(_ptr(keys), n, kb, _ptr(values), op, _ptr(out_k), _ptr(out_v), _ptr(g),
                                               _ptr(ws), wsb, _stream(stream)))
    k = int(g.item())
    return (out_k[:k] if out_k is not None else None), out_v[:k], k
