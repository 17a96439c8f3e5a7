"""ctypes/numpy binding of the C oracle (test infrastructure; see oracle/__init__.py)."""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

I8, I16, I32, I64, I128 = 1, 2, 3, 4, 5
EQ, NE, SLT, LT, SLE, LE, SGT, GT, SGE, GE = range(1, 11)
OPND_CONST, OPND_VAR = 0, 2
ADD, MUL, SUB, DIV, MOD = range(5)
NODE_OP, NODE_CONST, NODE_INDEX = 0, 1, 2


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


class Node(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("op", C.c_uint32), ("type", C.c_uint32),
                ("left", C.c_int32), ("right", C.c_int32), ("pad", C.c_uint32),
                ("value", C.c_uint64)]


class Arith(C.Structure):
    _fields_ = [("nodes", C.POINTER(Node)), ("nnodes", C.c_uint32), ("root", C.c_uint32),
                ("dest_type", C.c_uint32), ("dest_bits", C.c_uint32)]


def container_bytes(bits):
    for c in (8, 16, 32, 64, 128, 256, 512):
        if bits <= c:
            return c // 8
    raise ValueError("tuples wider than 512 bits are not supported")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so"])
        _LIB = C.CDLL(path)
        _declare(_LIB)
    return _LIB


def ref_lib():
    """The reference's own entry files built for the CPU, or None when absent."""
    global _REF
    if _REF is None:
        path = os.path.join(_HERE, "_ref", "libredfox_ref.so")
        if not os.path.exists(path):
            return None
        _REF = C.CDLL(path)
    return _REF


def _declare(L):
    P, u32, u64, i64, sz = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int64, C.c_size_t
    sig = {
        "orc_pack_rows": (None, [P, sz, P, P]),
        "orc_unpack_rows": (None, [P, sz, P, P]),
        "orc_sort_pairs_mt": (None, [P, P, sz, u32, u32, u32, u32, C.c_int]),
        "orc_find_bounds": (None, [P, P, P, P, sz, P, sz, u32]),
        "orc_join_expand": (None, [P, P, u64, P, P, sz]),
        "orc_join_gather": (None, [P, u32, u64, P, P, P, u32, P, u32, u32, P, u32, u32]),
        "orc_join_tuples": (u64, [P, u32, u64, P, sz, u32, u32, P, sz, u32, u32]),
        "orc_reduce_sum_i64": (u64, [P, sz, u32, P, P, P]),
        "orc_reduce_count": (u64, [P, sz, u32, P, P, P]),
        "orc_set_union": (u64, [P, P, sz, P, sz, u32]),
        "orc_set_difference": (u64, [P, P, sz, P, sz, u32]),
        "orc_set_intersection": (u64, [P, P, sz, P, sz, u32]),
        "orc_unique": (u64, [P, sz, u32]),
        "orc_select": (u64, [P, P, sz, P, P, u32]),
        "orc_arith_rows": (C.c_int, [P, P, sz, P, P]),
        "orc_project": (None, [P, P, sz, P, P, P]),
        "orc_filter_aggregate": (i64, [P, sz, P, P, u32, P, u32, P, u32, P, u32, P, P, P, u64, C.c_int]),
        "orc_str_sort": (None, [P, P, sz, P, u32]),
        "orc_str_find_bounds": (None, [P, P, P, P, P, sz, P, sz]),
        "orc_str_count": (u64, [P, P, sz, P, P, P]),
        "orc_str_codes": (u64, [P, P, sz, P]),
        "orc_reduce_f64_seq": (u64, [P, sz, u32, P, P, P, C.c_int]),
        "orc_rand": (u64, [u64, u64, u64]),
        "orc_uniform": (u64, [u64, u64, u64, u64, u64]),
        "orc_gen_uniform_u64": (None, [P, sz, u64, u64, u64, u64, C.c_int]),
        "orc_zipf_cdf": (None, [P, sz, C.c_double]),
        "orc_gen_zipf_u64": (None, [P, sz, u64, u64, P, sz, C.c_int]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _threads():
    return os.cpu_count() or 1


# ---------------------------------------------------------------- codec
def pack(widths, cols):
    """Pack field columns (uint64 arrays) into a byte matrix [n, container_bytes]."""
    t = Tuple.of(widths)
    n = len(cols[0])
    W = container_bytes(sum(widths))
    cols = [np.ascontiguousarray(c, dtype=np.uint64) for c in cols]
    ptrs = (C.c_void_p * len(cols))(*[c.ctypes.data for c in cols])
    out = np.zeros((n, W), dtype=np.uint8)
    lib().orc_pack_rows(_p(out), n, C.byref(t), ptrs)
    return out


def unpack(widths, rows):
    t = Tuple.of(widths)
    rows = np.ascontiguousarray(rows, dtype=np.uint8)
    n = rows.shape[0]
    cols = [np.zeros(n, dtype=np.uint64) for _ in widths]
    ptrs = (C.c_void_p * len(cols))(*[c.ctypes.data for c in cols])
    lib().orc_unpack_rows(_p(rows), n, C.byref(t), ptrs)
    return cols


# ---------------------------------------------------------------- sort
def sort_pairs(keys, vals=None, begin_bit=0, end_bit=None, threads=1):
    """Stable LSD sort of a [n, kbytes] (or 1-D unsigned) key array, in place copy."""
    k = np.ascontiguousarray(keys).copy()
    kb = k.dtype.itemsize if k.ndim == 1 else k.shape[1]
    n = k.shape[0]
    v = None if vals is None else np.ascontiguousarray(vals).copy()
    vb = 0 if v is None else (v.dtype.itemsize if v.ndim == 1 else v.shape[1] * v.dtype.itemsize)
    if end_bit is None:
        end_bit = kb * 8
    lib().orc_sort_pairs_mt(_p(k), _p(v), n, kb, vb, begin_bit, end_bit, threads)
    return (k, v) if vals is not None else k


# ---------------------------------------------------------------- join
def find_bounds(left, right):
    left = np.ascontiguousarray(left)
    right = np.ascontiguousarray(right)
    kb = left.dtype.itemsize if left.ndim == 1 else left.shape[1]
    nl, nr = left.shape[0], right.shape[0]
    lb = np.zeros(nl, dtype=np.int32)
    cnt = np.zeros(nl, dtype=np.int32)
    tot = np.zeros(1, dtype=np.uint64)
    lib().orc_find_bounds(_p(lb), _p(cnt), _p(tot), _p(left), nl, _p(right), nr, kb)
    return lb, cnt, int(tot[0])


def join_expand(lb, scan, nout):
    li = np.zeros(nout, dtype=np.int32)
    ri = np.zeros(nout, dtype=np.int32)
    lib().orc_join_expand(_p(li), _p(ri), nout, _p(np.ascontiguousarray(lb, np.int32)),
                          _p(np.ascontiguousarray(scan, np.int32)), len(lb))
    return li, ri


def join_gather(obytes, li, ri, lkey, lval, lv_bits, rval, rv_bits):
    nout = len(li)
    out = np.zeros((nout, obytes), dtype=np.uint8)

    def wb(a):
        if a is None:
            return 0
        return a.dtype.itemsize if a.ndim == 1 else a.shape[1]
    lib().orc_join_gather(_p(out), obytes, nout, _p(np.ascontiguousarray(li, np.int32)),
                          _p(np.ascontiguousarray(ri, np.int32)), _p(lkey), wb(lkey),
                          _p(lval), wb(lval), lv_bits, _p(rval), wb(rval), rv_bits)
    return out


def join_tuples(left, lbits_val, right, rbits_val, obytes):
    left = np.ascontiguousarray(left, np.uint8)
    right = np.ascontiguousarray(right, np.uint8)
    total = lib().orc_join_tuples(None, obytes, 0, _p(left), left.shape[0], left.shape[1], lbits_val,
                                  _p(right), right.shape[0], right.shape[1], rbits_val)
    out = np.zeros((total, obytes), dtype=np.uint8)
    lib().orc_join_tuples(_p(out), obytes, total, _p(left), left.shape[0], left.shape[1], lbits_val,
                          _p(right), right.shape[0], right.shape[1], rbits_val)
    return out


# ---------------------------------------------------------------- reduce
def reduce_sum_i64(keys, vals):
    keys = np.ascontiguousarray(keys)
    kb = keys.dtype.itemsize if keys.ndim == 1 else keys.shape[1]
    n = keys.shape[0]
    ok = np.zeros_like(keys)
    ov = np.zeros(n, dtype=np.int64)
    g = lib().orc_reduce_sum_i64(_p(keys), n, kb, _p(np.ascontiguousarray(vals, np.int64)), _p(ok), _p(ov))
    return ok[:g], ov[:g]


def reduce_count(keys, vals=None):
    keys = np.ascontiguousarray(keys)
    kb = keys.dtype.itemsize if keys.ndim == 1 else keys.shape[1]
    n = keys.shape[0]
    ok = np.zeros_like(keys)
    oc = np.zeros(n, dtype=np.uint32)
    v = None if vals is None else np.ascontiguousarray(vals, np.uint32)
    g = lib().orc_reduce_count(_p(keys), n, kb, _p(v), _p(ok), _p(oc))
    return ok[:g], oc[:g]


# ---------------------------------------------------------------- double values
def reduce_f64_seq(keys, vals, op_min=False):
    """The reference's sequential fold per run of equal keys (keys None: one run)."""
    v = np.ascontiguousarray(vals, np.float64)
    n = v.shape[0]
    if keys is None:
        kb, k, ok = 0, None, None
    else:
        k = np.ascontiguousarray(keys)
        kb = k.dtype.itemsize * (1 if k.ndim == 1 else k.shape[1])
        ok = np.zeros_like(k)
    ov = np.zeros(n, np.float64)
    g = lib().orc_reduce_f64_seq(_p(k), n, kb, _p(v), _p(ok), _p(ov), int(op_min))
    return (ok[:g] if ok is not None else None), ov[:g]


def run_starts(keys, n):
    """Start index of every run of equal keys (rows of a 2-D byte array compare whole)."""
    if n == 0:
        return np.zeros(0, np.int64)
    if keys is None:
        return np.zeros(1, np.int64)
    k = np.ascontiguousarray(keys)
    diff = (k[1:] != k[:-1]) if k.ndim == 1 else np.any(k[1:] != k[:-1], axis=1)
    return np.concatenate([[0], np.nonzero(diff)[0] + 1]).astype(np.int64)


def exact_sum(x):
    """The sum of the doubles x computed exactly and rounded once to nearest-even, with
    IEEE addition's specials: NaN for a NaN or both infinities, else the infinity; an
    exact zero is -0 only if every term is -0; overflow gives the signed infinity."""
    import math
    from fractions import Fraction
    x = np.asarray(x, np.float64)
    if np.isnan(x).any() or (np.isposinf(x).any() and np.isneginf(x).any()):
        return math.nan
    if np.isposinf(x).any():
        return math.inf
    if np.isneginf(x).any():
        return -math.inf
    try:
        s = math.fsum(x.tolist())
    except OverflowError:
        f = sum((Fraction(float(v)) for v in x.tolist()), Fraction(0))
        try:
            return float(f)   # int / int division in Python rounds correctly
        except OverflowError:
            return math.inf if f > 0 else -math.inf
    if s == 0.0:
        return -0.0 if np.all(np.signbit(x)) and not np.any(x) else 0.0
    return s


def reduce_f64_exact(keys, vals):
    """Per run of equal keys: (first key, exact_sum of the run's values)."""
    v = np.ascontiguousarray(vals, np.float64)
    st = run_starts(keys, v.shape[0])
    ends = np.concatenate([st[1:], [v.shape[0]]]) if st.size else st
    sums = np.array([exact_sum(v[a:b]) for a, b in zip(st, ends)], np.float64)
    ok = None if keys is None else np.ascontiguousarray(keys)[st]
    return ok, sums


# ---------------------------------------------------------------- string keys
def str_pool(strings):
    """(pool, offs): the byte strings (no NUL inside) NUL-terminated back to back in one
    uint8 array, and their uint64 offsets -- a string column, offsets standing for the
    reference's pointers."""
    lens = np.fromiter((len(x) + 1 for x in strings), dtype=np.uint64, count=len(strings))
    offs = np.zeros(len(strings), dtype=np.uint64)
    if len(strings) > 1:
        np.cumsum(lens[:-1], out=offs[1:])
    pool = np.frombuffer(b"".join(x + b"\0" for x in strings) or b"\0", dtype=np.uint8).copy()
    return pool, offs


def str_sort(pool, offs, vals=None):
    """Stable sort of a string column (sort_string_key / sort_string_pair); returns the
    sorted offsets (and values)."""
    o = np.ascontiguousarray(offs, np.uint64).copy()
    v = None if vals is None else np.ascontiguousarray(vals).copy()
    vb = 0 if v is None else v.dtype.itemsize * (1 if v.ndim == 1 else v.shape[1])
    lib().orc_str_sort(_p(pool), _p(o), o.shape[0], _p(v), vb)
    return o if v is None else (o, v)


def str_find_bounds(pool, loffs, roffs):
    lo = np.ascontiguousarray(loffs, np.uint64)
    ro = np.ascontiguousarray(roffs, np.uint64)
    lb = np.zeros(lo.shape[0], np.int32)
    sc = np.zeros(lo.shape[0], np.int32)
    tot = np.zeros(1, np.uint64)
    lib().orc_str_find_bounds(_p(lb), _p(sc), _p(tot), _p(pool), _p(lo), lo.shape[0], _p(ro), ro.shape[0])
    return lb, sc, int(tot[0])


def str_count(pool, offs, vals):
    """count_string: (first offset of each run of equal strings, u32 sums)."""
    o = np.ascontiguousarray(offs, np.uint64)
    v = np.ascontiguousarray(vals, np.uint32)
    oo = np.zeros(o.shape[0], np.uint64)
    os_ = np.zeros(o.shape[0], np.uint32)
    g = lib().orc_str_count(_p(pool), _p(o), o.shape[0], _p(v), _p(oo), _p(os_))
    return oo[:g], os_[:g]


def str_codes(pool, offs):
    """(codes, distinct): the rank of each string among the column's distinct strings."""
    o = np.ascontiguousarray(offs, np.uint64)
    c = np.zeros(o.shape[0], np.uint32)
    d = lib().orc_str_codes(_p(pool), _p(o), o.shape[0], _p(c))
    return c, int(d)


# ---------------------------------------------------------------- set ops
def _setop(fn, a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    e = a.dtype.itemsize if a.ndim == 1 else a.shape[1]
    out = np.zeros((a.shape[0] + b.shape[0],) + a.shape[1:], dtype=a.dtype)
    k = fn(_p(out), _p(a), a.shape[0], _p(b), b.shape[0], e)
    return out[:k]


def set_union(a, b):
    return _setop(lib().orc_set_union, a, b)


def set_difference(a, b):
    return _setop(lib().orc_set_difference, a, b)


def set_intersection(a, b):
    return _setop(lib().orc_set_intersection, a, b)


def unique(a):
    a = np.ascontiguousarray(a).copy()
    e = a.dtype.itemsize if a.ndim == 1 else a.shape[1]
    k = lib().orc_unique(_p(a), a.shape[0], e)
    return a[:k]


# ---------------------------------------------------------------- select / arith / project
def make_cmps(cmps):
    """cmps: list of dicts {op, a:(kind, field|const), b:(kind, ...), type}."""
    arr = (Cmp * max(1, len(cmps)))()
    for i, c in enumerate(cmps):
        arr[i].op = c["op"]
        arr[i].value_type = c.get("type", I64)
        for side in ("a", "b"):
            kind, val = c[side]
            setattr(arr[i], side + "_kind", kind)
            if kind == OPND_VAR:
                setattr(arr[i], side + "_field", val)
            else:
                setattr(arr[i], side + "_const", val)
    return arr


def make_arith(nodes, root, dest_type, dest_bits):
    """nodes: list of tuples (kind, op, type, left, right, value)."""
    arr = (Node * len(nodes))()
    for i, (kind, op, typ, left, right, value) in enumerate(nodes):
        arr[i].kind, arr[i].op, arr[i].type = kind, op, typ
        arr[i].left, arr[i].right, arr[i].value = left, right, value
    a = Arith()
    a.nodes = arr
    a.nnodes = len(nodes)
    a.root = root
    a.dest_type = dest_type
    a.dest_bits = dest_bits
    a._keep = arr
    return a


def select(rows, widths, cmps):
    rows = np.ascontiguousarray(rows, np.uint8)
    t = Tuple.of(widths)
    arr = make_cmps(cmps)
    out = np.zeros_like(rows)
    k = lib().orc_select(_p(out), _p(rows), rows.shape[0], C.byref(t), arr, len(cmps))
    return out[:k]


def arith(rows, widths, arith_desc):
    rows = np.ascontiguousarray(rows, np.uint8)
    t = Tuple.of(widths)
    ow = container_bytes(sum(widths) + arith_desc.dest_bits)
    out = np.zeros((rows.shape[0], ow), dtype=np.uint8)
    rc = lib().orc_arith_rows(_p(out), _p(rows), rows.shape[0], C.byref(t), C.byref(arith_desc))
    if rc:
        raise ValueError("bad arith descriptor")
    return out


def project(rows, in_widths, out_widths, fmap):
    rows = np.ascontiguousarray(rows, np.uint8)
    it, ot = Tuple.of(in_widths), Tuple.of(out_widths)
    m = (C.c_uint32 * 16)(*(list(fmap) + [100] * (16 - len(fmap))))
    out = np.zeros((rows.shape[0], container_bytes(sum(out_widths))), dtype=np.uint8)
    lib().orc_project(_p(out), _p(rows), rows.shape[0], C.byref(it), C.byref(ot), m)
    return out


def filter_aggregate(rows, widths, cmps, ariths, group_fields, sum_fields, cap=4096, threads=None):
    rows = np.ascontiguousarray(rows, np.uint8)
    t = Tuple.of(widths)
    carr = make_cmps(cmps)
    aarr = (Arith * max(1, len(ariths)))(*ariths)
    g = (C.c_uint32 * 16)(*group_fields)
    s = (C.c_uint32 * 8)(*sum_fields)
    ok = np.zeros(cap, dtype=np.uint64)
    osum = np.zeros((cap, max(1, len(sum_fields))), dtype=np.int64)
    oc = np.zeros(cap, dtype=np.uint64)
    ng = lib().orc_filter_aggregate(_p(rows), rows.shape[0], C.byref(t), carr, len(cmps), aarr, len(ariths),
                                    g, len(group_fields), s, len(sum_fields), _p(ok), _p(osum), _p(oc), cap,
                                    threads or _threads())
    if ng < 0:
        raise ValueError("filter_aggregate failed: %d" % ng)
    return ok[:ng], osum[:ng, :len(sum_fields)], oc[:ng]


# ---------------------------------------------------------------- synthetic data
def uniform(n, seed, stream, lo, hi, threads=None):
    out = np.empty(n, dtype=np.uint64)
    lib().orc_gen_uniform_u64(_p(out), n, seed, stream, lo, hi, threads or _threads())
    return out


def zipf(n, seed, stream, domain, s=1.0, threads=None):
    cdf = np.empty(domain, dtype=np.float64)
    lib().orc_zipf_cdf(_p(cdf), domain, s)
    out = np.empty(n, dtype=np.uint64)
    lib().orc_gen_zipf_u64(_p(out), n, seed, stream, _p(cdf), domain, threads or _threads())
    return out
