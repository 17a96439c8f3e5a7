"""The reference's own redfox:: entry points (C++ linkage, the signatures of
redfox/ra/interface/*.h, string keys included) exported by the shim libraries over librfx.so: the exact
signatures are present, and on the GPU each computes what the oracle does."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from redfox_b200 import rfx as R

from helpers import to_np

PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "redfox_b200")
ULL = "unsigned long long"

EXPECTED = {
    "ra": ["redfox::find_bounds_%d(void*, void*, %s*, void*, %s, void*, %s)" % (w, ULL, ULL, ULL)
           for w in (8, 16, 32, 64, 128)]
    + ["redfox::join(int*, int*, %s, int*, int*, %s)" % (ULL, ULL)]
    + ["redfox::count_%d(void const*, void const*, void*, void*, %s*, %s*)" % (w, ULL, ULL)
       for w in (8, 16, 32, 128, 256)]
    + ["redfox::total_64_32(void const*, void const*, void*, void*, %s*, %s*)" % (ULL, ULL),
       "redfox::set_union(void*, %s*, void*, void*, void*, void*, unsigned int)" % ULL,
       "redfox::difference(void*, %s*, void*, void*, void*, void*, unsigned int)" % ULL,
       "redfox::unique(void*, %s*, %s)" % (ULL, ULL),
       "redfox::find_bounds_string(void*, void*, %s*, void*, %s, void*, %s)" % (ULL, ULL, ULL),
       "redfox::count_string(void const*, void const*, void*, void*, %s*, %s*)" % (ULL, ULL),
       "redfox::total_string_32(void const*, void const*, void*, void*, %s*, %s*)" % (ULL, ULL),
       "redfox::sort(void*, void*, %s)" % ULL,
       "redfox::sort_string(void*, void*)"]
    + ["redfox::total_%d_double(void const*, void const*, void*, void*, %s*, %s*)" % (w, ULL, ULL)
       for w in (8, 16, 32, 64, 128)]
    + ["redfox::total_string_double(void const*, void const*, void*, void*, %s*, %s*)" % (ULL, ULL),
       "redfox::min_32_double(void const*, void const*, void*, void*, %s*, %s*)" % (ULL, ULL),
       "redfox::total_double(void*, void const*, void const*)",
       "redfox::max_double(void*, void const*, void const*)",
       "redfox::count(void*, void const*, void const*)"],
    "b40c": ["redfox::sort_pair(void*, void*, %s, %s, %s)" % (ULL, ULL, ULL),
             "redfox::sort_key(void*, %s, %s)" % (ULL, ULL)],
    "mgpu": ["redfox::sort_pair(void*, void*, %s, %s, %s)" % (ULL, ULL, ULL),
             "redfox::sort_key(void*, %s, %s)" % (ULL, ULL),
             "redfox::sort_string_pair(void*, void*, %s, %s, %s)" % (ULL, ULL, ULL),
             "redfox::sort_string_key(void*, %s, %s)" % (ULL, ULL)],
}


def _symbols(lib):
    """demangled signature -> mangled name of the library's exported redfox:: functions."""
    path = os.path.join(PKG, "libredfox_%s.so" % lib)
    raw = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    mangled = [ln.split()[-1] for ln in raw.splitlines() if ln.split() and ln.split()[-1].startswith("_ZN6redfox")]
    dem = subprocess.run(["c++filt"], input="\n".join(mangled), capture_output=True, text=True, check=True).stdout
    return dict(zip(dem.splitlines(), mangled))


@pytest.mark.parametrize("lib", sorted(EXPECTED))
def test_shim_exports_reference_signatures(lib):
    syms = _symbols(lib)
    for sig in EXPECTED[lib]:
        assert sig in syms, (sig, sorted(syms))
    C.CDLL(os.path.join(PKG, "libredfox_%s.so" % lib))


def _fn(lib, sig, argtypes):
    handle = C.CDLL(os.path.join(PKG, "libredfox_%s.so" % lib))
    f = getattr(handle, _symbols(lib)[sig])
    f.restype = None
    f.argtypes = argtypes
    return f


def _dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


P, U = C.c_void_p, C.c_ulonglong


@pytest.mark.gpu
def test_shim_sorts(cuda):
    import torch
    n = 50000
    rng = np.random.default_rng(4)
    k = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    v = np.arange(n, dtype=np.uint64)
    dk, dv = _dev(k, cuda), _dev(v, cuda)
    torch.cuda.synchronize()
    _fn("b40c", EXPECTED["b40c"][0], [P, P, U, U, U])(dk.data_ptr(), dv.data_ptr(), n, 23, R.I64)
    ek, ev = O.sort_pairs(k, v, begin_bit=0, end_bit=23)
    assert np.array_equal(to_np(dk), ek) and np.array_equal(to_np(dv), ev)
    k64 = rng.integers(0, 2**63, n, dtype=np.uint64)
    dk = _dev(k64, cuda)
    torch.cuda.synchronize()
    _fn("mgpu", EXPECTED["mgpu"][1], [P, U, U])(dk.data_ptr(), n, R.I64)
    assert np.array_equal(to_np(dk), np.sort(k64))


@pytest.mark.gpu
def test_shim_join_count_and_sets(cuda):
    import torch
    rng = np.random.default_rng(5)
    left = np.sort(rng.integers(0, 3000, 5000)).astype(np.uint32)
    right = np.sort(rng.integers(0, 3000, 7000)).astype(np.uint32)
    dl, dr = _dev(left, cuda), _dev(right, cuda)
    lb = torch.empty(5000, dtype=torch.int32, device=cuda)
    lc = torch.empty(5000, dtype=torch.int32, device=cuda)
    rs = torch.zeros(1, dtype=torch.int64, device=cuda)
    torch.cuda.synchronize()
    _fn("ra", EXPECTED["ra"][2], [P, P, P, P, U, P, U])(lb.data_ptr(), lc.data_ptr(), rs.data_ptr(), dl.data_ptr(),
                                                         5000, dr.data_ptr(), 7000)
    elb, esc, etot = O.find_bounds(left, right)
    assert int(rs.item()) == etot and np.array_equal(to_np(lb), elb) and np.array_equal(to_np(lc), esc)
    li = torch.empty(etot, dtype=torch.int32, device=cuda)
    ri = torch.empty(etot, dtype=torch.int32, device=cuda)
    _fn("ra", EXPECTED["ra"][5], [P, P, U, P, P, U])(li.data_ptr(), ri.data_ptr(), etot, lb.data_ptr(),
                                                      lc.data_ptr(), 5000)
    eli, eri = O.join_expand(elb, esc, etot)
    assert np.array_equal(to_np(li), eli) and np.array_equal(to_np(ri), eri)
    # count_32: u32 keys, u32 values, device-resident byte sizes
    vals = rng.integers(0, 1000, 5000).astype(np.uint32)
    dvals = _dev(vals, cuda)
    ok = torch.empty(5000, dtype=torch.int32, device=cuda)
    ov = torch.empty(5000, dtype=torch.int32, device=cuda)
    ksz = torch.tensor([4 * 5000], dtype=torch.int64, device=cuda)
    vsz = torch.tensor([4 * 5000], dtype=torch.int64, device=cuda)
    torch.cuda.synchronize()
    _fn("ra", EXPECTED["ra"][8], [P, P, P, P, P, P])(dl.data_ptr(), dvals.data_ptr(), ok.data_ptr(), ov.data_ptr(),
                                                      ksz.data_ptr(), vsz.data_ptr())
    ek, ec = O.reduce_count(left, vals)
    g = int(ksz.item()) // 4
    assert g == len(ek) and int(vsz.item()) // 4 == g
    assert np.array_equal(to_np(ok)[:g].view(np.uint32), ek) and np.array_equal(to_np(ov)[:g].view(np.uint32), ec)
    # set_union / difference / unique on u32 (DataType I32)
    a = np.unique(rng.integers(0, 20000, 6000)).astype(np.uint32)
    b = np.unique(rng.integers(0, 20000, 4000)).astype(np.uint32)
    da, db = _dev(a, cuda), _dev(b, cuda)
    out = torch.zeros(len(a) + len(b), dtype=torch.int32, device=cuda)
    size = torch.zeros(1, dtype=torch.int64, device=cuda)
    torch.cuda.synchronize()
    args = [P, P, P, P, P, P, C.c_uint]
    _fn("ra", EXPECTED["ra"][12], args)(out.data_ptr(), size.data_ptr(), da.data_ptr(), da.data_ptr() + 4 * len(a),
                                         db.data_ptr(), db.data_ptr() + 4 * len(b), R.I32)
    k = int(size.item()) // 4
    assert np.array_equal(to_np(out)[:k].view(np.uint32), O.set_union(a, b))
    _fn("ra", EXPECTED["ra"][13], args)(out.data_ptr(), size.data_ptr(), da.data_ptr(), da.data_ptr() + 4 * len(a),
                                         db.data_ptr(), db.data_ptr() + 4 * len(b), R.I32)
    k = int(size.item()) // 4
    assert np.array_equal(to_np(out)[:k].view(np.uint32), O.set_difference(a, b))
    dup = np.sort(rng.integers(0, 500, 3000)).astype(np.uint32)
    du = _dev(dup, cuda)
    usz = torch.tensor([4 * len(dup)], dtype=torch.int64, device=cuda)
    torch.cuda.synchronize()
    _fn("ra", EXPECTED["ra"][14], [P, P, U])(du.data_ptr(), usz.data_ptr(), R.I32)
    k = int(usz.item()) // 4
    assert np.array_equal(to_np(du)[:k].view(np.uint32), O.unique(dup))
    assert R.device_status() == R.OK
