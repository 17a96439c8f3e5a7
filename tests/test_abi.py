"""The C ABI library: it loads, exports every symbol include/rfx/*.h declares, and
rejects bad descriptors on the host before touching a device.  CPU only."""
import ctypes as C

from redfox_b200 import rfx as R


def test_library_exports_every_declared_symbol():
    names = R.declared_symbols()
    assert len(names) >= 8
    missing = [n for n in names if not hasattr(R.LIB, n)]
    assert not missing, missing


def test_version_string():
    assert b"sm_100a" in R.LIB.rfx_version()


def test_bad_descriptors_rejected_on_host():
    t = R.Tuple.of([32, 32])
    cmps = R.make_cmps([(99, (R.OPND_VAR, 0), (R.OPND_CONST, 1), R.I32)])
    buf = C.c_void_p(16)  # never dereferenced: validation fails first
    st = R.LIB.rfx_select(buf, buf, buf, 10, C.byref(t), cmps, 1, buf, 1 << 20, None)
    assert st == R.ERR_UNSUPPORTED
    wide = R.Tuple.of([65])
    st = R.LIB.rfx_select(buf, buf, buf, 10, C.byref(wide), cmps, 0, buf, 1 << 20, None)
    assert st == R.ERR_UNSUPPORTED
    bad_field = R.make_cmps([(R.EQ, (R.OPND_VAR, 5), (R.OPND_CONST, 1), R.I32)])
    st = R.LIB.rfx_select(buf, buf, buf, 10, C.byref(t), bad_field, 1, buf, 1 << 20, None)
    assert st == R.ERR_INVALID
    st = R.LIB.rfx_select(None, buf, buf, 10, C.byref(t), cmps, 0, buf, 1 << 20, None)
    assert st == R.ERR_INVALID


def test_aggregate_domain_limits_on_host():
    t = R.Tuple.of([16, 16])
    gf = (C.c_uint32 * 4)(0, 1)
    gd = (C.c_uint32 * 4)(1000, 1000)   # 10^6 groups > 4096
    sf = (C.c_uint32 * 4)(0)
    buf = C.c_void_p(16)
    st = R.LIB.rfx_filter_aggregate(buf, 10, C.byref(t), None, 0, None, 0, gf, gd, 2, sf, 1, buf, buf, buf, buf,
                                    buf, 1 << 20, None)
    assert st == R.ERR_UNSUPPORTED


def test_workspace_sizes_grow_with_input():
    t = R.Tuple.of([32, 64])
    assert R.LIB.rfx_select_workspace(10**8, C.byref(t)) > R.LIB.rfx_select_workspace(10**4, C.byref(t))
