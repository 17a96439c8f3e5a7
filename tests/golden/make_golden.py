"""Regenerates the golden fixtures in this directory from the reference's own code.

Run in a container that has the reference tree (default /root/reference):

    make -C oracle ref           # builds oracle/_ref/libredfox_ref.so from the reference
    python tests/golden/make_golden.py

Sources of truth:
  * tpch_A.bin       -- the reference's packed fixture TPC-H/data/A (5 x Tuple<32,32>),
                        made by TPC-H/data/TC_data_process.cu from TC.tbl; copied verbatim.
  * tuple_pack.npz   -- field columns and the bytes the reference's Tuple.h insert<>
                        produces for them (ref_pack_* in oracle/ref/ref_driver.cpp).
  * setops.npz       -- redfox::set_union / redfox::difference / redfox::unique
                        (Union.cu, Difference.cu, Unique.cu) and thrust set_intersection
                        on seeded sorted multisets of 1..16-byte elements.
  * reduce.npz       -- redfox::count_8/16/32/128 and total_64_32 (Reduce.cu) and
                        thrust::reduce_by_key with int64 sums.
  * sort.npz         -- redfox::sort (Sort.cu) per element type.
  * fact_plan.npz    -- the filter-project-aggregate plan written with the reference's
                        Tuple.h / Comparisons.h / Project.h and thrust (ref_fact_plan).
  * f64.npz          -- redfox::total_{8,16,32,64,128}_double, min_32_double, total_double,
                        max_double and count (Reduce.cu) on seeded double columns.
  * strings.npz      -- a seeded string column (pool + offsets) through redfox::sort_string
                        (Sort.cu) and redfox::count_string (Reduce.cu), sorted and unsorted.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REFROOT = os.environ.get("RFX_REFERENCE_ROOT",
                         os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))),
                                      "reference"))
sys.path.insert(0, REPO)

import oracle as O  # noqa: E402

P = C.c_void_p


def ptr(a):
    return a.ctypes.data_as(P)


def main():
    ref = O.ref_lib()
    if ref is None:
        sys.exit("oracle/_ref/libredfox_ref.so missing: run `make -C oracle ref` first")
    for fn in ("ref_set_union", "ref_difference", "ref_unique", "ref_intersection_u32",
               "ref_count_8", "ref_count_16", "ref_count_32", "ref_count_128", "ref_total_64_32",
               "ref_reduce_sum_i64_u32", "ref_reduce_sum_i64_u64", "ref_fact_plan", "ref_count_string",
               "ref_total_string_32"):
        getattr(ref, fn).restype = C.c_uint64 if fn != "ref_fact_plan" else C.c_int64
    rng = np.random.default_rng(20101130)

    # ---- packed fixture A
    with open(os.path.join(REFROOT, "TPC-H", "data", "A"), "rb") as f:
        data = f.read()
    with open(os.path.join(HERE, "tpch_A.bin"), "wb") as f:
        f.write(data)

    # ---- tuple packing through the reference's insert<>
    shapes = {"32_32": [32, 32], "16_16": [16, 16], "32_64": [32, 64], "32_8": [32, 8],
              "32_32_32": [32, 32, 32], "fact": [32, 64, 64, 64, 64, 8, 8],
              "fact_a2": [32, 64, 64, 64, 64, 8, 8, 64, 64], "proj": [8, 8, 64, 64],
              "odd": [3, 14, 23, 5, 19], "wide": [7, 33, 64, 40, 21]}
    pack = {}
    for name, widths in shapes.items():
        n = 64
        cols = [rng.integers(0, 2**63, n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, n, dtype=np.uint64)
                for _ in widths]
        cols = [c & np.uint64((1 << w) - 1 if w < 64 else 2**64 - 1) for c, w in zip(cols, widths)]
        getattr(ref, "ref_bytes_" + name).restype = C.c_uint
        W = getattr(ref, "ref_bytes_" + name)()
        out = np.zeros((n, W), dtype=np.uint8)
        arr = (P * len(cols))(*[c.ctypes.data for c in cols])
        getattr(ref, "ref_pack_" + name)(ptr(out), C.c_size_t(n), arr)
        pack[name + "_widths"] = np.array(widths, dtype=np.uint32)
        pack[name + "_cols"] = np.stack(cols)
        pack[name + "_bytes"] = out
    np.savez_compressed(os.path.join(HERE, "tuple_pack.npz"), **pack)

    # ---- set operations: DataType I8..I64 and I128 (two limbs)
    sets = {}
    for esize, dtype, code in ((1, np.uint8, 1), (2, np.uint16, 2), (4, np.uint32, 3), (8, np.uint64, 4), (16, None, 5)):
        for case in range(3):
            na, nb = [(0, 7), (300, 200), (1000, 1500)][case]
            hi = [50, 300, 2**31][case]
            if esize == 16:
                a = np.zeros((na, 16), np.uint8)
                b = np.zeros((nb, 16), np.uint8)
                ka = np.sort(rng.integers(0, hi, na)).astype(np.uint64)
                kb = np.sort(rng.integers(0, hi, nb)).astype(np.uint64)
                # high limb carries the key, low limb a small tag so both limbs matter
                a.view(np.uint64)[:, 1] = ka // 4
                a.view(np.uint64)[:, 0] = ka % 4
                b.view(np.uint64)[:, 1] = kb // 4
                b.view(np.uint64)[:, 0] = kb % 4
            else:
                a = np.sort(rng.integers(0, min(hi, np.iinfo(dtype).max), na).astype(dtype))
                b = np.sort(rng.integers(0, min(hi, np.iinfo(dtype).max), nb).astype(dtype))
            key = "e%d_c%d" % (esize, case)
            sets[key + "_a"], sets[key + "_b"] = a, b
            cap = na + nb + 1
            out = np.zeros((cap,) + a.shape[1:], dtype=a.dtype)
            k = ref.ref_set_union(ptr(out), ptr(a), C.c_size_t(na), ptr(b), C.c_size_t(nb), esize, code)
            sets[key + "_union"] = out[:k].copy()
            k = ref.ref_difference(ptr(out), ptr(a), C.c_size_t(na), ptr(b), C.c_size_t(nb), esize, code)
            sets[key + "_difference"] = out[:k].copy()
            if esize == 4:
                k = ref.ref_intersection_u32(ptr(out), ptr(a), C.c_size_t(na), ptr(b), C.c_size_t(nb))
                sets[key + "_intersection"] = out[:k].copy()
            if esize <= 8 and na > 1:
                u = a.copy()
                k = ref.ref_unique(ptr(u), C.c_size_t(na), esize, code)
                sets[key + "_unique"] = u[:k].copy()
    np.savez_compressed(os.path.join(HERE, "setops.npz"), **sets)

    # ---- reduce / count
    red = {}
    for esize, dtype, fn in ((1, np.uint8, "ref_count_8"), (2, np.uint16, "ref_count_16"), (4, np.uint32, "ref_count_32")):
        n = 2000
        k = np.sort(rng.integers(0, 40, n).astype(dtype))
        v = rng.integers(1, 5, n).astype(np.uint32)
        ok = np.zeros(n, dtype)
        ov = np.zeros(n, np.uint32)
        g = getattr(ref, fn)(ptr(k), ptr(v), ptr(ok), ptr(ov), C.c_size_t(n))
        red["count%d_keys" % esize], red["count%d_vals" % esize] = k, v
        red["count%d_okeys" % esize], red["count%d_ocounts" % esize] = ok[:g].copy(), ov[:g].copy()
    n = 2000
    k128 = np.zeros((n, 16), np.uint8)
    kk = np.sort(rng.integers(0, 60, n)).astype(np.uint64)
    k128.view(np.uint64)[:, 1] = kk // 3
    k128.view(np.uint64)[:, 0] = kk % 3
    v = rng.integers(1, 5, n).astype(np.uint32)
    ok = np.zeros_like(k128)
    ov = np.zeros(n, np.uint32)
    g = ref.ref_count_128(ptr(k128), ptr(v), ptr(ok), ptr(ov), C.c_size_t(n))
    red["count16_keys"], red["count16_vals"], red["count16_okeys"], red["count16_ocounts"] = k128, v, ok[:g].copy(), ov[:g].copy()
    k64 = np.sort(rng.integers(0, 2**40, 300)).astype(np.uint64).repeat(rng.integers(1, 9, 300))
    n = len(k64)
    v = rng.integers(0, 2**31, n).astype(np.uint32)
    ok = np.zeros(n, np.uint64)
    ov = np.zeros(n, np.uint32)
    g = ref.ref_total_64_32(ptr(k64), ptr(v), ptr(ok), ptr(ov), C.c_size_t(n))
    red["total64_32_keys"], red["total64_32_vals"], red["total64_32_okeys"], red["total64_32_osums"] = k64, v, ok[:g].copy(), ov[:g].copy()
    k32 = np.sort(rng.integers(0, 500, 5000)).astype(np.uint32)
    v = rng.integers(-2**62, 2**62, 5000).astype(np.int64)
    ok = np.zeros(5000, np.uint32)
    ov = np.zeros(5000, np.int64)
    g = ref.ref_reduce_sum_i64_u32(ptr(k32), ptr(v), ptr(ok), ptr(ov), C.c_size_t(5000))
    red["sum_i64_keys"], red["sum_i64_vals"], red["sum_i64_okeys"], red["sum_i64_osums"] = k32, v, ok[:g].copy(), ov[:g].copy()
    np.savez_compressed(os.path.join(HERE, "reduce.npz"), **red)

    # ---- sort (thrust::sort on full elements)
    srt = {}
    for esize, dtype, code in ((1, np.uint8, 1), (2, np.uint16, 2), (4, np.uint32, 3), (8, np.uint64, 4)):
        a = rng.integers(0, np.iinfo(dtype).max, 3000, dtype=np.uint64).astype(dtype)
        b = a.copy()
        ref.ref_sort(ptr(b), C.c_size_t(len(b)), esize, code)
        srt["e%d_in" % esize], srt["e%d_out" % esize] = a, b
    np.savez_compressed(os.path.join(HERE, "sort.npz"), **srt)

    # ---- the fact plan on a seeded sample (same generator as the workloads)
    n = 20000
    widths = [32, 64, 64, 64, 64, 8, 8]
    lo = [0, 1, 90000, 0, 0, 0, 0]
    hi = [2526, 51, 10500001, 11, 9, 3, 2]
    cols = [O.uniform(n, 0x5EED0001, f, lo[f], hi[f]) for f in range(7)]
    rows = O.pack(widths, cols)
    ok = np.zeros(16, np.uint64)
    s1 = np.zeros(16, np.int64)
    s2 = np.zeros(16, np.int64)
    cnt = np.zeros(16, np.uint64)
    g = ref.ref_fact_plan(ptr(rows), C.c_size_t(n), 2475, ptr(ok), ptr(s1), ptr(s2), ptr(cnt))
    np.savez_compressed(os.path.join(HERE, "fact_plan.npz"), n=np.array([n]), cutoff=np.array([2475]),
                        keys=ok[:g], s1=s1[:g], s2=s2[:g], counts=cnt[:g])
    # ---- string keys: columns of pointers into one pool (host pointers here)
    from redfox_b200 import workloads as WL
    pool, offs = WL.gen_strings(4000, seed=20101130, distinct=900)
    base = np.uint64(pool.ctypes.data)
    keys = offs + base
    ref.ref_sort_string(ptr(keys), C.c_size_t(len(keys)))
    sorted_offs = keys - base
    vals = rng.integers(0, 2**32, len(offs), dtype=np.uint64).astype(np.uint32)
    strs = {"pool": pool, "offs": offs, "sorted": sorted_offs, "vals": vals}
    for name, col in (("count_sorted", sorted_offs), ("count_unsorted", offs)):
        k = col + base
        ok = np.zeros(len(col), np.uint64)
        ov = np.zeros(len(col), np.uint32)
        g = ref.ref_count_string(ptr(k), ptr(vals), ptr(ok), ptr(ov), C.c_size_t(len(col)))
        strs[name + "_offs"], strs[name + "_sums"] = ok[:g] - base, ov[:g]
    np.savez_compressed(os.path.join(HERE, "strings.npz"), **strs)
    # ---- double values
    for fn in ("ref_total_8_double", "ref_total_16_double", "ref_total_32_double", "ref_total_64_double",
               "ref_total_128_double", "ref_min_32_double", "ref_max_double"):
        getattr(ref, fn).restype = C.c_uint64
    ref.ref_total_double.restype = C.c_double
    ref.ref_count.restype = C.c_uint32
    f64 = {}
    n = 5000
    vals = rng.uniform(1.0, 2.0, n) * np.exp2(rng.integers(-30, 31, n)) * rng.choice([1.0, -1.0], n)
    vals[rng.integers(0, n, 40)] = rng.choice([0.0, -0.0, np.nan, np.inf], 40)
    f64["vals"] = vals
    groups = np.sort(rng.integers(0, 300, n))
    for kb, dt in ((1, np.uint8), (2, np.uint16), (4, np.uint32), (8, np.uint64)):
        k = (groups.astype(np.uint64) * np.uint64(2654435761)).astype(dt)
        ok = np.zeros_like(k)
        ov = np.zeros(n, np.float64)
        g = getattr(ref, "ref_total_%d_double" % (kb * 8))(ptr(k), ptr(vals), ptr(ok), ptr(ov), C.c_size_t(n))
        f64["k%d" % kb], f64["k%d_okeys" % kb], f64["k%d_sums" % kb] = k, ok[:g].copy(), ov[:g].copy()
        if kb == 4:
            g = ref.ref_min_32_double(ptr(k), ptr(vals), ptr(ok), ptr(ov), C.c_size_t(n))
            f64["k4_min_okeys"], f64["k4_mins"] = ok[:g], ov[:g]
    k16 = np.zeros((n, 2), np.uint64)
    k16[:, 0] = groups.astype(np.uint64) * np.uint64(0x9E3779B97F4A7C15)
    k16[:, 1] = groups.astype(np.uint64)
    ok = np.zeros_like(k16)
    ov = np.zeros(n, np.float64)
    g = ref.ref_total_128_double(ptr(k16), ptr(vals), ptr(ok), ptr(ov), C.c_size_t(n))
    f64["k16"], f64["k16_okeys"], f64["k16_sums"] = k16, ok[:g], ov[:g]
    fin = np.ascontiguousarray(vals[np.isfinite(vals)])
    f64["total"] = np.array([ref.ref_total_double(ptr(fin), C.c_size_t(len(fin)))])
    f64["max_bits"] = np.array([ref.ref_max_double(ptr(vals), C.c_size_t(n))], np.uint64)
    u = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    f64["u32"], f64["count"] = u, np.array([ref.ref_count(ptr(u), C.c_size_t(n))], np.uint32)
    np.savez_compressed(os.path.join(HERE, "f64.npz"), **f64)

    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
