"""Radix sort against the oracle's stable LSD sort (bit-exact, stability included)."""
import numpy as np
import pytest

import oracle as O
from redfox_b200 import rfx as R

from helpers import to_np

pytestmark = pytest.mark.gpu


def _keys(n, kb, seed, hi_bits=None):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 256, (n, kb), dtype=np.uint8)
    if hi_bits is not None:  # keep only the low `hi_bits` bits
        bits = np.unpackbits(a, axis=1, bitorder="little")
        bits[:, hi_bits:] = 0
        a = np.packbits(bits, axis=1, bitorder="little")
    return a


def _dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


SIZES = [0, 1, 2, 31, 33, 1000, 4095, 4096, 4097, 100003]


@pytest.mark.parametrize("kb", [1, 2, 4, 8, 16, 32, 64])
@pytest.mark.parametrize("n", SIZES)
def test_sort_keys_full_width(cuda, kb, n):
    keys = _keys(n, kb, seed=kb * 31 + n)
    end = min(kb * 8, 128)
    d = _dev(keys, cuda)
    R.sort_pairs(d, begin_bit=0, end_bit=end)
    exp = O.sort_pairs(keys, begin_bit=0, end_bit=end)
    assert np.array_equal(to_np(d), exp)
    assert R.device_status() == R.OK


@pytest.mark.parametrize("kb,vb", [(4, 4), (4, 8), (8, 8), (8, 16), (16, 16), (16, 4), (1, 2), (2, 1), (64, 16), (32, 8)])
@pytest.mark.parametrize("n", [5, 4097, 200001])
def test_sort_pairs_stable(cuda, kb, vb, n):
    keys = _keys(n, kb, seed=n + kb * 7 + vb, hi_bits=min(kb * 8, 12))  # many duplicates
    vals = np.random.default_rng(n).integers(0, 256, (n, vb), dtype=np.uint8)
    dk, dv = _dev(keys, cuda), _dev(vals, cuda)
    end = min(kb * 8, 40)
    R.sort_pairs(dk, dv, begin_bit=0, end_bit=end)
    ek, ev = O.sort_pairs(keys, vals, begin_bit=0, end_bit=end)
    assert np.array_equal(to_np(dk), ek) and np.array_equal(to_np(dv), ev)


@pytest.mark.parametrize("begin,end", [(3, 17), (64, 96), (100, 128), (8, 9)])
def test_sort_bit_range_of_packed_tuples(cuda, begin, end):
    n = 50000
    keys = _keys(n, 16, seed=begin * 1000 + end)
    d = _dev(keys, cuda)
    R.sort_pairs(d, begin_bit=begin, end_bit=end)
    assert np.array_equal(to_np(d), O.sort_pairs(keys, begin_bit=begin, end_bit=end))


def test_sort_wide_range_over_128_bits(cuda):
    n = 20000
    keys = _keys(n, 32, seed=3, hi_bits=200)
    d = _dev(keys, cuda)
    R.sort_pairs(d, begin_bit=0, end_bit=256)
    assert np.array_equal(to_np(d), O.sort_pairs(keys, begin_bit=0, end_bit=256))


def test_all_equal_keys_keep_input_order(cuda):
    import torch
    n = 300000
    keys = torch.full((n,), 7, dtype=torch.int32, device=cuda)
    vals = torch.arange(n, dtype=torch.int32, device=cuda)
    R.sort_pairs(keys, vals)
    assert torch.equal(vals, torch.arange(n, dtype=torch.int32, device=cuda))


def test_skip_trivial_passes_same_result(cuda):
    n = 1_000_003
    keys = _keys(n, 4, seed=11, hi_bits=18)
    vals = np.arange(n, dtype=np.uint32)
    a, av = _dev(keys, cuda), _dev(vals, cuda)
    b, bv = _dev(keys, cuda), _dev(vals, cuda)
    R.sort_pairs(a, av)
    R.sort_pairs(b, bv, flags=R.SORT_SKIP_TRIVIAL)
    ek, ev = O.sort_pairs(keys, vals)
    for k, v in ((a, av), (b, bv)):
        assert np.array_equal(to_np(k), ek) and np.array_equal(to_np(v), ev)


def test_large_sort_properties(cuda):
    """Full-size property check: sorted, and a permutation (value checksum) at 8M pairs."""
    import torch
    n = 8_000_000
    g = torch.Generator(device=cuda).manual_seed(5)
    keys = torch.randint(0, 2**31 - 1, (n,), dtype=torch.int64, device=cuda, generator=g)
    vals = torch.arange(n, dtype=torch.int64, device=cuda)
    k0 = keys.clone()
    R.sort_pairs(keys, vals)
    assert bool((keys[1:] >= keys[:-1]).all())
    assert int(vals.sum()) == n * (n - 1) // 2
    assert torch.equal(k0[vals], keys)


def test_reference_compatible_entries(cuda):
    import ctypes as C
    import torch
    n = 70000
    rng = np.random.default_rng(1)
    # b40c sort_pair: 18-bit keys in u32 containers, I64 values (value_type code 4)
    k = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    v = np.arange(n, dtype=np.uint64)
    dk, dv = _dev(k, cuda), _dev(v, cuda)
    torch.cuda.synchronize()
    assert R.LIB.rfx_b40c_sort_pair(C.c_void_p(dk.data_ptr()), C.c_void_p(dv.data_ptr()), n, 18, R.I64) == R.OK
    ek, ev = O.sort_pairs(k, v, begin_bit=0, end_bit=18)
    assert np.array_equal(to_np(dk), ek) and np.array_equal(to_np(dv), ev)
    # mgpu sort_key on 128-bit keys (I128): whole-key order, high limb first
    k128 = rng.integers(0, 256, (n, 16), dtype=np.uint8)
    dk = _dev(k128, cuda)
    torch.cuda.synchronize()
    assert R.LIB.rfx_mgpu_sort_key(C.c_void_p(dk.data_ptr()), n, R.I128) == R.OK
    assert np.array_equal(to_np(dk), O.sort_pairs(k128))
    # b40c sort_key with 37 bits in u64 containers
    k64 = rng.integers(0, 2**63, n, dtype=np.uint64)
    dk = _dev(k64, cuda)
    torch.cuda.synchronize()
    assert R.LIB.rfx_b40c_sort_key(C.c_void_p(dk.data_ptr()), n, 37) == R.OK
    assert np.array_equal(to_np(dk), O.sort_pairs(k64, begin_bit=0, end_bit=37))


# Tile sizes of the two pass kernels: the per-tile pass (3072 / 5120 / 6144 keys of 16 / 8
# / 4 bytes) and the pipelined onesweep pass (3072 / 6144 / 8192 by default); sizes around
# both, and sizes with many tiles per block (persistent grids).
ONESWEEP_SIZES = {16: [3071, 3072, 3073, 9217, 2_000_003], 8: [5119, 5120, 5121, 6145, 18_433, 3_000_001],
                  4: [6143, 6144, 6145, 8193, 24_577, 4_000_037]}


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("kb", [4, 8, 16])
def test_sort_pass_variants_match_oracle(cuda, kb, variant):
    """Every pass kernel variant (pinned through the tuner) gives the oracle's stable
    order, on whole keys and on bit ranges that leave payload bits outside the key."""
    try:
        R.tune_force(R.TUNE_SORT_PASS, variant)
        for n in ONESWEEP_SIZES[kb]:
            keys = _keys(n, kb, seed=n * 3 + kb)
            # whole keys; a range leaving payload bits; odd pass counts (3 and 5 digits),
            # which end in the caller's buffer through the second alternate buffer
            for begin, end in ((0, kb * 8), (kb * 4, kb * 8 - 3), (kb * 8 - 24, kb * 8), (kb * 8 - 40, kb * 8 - 1)):
                if begin < 0:
                    continue
                d = _dev(keys, cuda)
                R.sort_pairs(d, begin_bit=begin, end_bit=end)
                assert np.array_equal(to_np(d), O.sort_pairs(keys, begin_bit=begin, end_bit=end, threads=8)), (n, begin)
        assert R.device_status() == R.OK
    finally:
        R.tune_force(R.TUNE_SORT_PASS, -1)


def test_sort_unaligned_slice_uses_per_tile_pass(cuda):
    """A key array that starts 8 bytes into an allocation (not 16-byte aligned) is sorted by
    the per-tile pass with the same result."""
    import torch
    n = 100_001
    keys = _keys(n + 1, 8, seed=77)
    d = _dev(keys, cuda)
    sub = d[1:]
    assert sub.data_ptr() % 16 == 8
    R.sort_pairs(sub, begin_bit=0, end_bit=64)
    assert np.array_equal(to_np(sub), O.sort_pairs(keys[1:], begin_bit=0, end_bit=64))
    assert torch.equal(d[0], _dev(keys[0], cuda))


@pytest.mark.parametrize("kb,vb,begin,end", [(4, 0, 0, 8), (4, 0, 0, 16), (8, 8, 8, 32), (16, 0, 64, 96),
                                             (8, 4, 0, 64), (16, 16, 0, 128), (64, 0, 0, 200)])
@pytest.mark.parametrize("n", [1, 33, 100003])
def test_sort_from_leaves_input_and_matches_in_place(cuda, kb, vb, begin, end, n):
    """rfx_sort_pairs_from sorts the input into other buffers (one to four passes, values,
    keys over 128 bits) with the in-place sort's result and leaves the input as it was."""
    import torch
    keys = _keys(n, kb, seed=kb + vb + n + end)
    vals = _keys(n, vb, seed=7 + n) if vb else None
    dk = _dev(keys, cuda)
    dv = _dev(vals, cuda) if vb else None
    ok, ov = R.sorted_copy(dk, dv, begin_bit=begin, end_bit=end)
    assert np.array_equal(to_np(dk), keys)
    if vb:
        assert np.array_equal(to_np(dv), vals)
    ek = _dev(keys, cuda)
    ev = _dev(vals, cuda) if vb else None
    R.sort_pairs(ek, ev, begin_bit=begin, end_bit=end)
    assert torch.equal(ok, ek)
    if vb:
        assert torch.equal(ov, ev)
    assert R.device_status() == R.OK


def test_sort_from_all_trivial_and_overlap(cuda):
    """Every digit constant with the skip flag: the output is a copy of the input.  Input
    and output overlapping: rejected."""
    import torch
    keys = np.zeros((5000, 4), np.uint8)
    keys[:, 0] = np.arange(5000) % 256
    dk = _dev(keys, cuda)
    out = torch.empty_like(dk)
    s = R.Sorter(5000, 4, 0, 8, 32, device=cuda)
    s(out, None, 1, None, src_keys=dk)
    assert np.array_equal(to_np(out), keys)
    st = R.LIB.rfx_sort_pairs_from(R._ptr(dk), None, R._ptr(dk[100:]), None, 4000, 4, 0, 0, 32, 0, R._ptr(s.ws), s.wsb,
                                   R._stream())
    assert st == R.ERR_INVALID
