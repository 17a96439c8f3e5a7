"""rfx_reduce_tuples (runs of equal high fields of packed rows -> key, SUM, COUNT)
against the oracle's reduce-by-key on the same keys and values, over row widths, tile
boundaries, tails that the tensor map does not cover, long runs that span many tiles,
a device-resident count and unaligned row pointers."""
import numpy as np
import pytest

import oracle as O
from redfox_b200 import rfx as R

from helpers import to_np

pytestmark = pytest.mark.gpu


def _rows(n, rb, ks, distinct, seed):
    """Random rows whose bytes from ks/8 up hold a sorted key id."""
    rng = np.random.default_rng(seed)
    rows = rng.integers(0, 256, (n, rb), dtype=np.uint8)
    kbytes = rb - ks // 8
    ids = np.sort(rng.integers(0, max(1, distinct), n)).astype(np.uint64)
    for b in range(kbytes):
        rows[:, ks // 8 + b] = ((ids >> np.uint64(8 * (b % 8))) & np.uint64(0xff)).astype(np.uint8) if b < 8 else 0
    return rows


def _expect(rows, ks, vs, vbits, okb):
    keys = np.ascontiguousarray(rows[:, ks // 8:])
    vals = np.zeros(rows.shape[0], np.uint64)
    for b in range(vbits // 8):
        vals |= rows[:, vs // 8 + b].astype(np.uint64) << np.uint64(8 * b)
    ek, es = O.reduce_sum_i64(keys, vals.view(np.int64))
    _, ec = O.reduce_count(keys)
    out = np.zeros((ek.shape[0], okb), np.uint8)
    w = min(okb, ek.shape[1])
    out[:, :w] = ek[:, :w]
    return out, es, ec


def _run(cuda, rows_np, ks, vs, vbits, okb, offset=0, d_n=None):
    import torch
    n, rb = rows_np.shape
    buf = torch.zeros((n + offset, rb), dtype=torch.uint8, device=cuda)
    buf[offset:] = torch.from_numpy(rows_np).to(cuda)
    rows = buf[offset:]
    dn = None
    if d_n is not None:
        dn = torch.tensor([d_n], dtype=torch.int64, device=cuda)
    keys, sums, counts, g = R.reduce_tuples(rows, ks, vs, vbits, okb, d_n=dn)
    k = to_np(keys).view(np.uint8).reshape(g, okb) if g else np.zeros((0, okb), np.uint8)
    assert R.device_status() == R.OK
    return k, to_np(sums), to_np(counts).view(np.uint32)


SHAPES = [(16, 96, 0, 64, 4), (16, 64, 0, 32, 8), (16, 32, 0, 32, 16), (8, 32, 0, 32, 4), (4, 16, 0, 16, 4)]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "rb%d_ks%d" % (s[0], s[1]))
@pytest.mark.parametrize("n,distinct", [(0, 1), (1, 1), (7, 3), (8, 8), (2047, 100), (2048, 2048), (2049, 1),
                                        (8193, 9000), (100003, 5000), (300001, 1), (1 << 20, 1 << 18)])
def test_reduce_tuples_matches_oracle(cuda, shape, n, distinct):
    rb, ks, vs, vbits, okb = shape
    rows = _rows(n, rb, ks, distinct, seed=n * 31 + rb)
    k, s, c = _run(cuda, rows, ks, vs, vbits, okb)
    ek, es, ec = _expect(rows, ks, vs, vbits, okb)
    assert np.array_equal(k, ek)
    assert np.array_equal(s, es)
    assert np.array_equal(c, ec)


@pytest.mark.parametrize("shape", [(16, 96, 0, 64, 4), (8, 32, 0, 32, 4), (4, 16, 0, 16, 4)],
                         ids=lambda s: "rb%d" % s[0])
def test_reduce_tuples_unaligned_rows(cuda, shape):
    """Rows that start off a 16-byte boundary take the register-tiled kernel."""
    rb, ks, vs, vbits, okb = shape
    rows = _rows(50001, rb, ks, 700, seed=5)
    k, s, c = _run(cuda, rows, ks, vs, vbits, okb, offset=1)
    ek, es, ec = _expect(rows, ks, vs, vbits, okb)
    assert np.array_equal(k, ek) and np.array_equal(s, es) and np.array_equal(c, ec)


@pytest.mark.parametrize("valid", [0, 1, 5000, 70000])
def test_reduce_tuples_device_count(cuda, valid):
    rows = _rows(70000, 16, 96, 900, seed=9)
    k, s, c = _run(cuda, rows, 96, 0, 64, 4, d_n=valid)
    ek, es, ec = _expect(rows[:valid], 96, 0, 64, 4)
    assert np.array_equal(k, ek) and np.array_equal(s, es) and np.array_equal(c, ec)


def test_reduce_tuples_repeat_is_stable(cuda):
    """Two calls in a row (workspace reuse) give identical results."""
    rows = _rows(123457, 16, 96, 4000, seed=3)
    a = _run(cuda, rows, 96, 0, 64, 4)
    b = _run(cuda, rows, 96, 0, 64, 4)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("variant", [0, 1, 2, 3], ids=["warps", "chunked", "lookback256", "lookback128"])
@pytest.mark.parametrize("n,distinct", [(5000, 3), (300001, 1), (1 << 20, 1 << 18), (3_000_000, 2_999_000),
                                        (2_000_003, 40000)])
def test_reduce_tuples_variants(cuda, variant, n, distinct):
    """Every staged variant: long runs across chunks, groups over the chunked form's
    scratch share (its second pass), and the join-output shape."""
    rows = _rows(n, 16, 96, distinct, seed=n + 7)
    R.tune_force(1, variant)
    try:
        k, s, c = _run(cuda, rows, 96, 0, 64, 4)
    finally:
        R.tune_force(1, -1)
    ek, es, ec = _expect(rows, 96, 0, 64, 4)
    assert np.array_equal(k, ek) and np.array_equal(s, es) and np.array_equal(c, ec)
