// search.cuh -- sorted-search primitives over packed keys.
//
// A key view reads element i of a sorted array of E-byte containers (E <= 16) as an
// unsigned 128-bit integer and shifts it right by `shift` bits: shift = 0 compares whole
// keys (the find_bounds_{8..128} entries compare the whole container, limb a[1] before
// a[0], ModernGPUJoin.cu:27-39), shift = value bits compares packed tuples on their key
// fields, which Tuple.h places in the high bits.
#pragma once

#include "rfx_device.cuh"

namespace rfx {

typedef unsigned __int128 u128;

template <int E>
__device__ __forceinline__ u128 load_u128(const uint8_t* base, uint64_t i) {
  if constexpr (E == 1) {
    return (u128)__ldg(base + i);
  } else if constexpr (E == 2) {
    return (u128)__ldg(reinterpret_cast<const uint16_t*>(base) + i);
  } else if constexpr (E == 4) {
    return (u128)__ldg(reinterpret_cast<const uint32_t*>(base) + i);
  } else if constexpr (E == 8) {
    return (u128)__ldg(reinterpret_cast<const unsigned long long*>(base) + i);
  } else {
    const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(base) + i);
    return ((u128)v.y << 64) | (u128)v.x;
  }
}

template <int E>
__device__ __forceinline__ void store_u128(uint8_t* base, uint64_t i, u128 v) {
  if constexpr (E == 1) {
    base[i] = (uint8_t)v;
  } else if constexpr (E == 2) {
    reinterpret_cast<uint16_t*>(base)[i] = (uint16_t)v;
  } else if constexpr (E == 4) {
    reinterpret_cast<uint32_t*>(base)[i] = (uint32_t)v;
  } else if constexpr (E == 8) {
    reinterpret_cast<unsigned long long*>(base)[i] = (unsigned long long)v;
  } else {
    reinterpret_cast<ulonglong2*>(base)[i] = make_ulonglong2((unsigned long long)v, (unsigned long long)(v >> 64));
  }
}

template <int E>
struct KeyView {
  const uint8_t* base;
  uint64_t n;
  uint32_t shift;
  __device__ __forceinline__ u128 key(uint64_t i) const { return load_u128<E>(base, i) >> shift; }
};

// First index in [lo, hi) whose key is >= k (strict = false) or > k (strict = true).
template <int E>
__device__ __forceinline__ uint64_t bsearch(const KeyView<E>& v, u128 k, uint64_t lo, uint64_t hi, bool strict) {
  while (lo < hi) {
    const uint64_t mid = lo + ((hi - lo) >> 1);
    const u128 m = v.key(mid);
    const bool before = strict ? (m <= k) : (m < k);
    if (before) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Same result as bsearch(v, k, from, n, strict) when the answer is >= from, found by
// galloping forward from `from` (cheap when consecutive searches land close together).
template <int E>
__device__ __forceinline__ uint64_t gallop(const KeyView<E>& v, u128 k, uint64_t from, bool strict) {
  uint64_t lo = from, step = 1, hi = from;
  while (hi < v.n) {
    const u128 m = v.key(hi);
    const bool before = strict ? (m <= k) : (m < k);
    if (!before) break;
    lo = hi + 1;
    hi = from + step;
    step <<= 1;
  }
  if (hi > v.n) hi = v.n;
  return bsearch<E>(v, k, lo, hi, strict);
}

// Warp-cooperative search: the first index in [lo, hi) whose key is >= k (> k when
// strict), or hi.  Each round the 32 lanes probe 32 evenly spaced keys and the range
// shrinks 32-fold, so a search over millions of keys costs ~5 dependent round trips
// instead of ~22 for a one-thread binary search.  All lanes return the same index.
template <int E>
__device__ __forceinline__ uint64_t warp_search(const KeyView<E>& v, u128 k, uint64_t lo, uint64_t hi, bool strict) {
  const uint32_t lane = threadIdx.x & 31;
  while (hi - lo > 32) {
    const uint64_t step = (hi - lo + 31) / 32;
    const uint64_t p = lo + lane * step;
    bool before = false;
    if (p < hi) {
      const u128 m = v.key(p);
      before = strict ? (m <= k) : (m < k);
    }
    const uint32_t cnt = __popc(__ballot_sync(0xffffffffu, before));
    if (cnt == 0) return lo;
    const uint64_t nlo = lo + (uint64_t)(cnt - 1) * step + 1;
    const uint64_t nhi = cnt < 32 ? min(hi, lo + (uint64_t)cnt * step) : hi;
    lo = nlo;
    hi = nhi;
  }
  bool before = false;
  if (lo + lane < hi) {
    const u128 m = v.key(lo + lane);
    before = strict ? (m <= k) : (m < k);
  }
  return lo + __popc(__ballot_sync(0xffffffffu, before));
}

// Block-strided copy of items [0, n): thread t moves items t, t + nt, ... as st(x, ld(x)),
// U loads in flight before their stores (a plain strided loop waits for each load in turn,
// one memory round trip per item).
template <int U, typename LD, typename ST>
__device__ __forceinline__ void block_stage(uint64_t n, uint32_t t, uint32_t nt, LD ld, ST st) {
  using V = decltype(ld(uint64_t(0)));
  for (uint64_t x0 = t; x0 < n; x0 += (uint64_t)U * nt) {
    V v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint64_t x = x0 + (uint64_t)u * nt;
      if (x < n) v[u] = ld(x);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint64_t x = x0 + (uint64_t)u * nt;
      if (x < n) st(x, v[u]);
    }
  }
}

}  // namespace rfx
