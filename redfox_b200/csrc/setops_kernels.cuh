// setops_kernels.cuh -- multiset set operations on sorted arrays and unique.
//
// STL / thrust semantics (thrust::set_union / set_difference in Union.cu:47-148 and
// Difference.cu:35-143; std::set_intersection as moderngpu's benchmarksets.cu:95-125
// checks it): a value occurring m times in A and n times in B occurs min(m, n) times in
// the intersection, max(m - n, 0) times in A - B and max(m, n) times in the union.
//   * intersection / difference keep A[i] when its rank within its run of equal values
//     is below / not below the number of equal values in B: keep bits per element, then a
//     stable compaction (the warp-segment form by default; the two-pass form and a
//     one-pass form with decoupled look-back as alternatives);
//   * union = merge(A, B - A) with A first on ties, by merge path (no scan needed);
//   * unique keeps the first of each run, in place.
#pragma once

#include <type_traits>

#include "search.cuh"

namespace rfx {

constexpr int kSetThreads = 256;
// Items per thread of the one-pass and two-pass forms: 8, with 4 and 16 as the tuner's
// alternatives (unique always 8); elements up to 8 bytes live in 64-bit registers.  The
// warp-segment form takes 16 (8 or 4 where a tile's window would not fit).
constexpr int kSetIPT = 8;
constexpr int kSetTile = kSetThreads * kSetIPT;
constexpr int kSetTileMin = kSetThreads * 4;   // the smallest tile: workspace sizing
constexpr int kMergeVT = 8;
constexpr int kMergeTile = kSetThreads * kMergeVT;

enum SetFilter : int { KEEP_MATCHED = 0, KEEP_UNMATCHED = 1, KEEP_HEADS = 2 };

// The register / shared-memory type of E-byte elements: compares in the narrowest word.
template <int E>
using SetWord = typename std::conditional<(E <= 4), uint32_t,
                                          typename std::conditional<(E <= 8), uint64_t, u128>::type>::type;

struct SetFilterArgs {
  const uint8_t* a;
  uint64_t na;
  const uint8_t* b;
  uint64_t nb;
  const uint8_t* prev;   // KEEP_HEADS: element before each tile (saved before in-place writes)
  const uint64_t* split; // KEEP_(UN)MATCHED: per tile (run start of its first element, B window)
  uint32_t wcap;         // two-pass and warp-segment forms: B window capacity (elements of dynamic shared memory)
  uint8_t* out;
  uint64_t* d_count;
  uint64_t* status;
  uint32_t* tile_counter;
  uint32_t* err;
};

__device__ __forceinline__ uint64_t block_exclusive_u32(uint32_t x, uint32_t* s_warp, uint32_t* total) {
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (uint32_t)o) incl += y;
  }
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  uint32_t wpre = 0, tot = 0;
  for (uint32_t w = 0; w < blockDim.x / 32; ++w) {
    if (w < warp) wpre += s_warp[w];
    tot += s_warp[w];
  }
  *total = tot;
  return wpre + incl - x;
}

// Binary searches in a sorted shared-memory window, compared in the window's own type
// (64-bit compares for elements up to 8 bytes).
template <typename T>
__device__ __forceinline__ uint32_t smem_lower(const T* w, uint32_t n, T k) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (w[mid] < k) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}
template <typename T>
__device__ __forceinline__ uint32_t smem_lower_strict(const T* w, uint32_t n, T k) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (w[mid] <= k) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Keep flags of one tile's items for KEEP_MATCHED / KEEP_UNMATCHED; every thread of the
// block calls it (it holds barriers).  v: the thread's IPT items (elements first ..);
// prev: the element before `first` when that lies in the tile; rs0 / blo0 / bhi: the
// tile's entries of set_split_kernel.
// The window of B values the tile's elements can equal, in shared memory.  A thread's
// items are consecutive and sorted: one binary search finds the first candidate in B
// for its first item, later items advance from there (merge order), and equal runs
// in B are measured by galloping.  An item's rank within its run of equal values is
// its distance from the run's first item: the last head (first item of a run) at or
// before it, from a block max-scan of the threads' last heads, or -- for the run that
// continues from the previous tile -- the run start found by set_split_kernel.
template <int E, int MODE, int IPT, typename WT>
__device__ __forceinline__ void set_keep_flags(const SetFilterArgs& p, uint64_t tile, const WT (&v)[IPT], WT prev,
                                               bool (&keep)[IPT], WT* s_b, uint32_t wcap, uint32_t* s_warp,
                                               uint64_t rs0, uint64_t blo0, uint64_t bhi) {
  constexpr int TILE = kSetThreads * IPT;
  const uint32_t t = threadIdx.x;
  const KeyView<E> B{p.b, p.nb, 0};
  // indices within the tile (32-bit): the thread's items are l0 .. l0 + IPT - 1
  const uint64_t tfirst = tile * TILE;
  const uint32_t tcount = (uint32_t)min((uint64_t)TILE, p.na - tfirst);
  const uint32_t l0 = t * IPT;
  const uint64_t bn = bhi > blo0 ? bhi - blo0 : 0;
  // staged windows keep one slot for a sentinel (the largest value) after their last element,
  // so the merge walk below needs no bounds check
  const bool staged = bn < (uint64_t)wcap;
  if (staged) {
    for (uint32_t x = t; x < (uint32_t)bn; x += kSetThreads) s_b[x] = (WT)B.key(blo0 + x);
    if (t == 0) s_b[bn] = ~(WT)0;
  }
  // heads of this thread's items (local index of its last head, or -1); the tile's first
  // item continues the previous tile's run unless it is the array's first
  int32_t last_head = -1;
  uint32_t heads = 0;
#pragma unroll
  for (int j = 0; j < IPT; ++j) {
    const uint32_t li = l0 + j;
    if (li >= tcount) continue;
    const bool h = li == 0 ? tfirst == 0 : v[j] != (j == 0 ? prev : v[j - 1]);
    if (h) {
      heads |= 1u << j;
      last_head = (int32_t)li;
    }
  }
  // exclusive max-scan of last_head over the block
  int32_t incl = last_head;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if ((t & 31) >= (uint32_t)o) incl = max(incl, y);
  }
  if ((t & 31) == 31) s_warp[t >> 5] = (uint32_t)(incl + 1);
  __syncthreads();
  int32_t before = -1;
  for (uint32_t w = 0; w < (t >> 5); ++w) before = max(before, (int32_t)s_warp[w] - 1);
  const int32_t ex = __shfl_up_sync(0xffffffffu, incl, 1);
  if ((t & 31) != 0) before = max(before, ex);
  // the run start as a tile-local index (negative: the run began in an earlier tile)
  int64_t run_start = before >= 0 ? (int64_t)before : (int64_t)rs0 - (int64_t)tfirst;
  // first candidate in B for the first item
  uint64_t pos = 0;
  if (l0 < tcount) {
    pos = staged ? (uint64_t)smem_lower(s_b, (uint32_t)bn, v[0]) : bsearch<E>(B, v[0], 0, p.nb, false);
  }
#pragma unroll
  for (int j = 0; j < IPT; ++j) {
    const uint32_t li = l0 + j;
    if (li >= tcount) continue;
    if ((heads >> j) & 1u) run_start = li;
    uint64_t nbeq;
    if (staged) {
      // usually zero or one step: two without a branch, then a loop for the rest (the
      // sentinel stops it at bn)
      uint32_t q = (uint32_t)pos;
      q += s_b[q] < v[j] ? 1u : 0u;
      q += s_b[q] < v[j] ? 1u : 0u;
      while (s_b[q] < v[j]) ++q;
      pos = q;
      nbeq = 0;
      if (q < (uint32_t)bn && s_b[q] == v[j]) {
        if (q + 1 >= (uint32_t)bn || s_b[q + 1] != v[j]) nbeq = 1;
        else nbeq = smem_lower_strict(s_b + q, (uint32_t)bn - q, v[j]);
      }
    } else {
      pos = j == 0 ? pos : (gallop<E>(B, v[j], pos, false));
      nbeq = gallop<E>(B, v[j], pos, true) - pos;
    }
    const uint64_t rank = (uint64_t)((int64_t)li - run_start);
    keep[j] = MODE == KEEP_MATCHED ? rank < nbeq : rank >= nbeq;
  }
  __syncthreads();
}

template <int E, int MODE, int IPT>
__global__ void __launch_bounds__(kSetThreads) set_filter_kernel(const SetFilterArgs p) {
  typedef SetWord<E> WT;
  constexpr int TILE = kSetThreads * IPT;
  constexpr int WCAP = E <= 8 ? 2048 : 1024;
  __shared__ WT s_b[MODE == KEEP_HEADS ? 1 : WCAP];
  __shared__ uint64_t s_rs0, s_blo, s_bhi;
  __shared__ uint32_t s_warp[kSetThreads / 32];
  __shared__ uint64_t s_prefix;
  __shared__ uint32_t s_tile;
  const uint32_t t = threadIdx.x;
  const uint64_t num_tiles = (p.na + TILE - 1) / TILE;
  const KeyView<E> A{p.a, p.na, 0};
  const KeyView<E> B{p.b, p.nb, 0};
  while (true) {
    if (t == 0) s_tile = atomicAdd(p.tile_counter, 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    if (tile >= num_tiles) break;
    const uint64_t first = tile * TILE + (uint64_t)t * IPT;
    WT v[IPT];
    bool keep[IPT];
    uint32_t kept = 0;
    // every input of this tile is read before its aggregate is published, which keeps
    // the in-place unique safe (writes land below the inputs of later tiles)
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
      const uint64_t i = first + j;
      keep[j] = false;
      if (i < p.na) v[j] = (WT)A.key(i);
    }
    if constexpr (MODE == KEEP_HEADS) {
      WT before = 0;
      if (first < p.na && first > 0) {
        before = (WT)((t == 0) ? load_u128<E>(p.prev, tile) : A.key(first - 1));
      }
#pragma unroll
      for (int j = 0; j < IPT; ++j) {
        const uint64_t i = first + j;
        if (i >= p.na) continue;
        keep[j] = i == 0 || v[j] != (j == 0 ? before : v[j - 1]);
      }
    } else {
      if (t == 0) s_rs0 = p.split[3 * tile];
      if (t == 1) s_blo = p.split[3 * tile + 1];
      if (t == 2) s_bhi = p.split[3 * tile + 2];
      __syncthreads();
      const uint64_t tfirst = tile * TILE;
      const WT prev = first < p.na && first > tfirst ? (WT)A.key(first - 1) : (WT)0;
      set_keep_flags<E, MODE, IPT, WT>(p, tile, v, prev, keep, s_b, WCAP, s_warp, s_rs0, s_blo, s_bhi);
    }
#pragma unroll
    for (int j = 0; j < IPT; ++j) kept += keep[j] ? 1u : 0u;
    uint32_t btot;
    const uint64_t ex = block_exclusive_u32(kept, s_warp, &btot);
    if ((t >> 5) == 0) {
      const uint64_t pre = lookback_exclusive<4>(p.status, (uint32_t)tile, btot, p.err);
      if (t == 0) {
        s_prefix = pre;
        if (tile == num_tiles - 1) *p.d_count = pre + btot;
      }
    }
    __syncthreads();
    uint64_t pos = s_prefix + ex;
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
      if (!keep[j]) continue;
      if (pos < p.na) store_u128<E>(p.out, pos, v[j]);
      ++pos;
    }
    __syncthreads();
  }
  if (p.na == 0 && blockIdx.x == 0 && t == 0) *p.d_count = 0;
}


// ------------------------------------------------------------------ two-pass filter
// Intersection / difference (and union's B - A) in two passes with no block waiting on
// another: set_mark_kernel finds every element's keep flag (the rule of set_filter_kernel)
// and writes one bit per element and a count per tile; set_offsets_kernel turns the counts
// into each tile's output offset and the total; set_compact_kernel writes the kept
// elements in order.  Tiles are assigned statically (block b takes tiles b, b + grid, ...),
// so nothing depends on blocks being resident together.  The output must not overlap A.

// One thread's keep bits for IPT items (IPT / 8 mask bytes).
template <int IPT>
using MaskWord = typename std::conditional<(IPT <= 8), uint8_t, uint16_t>::type;

template <typename T>
__device__ __forceinline__ T shfl_up_t(T x, int d) {
  if constexpr (sizeof(T) <= 8) {
    return (T)__shfl_up_sync(0xffffffffu, (unsigned long long)x, d);
  } else {
    const unsigned long long lo = __shfl_up_sync(0xffffffffu, (unsigned long long)x, d);
    const unsigned long long hi = __shfl_up_sync(0xffffffffu, (unsigned long long)(x >> 64), d);
    return ((T)hi << 64) | (T)lo;
  }
}

template <int E, int MODE, int IPT>
__global__ void __launch_bounds__(kSetThreads) set_mark_kernel(const SetFilterArgs p, uint8_t* mask, uint32_t* counts) {
  typedef SetWord<E> WT;
  constexpr int kMarkIPT = IPT;
  constexpr int kTile = kSetThreads * IPT;
  // the B window in dynamic shared memory: p.wcap elements, sized at launch from nb / na
  extern __shared__ __align__(16) uint8_t s_dyn[];
  WT* s_b = reinterpret_cast<WT*>(s_dyn);
  __shared__ uint32_t s_warp[kSetThreads / 32];
  const uint32_t t = threadIdx.x, lane = t & 31;
  const uint64_t num_tiles = (p.na + kTile - 1) / kTile;
  const KeyView<E> A{p.a, p.na, 0};
  // the split entries of the block's next tile are loaded one tile ahead, so the B window
  // can be staged while the tile's items are still in flight
  uint64_t rs0 = 0, blo0 = 0, bhi = 0;
  if (blockIdx.x < num_tiles) {
    rs0 = p.split[3ull * blockIdx.x];
    blo0 = p.split[3ull * blockIdx.x + 1];
    bhi = p.split[3ull * blockIdx.x + 2];
  }
  for (uint64_t tile = blockIdx.x; tile < num_tiles; tile += gridDim.x) {
    const uint64_t tfirst = tile * kTile;
    const uint64_t first = tfirst + (uint64_t)t * kMarkIPT;
    // the items and the element before them (the previous lane's last item, or loaded by
    // a warp's first lane): all loads in flight together with the B window's
    WT v[kMarkIPT];
#pragma unroll
    for (int j = 0; j < kMarkIPT; ++j) v[j] = first + j < p.na ? (WT)A.key(first + j) : (WT)0;
    WT before = lane == 0 && first < p.na && first > tfirst ? (WT)A.key(first - 1) : (WT)0;
    const uint64_t nt = tile + gridDim.x;
    uint64_t nrs0 = 0, nblo = 0, nbhi = 0;
    if (nt < num_tiles) {
      nrs0 = p.split[3 * nt];
      nblo = p.split[3 * nt + 1];
      nbhi = p.split[3 * nt + 2];
    }
    const WT up = shfl_up_t(v[kMarkIPT - 1], 1);
    if (lane != 0) before = up;
    bool keep[kMarkIPT];
#pragma unroll
    for (int j = 0; j < kMarkIPT; ++j) keep[j] = false;
    set_keep_flags<E, MODE, kMarkIPT, WT>(p, tile, v, before, keep, s_b, p.wcap, s_warp, rs0, blo0, bhi);
    uint32_t bits = 0;
#pragma unroll
    for (int j = 0; j < kMarkIPT; ++j) bits |= (keep[j] ? 1u : 0u) << j;
    reinterpret_cast<MaskWord<IPT>*>(mask)[tile * kSetThreads + t] = (MaskWord<IPT>)bits;
    const uint32_t wsum = __reduce_add_sync(0xffffffffu, (uint32_t)__popc(bits));
    if (lane == 0) s_warp[t >> 5] = wsum;
    __syncthreads();
    if (t == 0) {
      uint32_t c = 0;
      for (int w = 0; w < kSetThreads / 32; ++w) c += s_warp[w];
      counts[tile] = c;
    }
    __syncthreads();   // s_warp and s_b are reused by the next tile
    rs0 = nrs0;
    blo0 = nblo;
    bhi = nbhi;
  }
}

// Exclusive offsets of the per-tile counts and their total, by one block of 1024 threads:
// 8 consecutive counts per thread and round.
constexpr int kOffsetThreads = 1024;

__global__ void __launch_bounds__(kOffsetThreads)
set_offsets_kernel(const uint32_t* counts, uint64_t tiles, uint64_t* offsets, uint64_t* d_count) {
  __shared__ uint64_t s_w[kOffsetThreads / 32];
  __shared__ uint64_t s_carry;
  const uint32_t t = threadIdx.x, lane = t & 31, w = t >> 5;
  if (t == 0) s_carry = 0;
  __syncthreads();
  for (uint64_t base = 0; base < tiles; base += 8ull * kOffsetThreads) {
    const uint64_t i0 = base + 8ull * t;
    uint32_t c[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) c[j] = i0 + j < tiles ? counts[i0 + j] : 0u;
    uint64_t sum = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) sum += c[j];
    uint64_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t y = __shfl_up_sync(0xffffffffu, (unsigned long long)incl, o);
      if (lane >= (uint32_t)o) incl += y;
    }
    if (lane == 31) s_w[w] = incl;
    __syncthreads();
    uint64_t wpre = 0, tot = 0;
    for (uint32_t x = 0; x < kOffsetThreads / 32; ++x) {
      if (x < w) wpre += s_w[x];
      tot += s_w[x];
    }
    uint64_t run = s_carry + wpre + incl - sum;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (i0 + j < tiles) offsets[i0 + j] = run;
      run += c[j];
    }
    __syncthreads();   // every thread has read s_carry and s_w
    if (t == 0) s_carry += tot;
    __syncthreads();
  }
  if (t == 0) *d_count = s_carry;
}

// The kept elements of each tile (mask bits) at the tile's offset, in order; only kept
// elements are read.  Writes at or beyond `cap` are dropped.
template <int E, int IPT>
__global__ void __launch_bounds__(kSetThreads)
set_compact_kernel(const uint8_t* a, uint64_t na, const uint8_t* mask, const uint64_t* offsets, uint8_t* out,
                   uint64_t cap) {
  constexpr int kMarkIPT = IPT;
  constexpr int kTile = kSetThreads * IPT;
  __shared__ uint32_t s_warp[kSetThreads / 32];
  const uint32_t t = threadIdx.x, lane = t & 31, w = t >> 5;
  const uint64_t num_tiles = (na + kTile - 1) / kTile;
  for (uint64_t tile = blockIdx.x; tile < num_tiles; tile += gridDim.x) {
    const uint32_t bits = reinterpret_cast<const MaskWord<IPT>*>(mask)[tile * kSetThreads + t];
    const uint64_t base = offsets[tile];
    const uint32_t c = __popc(bits);
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o) incl += y;
    }
    if (lane == 31) s_warp[w] = incl;
    __syncthreads();
    uint32_t wpre = 0;
    for (uint32_t x = 0; x < w; ++x) wpre += s_warp[x];
    uint64_t pos = base + wpre + incl - c;
    const uint64_t first = tile * kTile + (uint64_t)t * kMarkIPT;
#pragma unroll
    for (int j = 0; j < kMarkIPT; ++j) {
      if (!((bits >> j) & 1u)) continue;
      if (pos < cap) store_u128<E>(out, pos, load_u128<E>(a, first + j));
      ++pos;
    }
    __syncthreads();   // s_warp is reused by the next tile
  }
}

// Per tile of A (TILE elements): the start of the run of equal values containing the
// tile's first element, and the window of B that can equal the tile's values -- one warp
// per search, all tiles at once, so the filter kernel's tiles do not each wait on chains
// of dependent loads.
template <int E, int TILE>
__global__ void set_split_kernel(const uint8_t* a, uint64_t na, const uint8_t* b, uint64_t nb, uint64_t* split) {
  const KeyView<E> A{a, na, 0};
  const KeyView<E> B{b, nb, 0};
  const uint64_t tiles = (na + TILE - 1) / TILE;
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x / 32);
  for (uint64_t x = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32; x < 3 * tiles; x += warps) {
    const uint64_t tile = x / 3, kind = x % 3;
    const uint64_t tfirst = tile * TILE;
    const uint64_t tlast = min(na, tfirst + TILE) - 1;
    uint64_t r;
    if (kind == 0) {
      const u128 k0 = A.key(tfirst);
      // a tile whose first element starts a new run needs no search
      r = (tfirst == 0 || A.key(tfirst - 1) != k0) ? tfirst : warp_search<E>(A, k0, 0, tfirst, false);
    } else if (kind == 1) {
      r = warp_search<E>(B, A.key(tfirst), 0, nb, false);
    } else {
      r = warp_search<E>(B, A.key(tlast), 0, nb, true);
    }
    if ((threadIdx.x & 31) == 0) split[x] = r;
  }
}

// ------------------------------------------------------------------ warp-segment filter
// The two-pass form with one barrier per tile, for 4- and 8-byte elements in 16-byte aligned
// arrays.  The block's only shared step is the tile's B window, bulk-copied into one of two
// buffers by cp.async while the previous tile is being filtered (the barrier that publishes
// a window also shows that every thread is done with the buffer the next copy overwrites).
// Everything else belongs to one warp and its segment of 32 x IPT consecutive elements:
// the run start of the segment's first element (from the element before it, a backward
// warp scan when its run crosses into the segment, or the tile's run start), the run heads
// by a warp max-scan, one binary search per thread into the window and a merge walk over
// its items, the keep bits and a count per warp.  An item of rank r within its run of equal
// values is matched when B holds at least r + 1 copies of it, that is when the window
// element r places after the item's lower bound still equals it.
constexpr int kSegWarps = kSetThreads / 32;

// Per boundary x of A's tiles (x < tiles: the tile's first element; x = tiles: A's last
// element), one warp: the start of the run of equal values containing the element (tile
// boundaries only) and the element's lower and upper bounds in B, as split[3x .. 3x + 2].
// Tile k's B window is [lower bound of boundary k, upper bound of boundary k + 1): every
// value of tile k lies between its own first element and boundary k + 1's.
template <int E, int TILE>
__global__ void set_bounds_kernel(const uint8_t* a, uint64_t na, const uint8_t* b, uint64_t nb, uint64_t* split) {
  const KeyView<E> A{a, na, 0};
  const KeyView<E> B{b, nb, 0};
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t tiles = (na + TILE - 1) / TILE;
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x / 32);
  for (uint64_t x = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32; x <= tiles; x += warps) {
    const uint64_t i = x < tiles ? x * TILE : na - 1;
    const u128 k = A.key(i);
    uint64_t rs = i;
    if (x < tiles && i > 0 && A.key(i - 1) == k) rs = warp_search<E>(A, k, 0, i, false);
    const uint64_t lb = warp_search<E>(B, k, 0, nb, false);
    // B's run of k starts at lb: its first 32 elements in one probe, a search past them
    const uint64_t p = lb + lane;
    const uint32_t m = __ballot_sync(0xffffffffu, p < nb && B.key(p) == k);
    uint64_t ub = lb + (uint64_t)__popc(m);
    if (m == 0xffffffffu) ub = warp_search<E>(B, k, lb + 32, nb, true);
    if (lane == 0) {
      split[3 * x] = rs;
      split[3 * x + 1] = lb;
      split[3 * x + 2] = ub;
    }
  }
}

// Elements of a B window buffer: the window's capacity, the elements before it that its
// 16-byte aligned copy brings along, and the sentinel.
template <int E>
__host__ __device__ constexpr uint32_t seg_buffer_elems(uint32_t wcap) {
  return wcap + 16u / E + 4u;
}

// Items first .. first + IPT - 1 of a 16-byte aligned array (first * E a multiple of 16).
template <int E, int IPT, typename WT>
__device__ __forceinline__ void load_items_vec(const uint8_t* a, uint64_t first, WT (&v)[IPT]) {
  static_assert((IPT * E) % 16 == 0, "whole 16-byte chunks");
  const uint4* p = reinterpret_cast<const uint4*>(a + first * E);
#pragma unroll
  for (int c = 0; c < IPT * E / 16; ++c) {
    const uint4 r = __ldg(p + c);
    if constexpr (E == 4) {
      v[4 * c] = r.x;
      v[4 * c + 1] = r.y;
      v[4 * c + 2] = r.z;
      v[4 * c + 3] = r.w;
    } else {
      v[2 * c] = ((uint64_t)r.y << 32) | r.x;
      v[2 * c + 1] = ((uint64_t)r.w << 32) | r.z;
    }
  }
}

template <int E, int MODE, int IPT>
__global__ void __launch_bounds__(kSetThreads)
set_mark_seg_kernel(const SetFilterArgs p, uint8_t* mask, uint32_t* counts, uint32_t* wcounts) {
  static_assert(E == 4 || E == 8, "4- and 8-byte elements");
  typedef SetWord<E> WT;
  constexpr int kTile = kSetThreads * IPT;
  constexpr uint32_t kSeg = 32 * IPT;
  extern __shared__ __align__(16) uint8_t s_dyn[];
  __shared__ uint32_t s_cnt[2];
  const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const uint64_t num_tiles = (p.na + kTile - 1) / kTile;
  const KeyView<E> A{p.a, p.na, 0};
  const KeyView<E> B{p.b, p.nb, 0};
  const uint32_t wcap = p.wcap, bufe = seg_buffer_elems<E>(wcap);
  if (t < 2) s_cnt[t] = 0;
  // a tile's window: [lo, hi) of B, staged when it holds fewer than wcap elements; the
  // entries are read one tile before its copy is issued
  struct Win {
    uint64_t rs, lo, hi;
  };
  auto entries = [&](uint64_t tile) -> Win {
    Win w{0, 0, 0};
    if (tile < num_tiles) {
      w.rs = p.split[3 * tile];
      w.lo = p.split[3 * tile + 1];
      w.hi = p.split[3 * tile + 5];
    }
    return w;
  };
  auto staged = [&](const Win& w) { return w.hi >= w.lo && w.hi - w.lo < wcap; };
  // the copy of window w into buffer `buf`: its elements from 16-byte aligned byte b0, the
  // window starting `off` elements in
  auto prefetch = [&](const Win& w, uint32_t buf) {
    if (!staged(w)) return;
    const uint64_t b0 = (w.lo * E) & ~15ull;
    block_prefetch16(s_dyn + (size_t)buf * bufe * sizeof(WT), p.b, b0, w.hi * E - b0, p.nb * E, kSetThreads);
  };
  uint64_t tile = blockIdx.x;
  Win cur = entries(tile);
  Win nxt = entries(tile + gridDim.x);
  prefetch(cur, 0);
  cp_async_commit();
  uint32_t it = 0;
  for (; tile < num_tiles; tile += gridDim.x, ++it) {
    const uint32_t buf = it & 1;
    const uint64_t tfirst = tile * kTile;
    const uint64_t seg = tfirst + (uint64_t)warp * kSeg;
    const uint64_t first = seg + (uint64_t)lane * IPT;
    // the items, and for a warp's first lane the element before them
    WT v[IPT];
    if (tfirst + kTile <= p.na) {
      load_items_vec<E, IPT, WT>(p.a, first, v);
    } else {
#pragma unroll
      for (int j = 0; j < IPT; ++j) v[j] = first + j < p.na ? (WT)A.key(first + j) : ~(WT)0;
    }
    WT before = lane == 0 && first > 0 && first < p.na ? (WT)A.key(first - 1) : (WT)0;
    const Win after = entries(tile + 2ull * gridDim.x);
    // this tile's window: its copies done, the sentinel after its last element written by
    // the thread whose copy covers that slot
    const bool st = staged(cur);
    const uint32_t off = (uint32_t)(((cur.lo * E) & 15ull) / E);
    const uint32_t bn = st ? (uint32_t)(cur.hi - cur.lo) : 0u;
    WT* s_b = reinterpret_cast<WT*>(s_dyn) + (size_t)buf * bufe + off;
    cp_async_wait<0>();
    if (st && t == (((off + bn) * E) / 16) % kSetThreads) s_b[bn] = ~(WT)0;
    __syncthreads();
    if (t == 0 && it > 0) {
      counts[tile - gridDim.x] = s_cnt[buf ^ 1u];
      s_cnt[buf ^ 1u] = 0;
    }
    prefetch(nxt, buf ^ 1u);
    cp_async_commit();
    uint32_t bits = 0;
    if (seg < p.na) {
      // heads: an item differing from the one before it (the array's first element is one)
      const WT up = shfl_up_t(v[IPT - 1], 1);
      if (lane != 0) before = up;
      uint32_t heads = 0;
      int32_t last_head = -1;
#pragma unroll
      for (int j = 0; j < IPT; ++j) {
        const bool h = j == 0 ? (first == 0 || v[0] != before) : v[j] != v[j - 1];
        if (h) {
          heads |= 1u << j;
          last_head = (int32_t)(lane * IPT + j);
        }
      }
      int32_t incl = last_head;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl = max(incl, y);
      }
      const int32_t prior = __shfl_up_sync(0xffffffffu, incl, 1);
      // the run start of the segment's first element, relative to the segment
      int64_t wstart = 0;
      const WT v0 = __shfl_sync(0xffffffffu, v[0], 0);
      if (warp == 0) {
        wstart = (int64_t)cur.rs - (int64_t)seg;
      } else if (__shfl_sync(0xffffffffu, before, 0) == v0) {
        // the run crosses into this segment: the last element before it that differs, at
        // or after the tile's first element, else the tile's run start
        int64_t found = -1;
        for (uint64_t hi = seg;;) {
          const bool diff = hi > tfirst + lane && (WT)A.key(hi - 1 - lane) != v0;
          const uint32_t m = __ballot_sync(0xffffffffu, diff);
          if (m) {
            found = (int64_t)(hi - (uint64_t)__ffs(m));
            break;
          }
          if (hi <= tfirst + 32) break;
          hi -= 32;
        }
        wstart = (found >= 0 ? found + 1 : (int64_t)cur.rs) - (int64_t)seg;
      }
      int64_t rs = lane != 0 && prior >= 0 ? (int64_t)prior : wstart;
      if (st) {
        // s_b[bn] is the largest value: the walk stops there without a bounds check
        uint32_t q = smem_lower(s_b, bn, v[0]);
        WT bq = s_b[q];
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
          const WT x = v[j];
          while (bq < x) bq = s_b[++q];
          const bool head = (heads >> j) & 1u;
          const int64_t li = (int64_t)(lane * IPT + j);
          if (head) rs = li;
          bool m = bq == x && q < bn;
          if (m && !head) {
            const uint64_t r = (uint64_t)(li - rs);
            m = r < (uint64_t)(bn - q) && s_b[q + (uint32_t)r] == x;
          }
          bits |= (MODE == KEEP_MATCHED ? m : !m) ? 1u << j : 0u;
        }
      } else {
        uint64_t pos = bsearch<E>(B, v[0], cur.lo, cur.hi, false);
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
          const WT x = v[j];
          pos = gallop<E>(B, x, pos, false);
          const bool head = (heads >> j) & 1u;
          const int64_t li = (int64_t)(lane * IPT + j);
          if (head) rs = li;
          uint64_t nbeq = 0;
          if (pos < p.nb && (WT)B.key(pos) == x) nbeq = head ? 1 : gallop<E>(B, x, pos, true) - pos;
          const bool m = (uint64_t)(li - rs) < nbeq;
          bits |= (MODE == KEEP_MATCHED ? m : !m) ? 1u << j : 0u;
        }
      }
      if (first >= p.na) bits = 0;
      else if (p.na - first < (uint64_t)IPT) bits &= (1u << (uint32_t)(p.na - first)) - 1u;
    }
    reinterpret_cast<MaskWord<IPT>*>(mask)[tile * kSetThreads + t] = (MaskWord<IPT>)bits;
    const uint32_t wsum = __reduce_add_sync(0xffffffffu, (uint32_t)__popc(bits));
    if (lane == 0) {
      wcounts[tile * kSegWarps + warp] = wsum;
      atomicAdd(&s_cnt[buf], wsum);
    }
    cur = nxt;
    nxt = after;
  }
  cp_async_wait<0>();
  __syncthreads();
  if (t == 0 && it > 0) counts[tile - gridDim.x] = s_cnt[(it - 1) & 1u];
}

// The kept elements of each segment at the tile's offset plus the counts of the tile's
// earlier segments, gathered per warp in shared memory and written out in coalesced runs.
// Writes at or beyond `cap` are dropped.
template <int E, int IPT>
__global__ void __launch_bounds__(kSetThreads)
set_compact_seg_kernel(const uint8_t* a, uint64_t na, const uint8_t* mask, const uint64_t* offsets,
                       const uint32_t* wcounts, uint8_t* out, uint64_t cap) {
  static_assert(E == 4 || E == 8, "4- and 8-byte elements");
  typedef SetWord<E> WT;
  constexpr int kTile = kSetThreads * IPT;
  constexpr uint32_t kSeg = 32 * IPT;
  __shared__ WT s_out[kSegWarps][kSeg];
  const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const uint64_t num_tiles = (na + kTile - 1) / kTile;
  const KeyView<E> A{a, na, 0};
  // a tile's keep bits, its warps' counts and its offset, loaded one tile ahead
  auto load = [&](uint64_t tile, uint32_t& bits, uint32_t& wc, uint64_t& off) {
    bits = wc = 0;
    off = 0;
    if (tile >= num_tiles) return;
    bits = reinterpret_cast<const MaskWord<IPT>*>(mask)[tile * kSetThreads + t];
    wc = lane < (uint32_t)kSegWarps ? wcounts[tile * kSegWarps + lane] : 0u;
    off = offsets[tile];
  };
  uint32_t bits, wc;
  uint64_t off;
  load(blockIdx.x, bits, wc, off);
  for (uint64_t tile = blockIdx.x; tile < num_tiles; tile += gridDim.x) {
    uint32_t nbits, nwc;
    uint64_t noff;
    load(tile + gridDim.x, nbits, nwc, noff);
    const uint32_t wpre = __reduce_add_sync(0xffffffffu, lane < warp ? wc : 0u);
    const uint32_t c = __popc(bits);
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o) incl += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    if (total != 0) {
      const uint64_t first = tile * kTile + (uint64_t)warp * kSeg + (uint64_t)lane * IPT;
      if (bits) {
        WT v[IPT];
        if (tile * kTile + kTile <= na) {
          load_items_vec<E, IPT, WT>(a, first, v);
        } else {
#pragma unroll
          for (int j = 0; j < IPT; ++j) v[j] = first + j < na ? (WT)A.key(first + j) : (WT)0;
        }
        uint32_t k = incl - c;
#pragma unroll
        for (int j = 0; j < IPT; ++j)
          if ((bits >> j) & 1u) s_out[warp][k++] = v[j];
      }
      __syncwarp();
      const uint64_t base = off + wpre;
      for (uint32_t x = lane; x < total; x += 32)
        if (base + x < cap) store_u128<E>(out, base + x, (u128)s_out[warp][x]);
      __syncwarp();   // s_out is reused by the warp's next segment
    }
    bits = nbits;
    wc = nwc;
    off = noff;
  }
}

// The element before each tile, saved before an in-place pass overwrites it.
template <int E>
__global__ void tile_prev_kernel(const uint8_t* a, uint64_t n, uint8_t* prev, uint64_t tile_items) {
  const uint64_t tiles = (n + tile_items - 1) / tile_items;
  for (uint64_t tl = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; tl < tiles; tl += (uint64_t)gridDim.x * blockDim.x)
    store_u128<E>(prev, tl, tl == 0 ? (u128)0 : load_u128<E>(a, tl * tile_items - 1));
}

// Merge of A and D (A first on ties): the union.  Merge path: per tile of kMergeTile
// outputs, two warps find where the tile's first and last diagonals cross (32-way searches
// over the global arrays), the tile's runs of A and D are staged in shared memory, each
// thread finds its own diagonal there and merges kMergeVT outputs.

// The number of A elements among the first k outputs of merge(A, D) (A first on ties), by
// one warp (all lanes return it).
template <int E>
__device__ __forceinline__ uint64_t merge_path_warp(const KeyView<E>& A, const KeyView<E>& D, uint64_t k) {
  const uint32_t lane = threadIdx.x & 31;
  // the answer is the first i in [lo, hi) with A[i] > D[k - i - 1], or hi
  uint64_t lo = k > D.n ? k - D.n : 0, hi = k < A.n ? k : A.n;
  while (hi - lo > 32) {
    const uint64_t step = (hi - lo + 31) / 32;
    const uint64_t p = lo + lane * step;
    const bool before = p < hi && A.key(p) <= D.key(k - p - 1);
    const uint32_t cnt = __popc(__ballot_sync(0xffffffffu, before));
    if (cnt == 0) return lo;
    const uint64_t nlo = lo + (uint64_t)(cnt - 1) * step + 1;
    const uint64_t nhi = cnt < 32 ? min(hi, lo + (uint64_t)cnt * step) : hi;
    lo = nlo;
    hi = nhi;
  }
  const uint64_t p = lo + lane;
  const bool before = p < hi && A.key(p) <= D.key(k - p - 1);
  return lo + __popc(__ballot_sync(0xffffffffu, before));
}

template <int E>
__global__ void __launch_bounds__(kSetThreads)
merge_kernel(const uint8_t* a, uint64_t na, const uint8_t* d, uint64_t nd_max, const uint64_t* d_nd, uint8_t* out,
             uint64_t* d_count) {
  typedef SetWord<E> WT;
  __shared__ WT s_m[kMergeTile];   // the tile's A run, then its D run
  __shared__ uint64_t s_i[2];
  const uint32_t t = threadIdx.x;
  const uint64_t nd = d_nd ? min(nd_max, *d_nd) : nd_max;
  const uint64_t total = na + nd;
  if (blockIdx.x == 0 && t == 0) *d_count = total;
  const KeyView<E> A{a, na, 0};
  const KeyView<E> D{d, nd, 0};
  for (uint64_t k0 = (uint64_t)blockIdx.x * kMergeTile; k0 < total; k0 += (uint64_t)gridDim.x * kMergeTile) {
    const uint64_t k1 = min(k0 + (uint64_t)kMergeTile, total);
    if (t < 32) {
      const uint64_t i = merge_path_warp<E>(A, D, k0);
      if (t == 0) s_i[0] = i;
    } else if (t < 64) {
      const uint64_t i = merge_path_warp<E>(A, D, k1);
      if (t == 32) s_i[1] = i;
    }
    __syncthreads();
    const uint64_t i0 = s_i[0], i1 = s_i[1];
    const uint32_t nat = (uint32_t)(i1 - i0), ndt = (uint32_t)((k1 - i1) - (k0 - i0));
    const uint64_t j0 = k0 - i0;
    for (uint32_t x = t; x < nat + ndt; x += kSetThreads)
      s_m[x] = x < nat ? (WT)A.key(i0 + x) : (WT)D.key(j0 + (x - nat));
    __syncthreads();
    const WT* sa = s_m;
    const WT* sd = s_m + nat;
    // this thread's diagonal within the tile
    const uint32_t kt = t * kMergeVT, kn = nat + ndt;
    if (kt < kn) {
      uint32_t lo = kt > ndt ? kt - ndt : 0u, hi = kt < nat ? kt : nat;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (sa[mid] <= sd[kt - mid - 1]) lo = mid + 1;
        else hi = mid;
      }
      uint32_t ia = lo, id = kt - lo;
#pragma unroll
      for (int v = 0; v < kMergeVT; ++v) {
        const uint32_t kk = kt + v;
        if (kk >= kn) break;
        const bool take_a = id >= ndt || (ia < nat && sa[ia] <= sd[id]);
        const WT x = take_a ? sa[ia] : sd[id];
        store_u128<E>(out, k0 + kk, (u128)x);
        if (take_a) ++ia;
        else ++id;
      }
    }
    __syncthreads();   // s_m and s_i are reused by the next tile
  }
}

// The staged merge for 4- and 8-byte elements in 16-byte aligned arrays: where each tile's
// diagonals cross is found beforehand for all tiles at once (merge_partition_kernel, one warp
// per tile boundary), the tile's runs of A and D are bulk-copied by cp.async into one of two
// buffers while the previous tile merges, and each thread merges kMergeVT consecutive outputs
// in registers and stores them as 16-byte vectors.
template <int E>
__global__ void merge_partition_kernel(const uint8_t* a, uint64_t na, const uint8_t* d, uint64_t nd_max,
                                       const uint64_t* d_nd, uint64_t* mp) {
  const uint64_t nd = d_nd ? min(nd_max, *d_nd) : nd_max;
  const uint64_t total = na + nd;
  const uint64_t tiles = (total + kMergeTile - 1) / kMergeTile;
  const KeyView<E> A{a, na, 0};
  const KeyView<E> D{d, nd, 0};
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x / 32);
  for (uint64_t x = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32; x <= tiles; x += warps) {
    const uint64_t i = merge_path_warp<E>(A, D, min(x * kMergeTile, total));
    if ((threadIdx.x & 31) == 0) mp[x] = i;
  }
}

// Elements of one merge input buffer: a tile's runs of A and D (kMergeTile together), each
// with the elements its 16-byte aligned copy brings along before and after it, and room for
// the reads a thread's merge makes past a run's end (at most kMergeVT, never used).
template <int E>
__host__ __device__ constexpr uint32_t merge_buffer_elems() {
  return kMergeTile + 4u * (16u / E) + 2u * kMergeVT;
}
// Dynamic shared memory of merge_staged_kernel<E>: two input buffers.
template <int E>
__host__ __device__ constexpr size_t merge_staged_smem() {
  return 2 * (size_t)merge_buffer_elems<E>() * E;
}

template <int E>
__global__ void __launch_bounds__(kSetThreads)
merge_staged_kernel(const uint8_t* a, uint64_t na, const uint8_t* d, uint64_t nd_max, const uint64_t* d_nd,
                    const uint64_t* mp, uint8_t* out, uint64_t* d_count) {
  static_assert(E == 4 || E == 8, "4- and 8-byte elements");
  typedef SetWord<E> WT;
  constexpr uint32_t kBuf = merge_buffer_elems<E>();
  // dynamic shared memory: two input buffers of kBuf elements
  extern __shared__ __align__(16) uint8_t s_dyn[];
  WT* const s_in0 = reinterpret_cast<WT*>(s_dyn);
  const uint32_t t = threadIdx.x;
  const uint64_t nd = d_nd ? min(nd_max, *d_nd) : nd_max;
  const uint64_t total = na + nd;
  const uint64_t tiles = (total + kMergeTile - 1) / kMergeTile;
  if (blockIdx.x == 0 && t == 0) *d_count = total;
  // a tile's runs: A [i0, i1), D [k0 - i0, k1 - i1); where each sits in its buffer
  struct Runs {
    uint64_t k0, i0, i1, j0, j1;
    uint32_t offa, dstart;
  };
  auto runs = [&](uint64_t tile) -> Runs {
    Runs r{};
    r.k0 = total;   // past the last tile: nothing to copy
    if (tile < tiles) {
      r.k0 = tile * kMergeTile;
      const uint64_t k1 = min(r.k0 + (uint64_t)kMergeTile, total);
      r.i0 = mp[tile];
      r.i1 = mp[tile + 1];
      r.j0 = r.k0 - r.i0;
      r.j1 = k1 - r.i1;
      r.offa = (uint32_t)(((r.i0 * E) & 15ull) / E);
      // D's copy starts at the next 16-byte boundary after A's
      const uint64_t abytes = r.i1 * E - ((r.i0 * E) & ~15ull);
      r.dstart = (uint32_t)(((abytes + 15ull) & ~15ull) / E);
    }
    return r;
  };
  auto prefetch = [&](const Runs& r, uint32_t buf) {
    if (r.k0 >= total) return;
    uint8_t* base = reinterpret_cast<uint8_t*>(s_in0 + (size_t)buf * kBuf);
    const uint64_t a0 = (r.i0 * E) & ~15ull, d0 = (r.j0 * E) & ~15ull;
    block_prefetch16(base, a, a0, r.i1 * E - a0, na * E, kSetThreads);
    block_prefetch16(base + (size_t)r.dstart * E, d, d0, r.j1 * E - d0, nd * E, kSetThreads);
  };
  uint64_t tile = blockIdx.x;
  Runs cur = runs(tile);
  prefetch(cur, 0);
  cp_async_commit();
  for (uint32_t it = 0; tile < tiles; tile += gridDim.x, ++it) {
    const uint32_t buf = it & 1;
    const Runs nxt = runs(tile + gridDim.x);
    cp_async_wait<0>();
    __syncthreads();   // this tile's runs are in; every thread is done with the other buffer
    prefetch(nxt, buf ^ 1u);
    cp_async_commit();
    const WT* sa = s_in0 + (size_t)buf * kBuf + cur.offa;
    const WT* sd = s_in0 + (size_t)buf * kBuf + cur.dstart + (uint32_t)(((cur.j0 * E) & 15ull) / E);
    const uint32_t nat = (uint32_t)(cur.i1 - cur.i0), ndt = (uint32_t)(cur.j1 - cur.j0);
    const uint32_t kn = nat + ndt, kt = t * kMergeVT;
    if (kt < kn) {
      uint32_t lo = kt > ndt ? kt - ndt : 0u, hi = kt < nat ? kt : nat;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (sa[mid] <= sd[kt - mid - 1]) lo = mid + 1;
        else hi = mid;
      }
      // the thread's outputs in registers; the heads of both runs carried, one load a step
      uint32_t ia = lo, id = kt - lo;
      WT va = sa[ia], vd = sd[id];   // past a run's end: buffer slack, never taken
      WT o[kMergeVT];
#pragma unroll
      for (int v = 0; v < kMergeVT; ++v) {
        const bool take_a = id >= ndt || (ia < nat && va <= vd);
        o[v] = take_a ? va : vd;
        if (take_a) va = sa[++ia];
        else vd = sd[++id];
      }
      if (kt + kMergeVT <= kn) {
        // kMergeVT consecutive outputs from a 16-byte aligned position
        uint4* dst = reinterpret_cast<uint4*>(out + (cur.k0 + kt) * E);
#pragma unroll
        for (int c = 0; c < kMergeVT * E / 16; ++c) {
          if constexpr (E == 4)
            dst[c] = make_uint4(o[4 * c], o[4 * c + 1], o[4 * c + 2], o[4 * c + 3]);
          else
            dst[c] = make_uint4((uint32_t)o[2 * c], (uint32_t)(o[2 * c] >> 32), (uint32_t)o[2 * c + 1],
                                (uint32_t)(o[2 * c + 1] >> 32));
        }
      } else {
#pragma unroll
        for (int v = 0; v < kMergeVT; ++v)
          if (kt + v < kn) store_u128<E>(out, cur.k0 + kt + v, (u128)o[v]);
      }
    }
    cur = nxt;
  }
  cp_async_wait<0>();
}

}  // namespace rfx
