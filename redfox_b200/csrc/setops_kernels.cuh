// setops_kernels.cuh -- multiset set operations on sorted arrays and unique.
//
// STL / thrust semantics (thrust::set_union / set_difference in Union.cu:47-148 and
// Difference.cu:35-143; std::set_intersection as moderngpu's benchmarksets.cu:95-125
// checks it): a value occurring m times in A and n times in B occurs min(m, n) times in
// the intersection, max(m - n, 0) times in A - B and max(m, n) times in the union.
//   * intersection / difference keep A[i] when its rank within its run of equal values
//     is below / not below the number of equal values in B -- one filtering pass with
//     stable compaction (decoupled look-back);
//   * union = merge(A, B - A) with A first on ties, by merge path (no scan needed);
//   * unique keeps the first of each run, in place.
#pragma once

#include <type_traits>

#include "search.cuh"

namespace rfx {

constexpr int kSetThreads = 256;
// Items per thread: 8 by default, 4 and 16 as the tuner's alternatives (unique always 8);
// elements up to 8 bytes live in 64-bit registers.
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
  uint32_t wcap;         // two-pass form: B window capacity (elements of dynamic shared memory)
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
constexpr int kMarkTile = kSetThreads * 8;        // the smallest tile (8 items per thread): sizing

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

}  // namespace rfx
