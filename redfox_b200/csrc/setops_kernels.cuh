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

struct SetFilterArgs {
  const uint8_t* a;
  uint64_t na;
  const uint8_t* b;
  uint64_t nb;
  const uint8_t* prev;   // KEEP_HEADS: element before each tile (saved before in-place writes)
  const uint64_t* split; // KEEP_(UN)MATCHED: per tile (run start of its first element, B window)
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

template <int E, int MODE, int IPT>
__global__ void __launch_bounds__(kSetThreads) set_filter_kernel(const SetFilterArgs p) {
  typedef typename std::conditional<(E <= 8), uint64_t, u128>::type WT;
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
      // The window of B values the tile's elements can equal, in shared memory.  A thread's
      // items are consecutive and sorted: one binary search finds the first candidate in B
      // for its first item, later items advance from there (merge order), and equal runs
      // in B are measured by galloping.  An item's rank within its run of equal values is
      // its distance from the run's first item: the last head (first item of a run) at or
      // before it, from a block max-scan of the threads' last heads, or -- for the run that
      // continues from the previous tile -- the run start found by set_split_kernel.
      const uint64_t tfirst = tile * TILE;
      if (t == 0) s_rs0 = p.split[3 * tile];
      if (t == 1) s_blo = p.split[3 * tile + 1];
      if (t == 2) s_bhi = p.split[3 * tile + 2];
      __syncthreads();
      const uint64_t blo0 = s_blo, bn = s_bhi > s_blo ? s_bhi - s_blo : 0;
      const bool staged = bn <= (uint64_t)WCAP;
      if (staged)
        for (uint64_t x = t; x < bn; x += kSetThreads) s_b[x] = (WT)B.key(blo0 + x);
      // heads of this thread's items (local index of its last head, or -1)
      int32_t last_head = -1;
      uint32_t heads = 0;
      WT prev = 0;
      if (first < p.na && first > tfirst) prev = (WT)A.key(first - 1);
#pragma unroll
      for (int j = 0; j < IPT; ++j) {
        const uint64_t i = first + j;
        if (i >= p.na) continue;
        const bool h = i == 0 || (i > tfirst && v[j] != (j == 0 ? prev : v[j - 1]));
        if (h) {
          heads |= 1u << j;
          last_head = (int32_t)(i - tfirst);
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
      uint64_t run_start = before >= 0 ? tfirst + (uint64_t)before : s_rs0;
      // first candidate in B for the first item
      uint64_t pos = 0;
      if (first < p.na) {
        pos = staged ? (uint64_t)smem_lower(s_b, (uint32_t)bn, v[0]) : bsearch<E>(B, v[0], 0, p.nb, false);
      }
#pragma unroll
      for (int j = 0; j < IPT; ++j) {
        const uint64_t i = first + j;
        if (i >= p.na) continue;
        if ((heads >> j) & 1u) run_start = i;
        uint64_t nbeq;
        if (staged) {
          while (pos < bn && s_b[pos] < v[j]) ++pos;
          nbeq = 0;
          if (pos < bn && s_b[pos] == v[j]) {
            if (pos + 1 >= bn || s_b[pos + 1] != v[j]) nbeq = 1;
            else nbeq = smem_lower_strict(s_b + pos, (uint32_t)(bn - pos), v[j]);
          }
        } else {
          pos = j == 0 ? pos : (gallop<E>(B, v[j], pos, false));
          nbeq = gallop<E>(B, v[j], pos, true) - pos;
        }
        const uint64_t rank = i - run_start;
        keep[j] = MODE == KEEP_MATCHED ? rank < nbeq : rank >= nbeq;
      }
      __syncthreads();
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

// Merge of A and D (A first on ties): the union.
template <int E>
__global__ void __launch_bounds__(kSetThreads)
merge_kernel(const uint8_t* a, uint64_t na, const uint8_t* d, uint64_t nd_max, const uint64_t* d_nd, uint8_t* out,
             uint64_t* d_count) {
  const uint64_t nd = d_nd ? min(nd_max, *d_nd) : nd_max;
  const uint64_t total = na + nd;
  if (blockIdx.x == 0 && threadIdx.x == 0) *d_count = total;
  const KeyView<E> A{a, na, 0};
  const KeyView<E> D{d, nd, 0};
  const uint64_t stride = (uint64_t)gridDim.x * kMergeTile;
  for (uint64_t k0 = (uint64_t)blockIdx.x * kMergeTile + (uint64_t)threadIdx.x * kMergeVT; k0 < total; k0 += stride) {
    // merge path: i = number of A elements among the first k0 outputs
    uint64_t lo = k0 > nd ? k0 - nd : 0, hi = k0 < na ? k0 : na;
    while (lo < hi) {
      const uint64_t mid = lo + ((hi - lo) >> 1);
      if (A.key(mid) <= D.key(k0 - mid - 1)) lo = mid + 1;
      else hi = mid;
    }
    uint64_t i = lo, j = k0 - lo;
#pragma unroll
    for (int v = 0; v < kMergeVT; ++v) {
      const uint64_t k = k0 + v;
      if (k >= total) break;
      const bool take_a = j >= nd || (i < na && A.key(i) <= D.key(j));
      if (take_a) store_u128<E>(out, k, A.key(i++));
      else store_u128<E>(out, k, D.key(j++));
    }
  }
}

}  // namespace rfx
