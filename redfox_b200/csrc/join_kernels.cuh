// join_kernels.cuh -- sort-merge join: find_bounds (lower bound + equality count + scan
// in one pass), load-balanced expansion into (left, right) index pairs, the gather that
// assembles output tuples, and the fused tuple join that expands and assembles without
// materialising indices.
//
// Output order is the reference's: left row ascending, then right row ascending
// (KernelLeftJoin<Tuning, false>, ModernGPUJoin.cu:665-733; CPUJoin,
// moderngpu/tests/benchmarkjoin.cu:40-128).  Expansion is balanced over output rows, so a
// skewed key (one left row with millions of matches) spreads over all blocks.
#pragma once

#include <type_traits>

#include "search.cuh"
#include "sort_kernels.cuh"
#include "tile_ring.cuh"

namespace rfx {

constexpr int kJoinThreads = 256;
constexpr int kFbIPT = 4;                        // left rows per thread in find_bounds
constexpr int kFbTile = kJoinThreads * kFbIPT;
constexpr int kExpVT = 8;                        // outputs per thread in the expansion
constexpr int kExpTile = kJoinThreads * kExpVT;

struct FindBoundsArgs {
  const uint8_t* left;
  uint64_t nl;
  const uint8_t* right;
  uint64_t nr;
  uint32_t lshift, rshift;   // key = container >> shift
  uint32_t window_bytes;     // dynamic shared memory of the launch (the window)
  int32_t* lb32;             // reference outputs (may be null)
  int32_t* scan32;
  uint64_t* lb64;            // workspace outputs for the fused join (may be null)
  uint64_t* off64;           // exclusive offsets, off64[nl] = total
  uint64_t* tile_owner;      // fused join: per output tile of kExpTile rows, the left row
  uint64_t n_owner;          // that owns its first output (tiles >= n_owner are not recorded)
  uint64_t* d_total;
  uint64_t* status;
  uint32_t* tile_counter;
  uint32_t* err;
  // join-aggregate mode: the left side is a table of groups (one row per distinct key,
  // with its SUM and COUNT); a group is kept when its key occurs on the right, with its
  // SUM and COUNT multiplied by the number of right rows that carry the key
  const uint64_t* d_nl;      // device-resident left size (<= nl), or null
  const int64_t* gsum;
  const uint32_t* gcnt;
  uint8_t* okey;             // kept keys, LE bytes each
  int64_t* osum;
  uint32_t* ocnt;
};

// Block-wide exclusive sum of one 64-bit value per thread.
__device__ __forceinline__ uint64_t block_exclusive_u64(uint64_t x, uint64_t* s_warp, uint64_t* total) {
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (uint32_t)o) incl += y;
  }
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  uint64_t wpre = 0, tot = 0;
  for (uint32_t w = 0; w < blockDim.x / 32; ++w) {
    if (w < warp) wpre += s_warp[w];
    tot += s_warp[w];
  }
  *total = tot;
  return wpre + incl - x;
}

// Right-side keys a block's left keys can match, staged in dynamic shared memory of
// FindBoundsArgs::window_bytes (at most kFbWindowBytes): u32 keys when the right
// container has at most 4 bytes (or, for the join-aggregate, its key (container >> shift)
// at most 32 bits), u64 when the key has at most 64 bits, u128 otherwise.  A window that
// does not fit falls back to searches in global memory.
constexpr uint32_t kFbWindowBytes = 64 * 1024;

// First index in [lo, n) of the sorted window with w[i] >= k (strict: > k).
template <bool STRICT, typename T>
__device__ __forceinline__ uint32_t smem_bound_t(const T* w, uint32_t lo, uint32_t n, T k) {
  uint32_t hi = n;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    const T m = w[mid];
    if (STRICT ? (m <= k) : (m < k)) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// The same bound found by galloping forward from `from` (every w[i] with i < from lies
// before k): cheap when consecutive sorted keys land close together.
template <bool STRICT, typename T>
__device__ __forceinline__ uint32_t smem_gallop_t(const T* w, uint32_t from, uint32_t n, T k) {
  uint32_t lo = from, hi = from, step = 1;
  while (hi < n && (STRICT ? (w[hi] <= k) : (w[hi] < k))) {
    lo = hi + 1;
    hi = lo + step;
    step <<= 1;
  }
  return smem_bound_t<STRICT>(w, lo, hi < n ? hi : n, k);
}

// GROUP = false: find_bounds (lower bounds, equality counts, their exclusive scan, total).
// GROUP = true: the join-aggregate (see FindBoundsArgs): the block scan counts kept groups
// instead of matches and *d_total receives the number of kept groups.
template <int LE, int RE, bool GROUP = false>
__global__ void __launch_bounds__(kJoinThreads) find_bounds_kernel(const FindBoundsArgs a) {
  extern __shared__ __align__(16) uint8_t fb_window[];
  // the narrow window type; keys above its range lie above the whole window
  using W = std::conditional_t<(RE <= 4), uint32_t, uint64_t>;
  W* s_win = reinterpret_cast<W*>(fb_window);
  u128* s_win128 = reinterpret_cast<u128*>(fb_window);
  uint32_t* s_win32 = reinterpret_cast<uint32_t*>(fb_window);
  const bool narrow = RE <= 4 || (uint32_t)RE * 8u - a.rshift <= 64u;
  // the join-aggregate's wider containers whose key (container >> shift) has at most 32
  // bits: a u32 window, twice the keys in the same shared memory (its window is the
  // largest one, sized without the group count; the plain find_bounds sizes its window
  // from the two sides' lengths and keeps the wider type, which measured faster there)
  const bool n32 = GROUP && RE > 4 && (uint32_t)RE * 8u - a.rshift <= 32u;
  const uint64_t WB = a.window_bytes;
  __shared__ uint64_t s_warp[kJoinThreads / 32];
  __shared__ uint64_t s_prefix;
  __shared__ uint32_t s_tile;
  __shared__ uint64_t s_lo, s_hi;
  const uint32_t t = threadIdx.x;
  const uint64_t nl = a.d_nl ? min(a.nl, *a.d_nl) : a.nl;
  const uint64_t num_tiles = (nl + kFbTile - 1) / kFbTile;
  const KeyView<LE> L{a.left, nl, a.lshift};
  const KeyView<RE> R{a.right, a.nr, a.rshift};
  // a tile is claimed when the block is ready for it (claiming one ahead measured slower:
  // a claimed tile's successors wait in their look-back until its block gets to it)
  while (true) {
    __syncthreads();
    if (t == 0) s_tile = atomicAdd(a.tile_counter, 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    if (tile >= num_tiles) break;
    const uint64_t tfirst = tile * kFbTile;
    const uint64_t tlast = min(tfirst + kFbTile, nl) - 1;
    // the window of right keys between the tile's smallest and largest left key
    if (t < 32) {
      const uint64_t lo = warp_search<RE>(R, L.key(tfirst), 0, a.nr, false);
      if (t == 0) s_lo = lo;
    } else if (t < 64) {
      const uint64_t hi = warp_search<RE>(R, L.key(tlast), 0, a.nr, true);
      if (t == 32) s_hi = hi;
    }
    __syncthreads();
    const uint64_t wlo = s_lo, wn = s_hi > s_lo ? s_hi - s_lo : 0;
    const bool staged = wn * (n32 ? 4u : narrow ? sizeof(W) : 16u) <= WB;
    // a few loads in flight per thread while staging (one round trip per key otherwise)
    if (staged && n32)
      block_stage<8>(wn, t, kJoinThreads, [&](uint64_t x) { return (uint32_t)R.key(wlo + x); },
                     [&](uint64_t x, uint32_t v) { s_win32[x] = v; });
    else if (staged && narrow)
      block_stage<(sizeof(W) == 4 ? 8 : 4)>(wn, t, kJoinThreads, [&](uint64_t x) { return (W)R.key(wlo + x); },
                                             [&](uint64_t x, W v) { s_win[x] = v; });
    else if (staged)
      block_stage<2>(wn, t, kJoinThreads, [&](uint64_t x) { return R.key(wlo + x); },
                     [&](uint64_t x, u128 v) { s_win128[x] = v; });
    __syncthreads();
    const uint64_t first = tfirst + (uint64_t)t * kFbIPT;
    uint64_t lo[kFbIPT], cnt[kFbIPT];
    uint64_t tsum = 0;
    u128 prevk = 0;
    uint64_t plo = 0, phi = 0;
    // the thread's keys first, all loads in flight together (the searches below branch on
    // them, which would otherwise serialise the loads)
    u128 keys[kFbIPT];
#pragma unroll
    for (int j = 0; j < kFbIPT; ++j) keys[j] = first + j < nl ? L.key(first + j) : (u128)0;
#pragma unroll
    for (int j = 0; j < kFbIPT; ++j) {
      const uint64_t i = first + j;
      lo[j] = 0;
      cnt[j] = 0;
      if (i >= nl) continue;
      const u128 k = keys[j];
      if (j > 0 && k == prevk) {
        lo[j] = plo;
        cnt[j] = phi - plo;
      } else {
        uint64_t l, h;
        // the thread's keys ascend: the first is searched in the whole window, the next
        // ones gallop forward from the previous key's upper bound
        const uint32_t from = j == 0 ? 0u : (uint32_t)(phi - wlo);
        if (staged && n32) {
          if ((k >> 32) != 0) {
            l = h = wlo + wn;
          } else {
            const uint32_t lw = j == 0 ? smem_bound_t<false>(s_win32, 0u, (uint32_t)wn, (uint32_t)k)
                                       : smem_gallop_t<false>(s_win32, from, (uint32_t)wn, (uint32_t)k);
            l = wlo + lw;
            h = wlo + smem_gallop_t<true>(s_win32, lw, (uint32_t)wn, (uint32_t)k);
          }
        } else if (staged && narrow) {
          // compares in the window's type (a larger left key lies above the whole window)
          if ((k >> (8 * sizeof(W))) != 0) {
            l = h = wlo + wn;
          } else {
            const uint32_t lw = j == 0 ? smem_bound_t<false>(s_win, 0u, (uint32_t)wn, (W)k)
                                       : smem_gallop_t<false>(s_win, from, (uint32_t)wn, (W)k);
            l = wlo + lw;
            h = wlo + smem_gallop_t<true>(s_win, lw, (uint32_t)wn, (W)k);
          }
        } else if (staged) {
          const uint32_t lw = j == 0 ? smem_bound_t<false>(s_win128, 0u, (uint32_t)wn, k)
                                     : smem_gallop_t<false>(s_win128, from, (uint32_t)wn, k);
          l = wlo + lw;
          h = wlo + smem_gallop_t<true>(s_win128, lw, (uint32_t)wn, k);
        } else {
          l = j == 0 ? bsearch<RE>(R, k, 0, a.nr, false) : gallop<RE>(R, k, phi, false);
          h = gallop<RE>(R, k, l, true);
        }
        lo[j] = l;
        cnt[j] = h - l;
        plo = l;
        phi = h;
        prevk = k;
      }
      tsum += GROUP ? (cnt[j] != 0) : cnt[j];
    }
    uint64_t btot;
    const uint64_t ex = block_exclusive_u64(tsum, s_warp, &btot);
    if ((t >> 5) == 0) {
      const uint64_t pre = lookback_exclusive(a.status, (uint32_t)tile, btot, a.err);
      if (t == 0) {
        s_prefix = pre;
        if (tile == num_tiles - 1) {
          *a.d_total = pre + btot;
          if (a.off64) a.off64[nl] = pre + btot;
        }
      }
    }
    __syncthreads();
    uint64_t run = s_prefix + ex;
    if constexpr (GROUP) {
      // kept groups in left order; products wrap like the sums of the join rows would
#pragma unroll
      for (int j = 0; j < kFbIPT; ++j) {
        const uint64_t i = first + j;
        if (i >= nl || cnt[j] == 0) continue;
        store_u128<LE>(a.okey, run, load_u128<LE>(a.left, i));
        a.osum[run] = (int64_t)((uint64_t)a.gsum[i] * cnt[j]);
        a.ocnt[run] = a.gcnt[i] * (uint32_t)cnt[j];
        ++run;
      }
      continue;
    }
#pragma unroll
    for (int j = 0; j < kFbIPT; ++j) {
      const uint64_t i = first + j;
      if (i >= nl) continue;
      if (a.tile_owner && cnt[j]) {
        // every output tile that starts inside this row's outputs [run, run + cnt) is owned
        // by it at its first output
        for (uint64_t b = (run + kExpTile - 1) / kExpTile; b < a.n_owner && b * kExpTile < run + cnt[j]; ++b)
          a.tile_owner[b] = i;
      }
      if (a.lb32) a.lb32[i] = (int32_t)lo[j];
      if (a.scan32) a.scan32[i] = (int32_t)(uint32_t)run;
      if (a.lb64) a.lb64[i] = lo[j];
      if (a.off64) a.off64[i] = run;
      run += cnt[j];
    }
  }
  if (nl == 0 && blockIdx.x == 0 && t == 0) {
    *a.d_total = 0;
    if (a.off64) a.off64[0] = 0;
  }
}

// ------------------------------------------------------------------ index expansion
// Output k belongs to the last left row i with scan[i] <= k; right row lb[i] + k - scan[i].
// A block stages the scan entries covering its outputs in shared memory.
constexpr int kExpCap = 2048 + 1;

__device__ __forceinline__ uint64_t owner_scan(const int32_t* scan, uint64_t n, uint64_t k) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t mid = lo + ((hi - lo) >> 1);
    if ((uint64_t)(uint32_t)__ldg(scan + mid) <= k) lo = mid + 1;
    else hi = mid;
  }
  return lo - 1;
}

// owner_scan found by one warp in ~log32(nl) rounds (all lanes return it).
__device__ __forceinline__ uint64_t owner_scan_warp(const int32_t* scan, uint64_t n, uint64_t k) {
  const uint32_t lane = threadIdx.x & 31;
  uint64_t lo = 0, hi = n;   // the first index with scan > k lies in [lo, hi]
  while (hi - lo > 32) {
    const uint64_t step = (hi - lo + 31) / 32;
    const uint64_t p = lo + lane * step;
    const bool le = p < hi && (uint64_t)(uint32_t)__ldg(scan + p) <= k;
    const uint32_t cnt = __popc(__ballot_sync(0xffffffffu, le));
    if (cnt == 0) return lo - 1;   // lo > 0 here: scan[lo - 1] <= k held on entry
    const uint64_t nlo = lo + (uint64_t)(cnt - 1) * step + 1;
    const uint64_t nhi = cnt < 32 ? min(hi, lo + (uint64_t)cnt * step) : hi;
    lo = nlo;
    hi = nhi;
  }
  const bool le = lo + lane < hi && (uint64_t)(uint32_t)__ldg(scan + lo + lane) <= k;
  return lo + __popc(__ballot_sync(0xffffffffu, le)) - 1;
}

__global__ void __launch_bounds__(kJoinThreads)
join_expand_kernel(int32_t* __restrict__ li, int32_t* __restrict__ ri, uint64_t nout_max, const uint64_t* d_nout,
                   const int32_t* __restrict__ lb, const int32_t* __restrict__ scan, uint64_t nl) {
  __shared__ uint32_t s_scan[kExpCap];
  __shared__ int32_t s_lb[kExpCap];
  __shared__ uint64_t s_i0, s_i1;
  const uint32_t t = threadIdx.x;
  uint64_t nout = nout_max;
  if (d_nout) nout = min(nout, *d_nout);
  for (uint64_t k0 = (uint64_t)blockIdx.x * kExpTile; k0 < nout; k0 += (uint64_t)gridDim.x * kExpTile) {
    const uint64_t k1 = min(k0 + (uint64_t)kExpTile, nout);
    if (t < 32) {
      const uint64_t i0 = owner_scan_warp(scan, nl, k0);
      if (t == 0) s_i0 = i0;
    } else if (t < 64) {
      const uint64_t i1 = owner_scan_warp(scan, nl, k1 - 1);
      if (t == 32) s_i1 = i1;
    }
    __syncthreads();
    const uint64_t i0 = s_i0, span = s_i1 - i0 + 1;
    const bool staged = span <= (uint64_t)kExpCap;
    if (staged)
      block_stage<8>(span, t, kJoinThreads,
                     [&](uint64_t x) { return make_int2(__ldg(scan + i0 + x), __ldg(lb + i0 + x)); },
                     [&](uint64_t x, int2 v) {
                       s_scan[x] = (uint32_t)v.x;
                       s_lb[x] = v.y;
                     });
    __syncthreads();
    for (int v = 0; v < kExpVT; ++v) {
      const uint64_t k = k0 + (uint64_t)v * kJoinThreads + t;
      if (k >= k1) break;
      uint64_t i;
      uint32_t sc;
      int32_t l;
      if (staged) {
        uint32_t lo = 0, hi = (uint32_t)span;
        while (lo < hi) {
          const uint32_t mid = (lo + hi) >> 1;
          if (s_scan[mid] <= k) lo = mid + 1;
          else hi = mid;
        }
        i = i0 + lo - 1;
        sc = s_scan[lo - 1];
        l = s_lb[lo - 1];
      } else {
        i = owner_scan(scan, nl, k);
        sc = (uint32_t)__ldg(scan + i);
        l = __ldg(lb + i);
      }
      li[k] = (int32_t)i;
      ri[k] = l + (int32_t)(k - (uint64_t)sc);
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ gather
// out = lkey << (lv_bits + rv_bits) | lval << rv_bits | rval over containers of up to
// 64 bytes (gather_{key_key,key_value,value_key,value_value}, ModernGPUJoin.h:43-200).
struct GatherArgs {
  uint8_t* out;
  uint32_t ob;
  uint64_t nout_max;
  const uint64_t* d_nout;
  const int32_t* li;
  const int32_t* ri;
  const uint8_t* lkey;
  uint32_t lkb;
  const uint8_t* lval;
  uint32_t lvb;
  uint32_t lv_bits;
  const uint8_t* rval;
  uint32_t rvb;
  uint32_t rv_bits;
};

__device__ __forceinline__ void limb_load(uint64_t (&L)[8], const uint8_t* p, uint32_t bytes) {
#pragma unroll
  for (int k = 0; k < 8; ++k) L[k] = 0;
  if (bytes >= 8) {
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if ((uint32_t)k * 8 < bytes) L[k] = reinterpret_cast<const unsigned long long*>(p)[k];
  } else if (bytes == 4) {
    L[0] = *reinterpret_cast<const uint32_t*>(p);
  } else if (bytes == 2) {
    L[0] = *reinterpret_cast<const uint16_t*>(p);
  } else {
    L[0] = *p;
  }
}

__device__ __forceinline__ void limb_shl_or(uint64_t (&acc)[8], const uint64_t (&v)[8], uint32_t s) {
  const uint32_t q = s >> 6, r = s & 63;
#pragma unroll
  for (int k = 7; k >= 0; --k) {
    const int src = k - (int)q;
    if (src < 0) continue;
    uint64_t x = v[src] << r;
    if (r && src > 0) x |= v[src - 1] >> (64 - r);
    acc[k] |= x;
  }
}

__global__ void __launch_bounds__(kJoinThreads) join_gather_kernel(const GatherArgs a) {
  uint64_t nout = a.nout_max;
  if (a.d_nout) nout = min(nout, *a.d_nout);
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nout; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = (uint32_t)a.li[k];
    uint64_t acc[8] = {0, 0, 0, 0, 0, 0, 0, 0}, v[8];
    limb_load(v, a.lkey + i * a.lkb, a.lkb);
    limb_shl_or(acc, v, a.lv_bits + a.rv_bits);
    if (a.lval) {
      limb_load(v, a.lval + i * a.lvb, a.lvb);
      limb_shl_or(acc, v, a.rv_bits);
    }
    if (a.rval) {
      const uint64_t j = (uint32_t)a.ri[k];
      limb_load(v, a.rval + j * a.rvb, a.rvb);
      limb_shl_or(acc, v, 0);
    }
    uint8_t* o = a.out + k * a.ob;
    if (a.ob >= 8) {
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if ((uint32_t)q * 8 < a.ob) reinterpret_cast<unsigned long long*>(o)[q] = acc[q];
    } else if (a.ob == 4) {
      *reinterpret_cast<uint32_t*>(o) = (uint32_t)acc[0];
    } else if (a.ob == 2) {
      *reinterpret_cast<uint16_t*>(o) = (uint16_t)acc[0];
    } else {
      *o = (uint8_t)acc[0];
    }
  }
}

// ------------------------------------------------------------------ fused tuple join
// out[k] = (L[i] << rv_bits) | (R[j] & mask(rv_bits)) -- combine<> of Tuple.h:942-955, the
// same bytes as gather_value_value on the split key/value arrays -- for the k < cap
// output rows, i and j found from the find_bounds offsets.
struct TupleJoinArgs {
  const uint8_t* left;
  uint64_t nl;
  const uint8_t* right;
  uint64_t nr;
  uint32_t rv_bits;
  const uint64_t* lb64;
  const uint64_t* off64;   // nl + 1 entries
  uint8_t* out;
  uint64_t cap;
  const uint64_t* tile_owner;   // from the count pass (may be null)
  uint64_t n_owner;
  uint32_t* err;
};

// Offsets of the left rows that cover a block's outputs, staged in shared memory.
constexpr int kStageCap = kExpTile + 1;

// Last index i in [0, n) with off[i] <= k (off non-decreasing, off[0] = 0).
__device__ __forceinline__ uint64_t owner_global(const uint64_t* off, uint64_t n, uint64_t k) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t mid = lo + ((hi - lo) >> 1);
    if (__ldg(off + mid) <= k) lo = mid + 1;
    else hi = mid;
  }
  return lo - 1;
}

// The same index found by one warp in ~log32(n) rounds of 32 loads in flight each
// (instead of ~log2(n) dependent loads); all lanes return it.
__device__ __forceinline__ uint64_t owner_warp(const uint64_t* off, uint64_t n, uint64_t k) {
  const uint32_t lane = threadIdx.x & 31;
  uint64_t lo = 0, hi = n;   // the first index with off > k lies in [lo, hi]
  while (hi - lo > 32) {
    const uint64_t step = (hi - lo + 31) / 32;
    const uint64_t p = lo + lane * step;
    const bool le = p < hi && __ldg(off + p) <= k;
    const uint32_t cnt = __popc(__ballot_sync(0xffffffffu, le));
    if (cnt == 0) return lo - 1;   // lo > 0 here: off[lo - 1] <= k held on entry to this round
    const uint64_t nlo = lo + (uint64_t)(cnt - 1) * step + 1;
    const uint64_t nhi = cnt < 32 ? min(hi, lo + (uint64_t)cnt * step) : hi;
    lo = nlo;
    hi = nhi;
  }
  const bool le = lo + lane < hi && __ldg(off + lo + lane) <= k;
  return lo + __popc(__ballot_sync(0xffffffffu, le)) - 1;
}

template <int LE, int RE, int OE>
__global__ void __launch_bounds__(kJoinThreads) tuple_join_kernel(const TupleJoinArgs a) {
  __shared__ uint64_t s_off[kStageCap + 1];
  __shared__ uint64_t s_lb[kStageCap];
  __shared__ uint32_t s_own[kExpTile];      // staged row owning each output of the tile
  __shared__ uint32_t s_wmax[kJoinThreads / 32];
  __shared__ uint64_t s_i0, s_i1;
  const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const uint64_t total = a.off64[a.nl];
  const uint64_t nout = total < a.cap ? total : a.cap;
  const u128 rmask = a.rv_bits >= 128 ? ~(u128)0 : (((u128)1 << a.rv_bits) - 1);
  for (uint64_t k0 = (uint64_t)blockIdx.x * kExpTile; k0 < nout; k0 += (uint64_t)gridDim.x * kExpTile) {
    const uint64_t k1 = min(k0 + (uint64_t)kExpTile, nout);
    if (t < 32) {
      const uint64_t i0 = owner_warp(a.off64, a.nl, k0);
      if (t == 0) s_i0 = i0;
    } else if (t < 64) {
      const uint64_t i1 = owner_warp(a.off64, a.nl, k1 - 1);
      if (t == 32) s_i1 = i1;
    }
    __syncthreads();
    const uint64_t i0 = s_i0, span = s_i1 - i0 + 1;
    const bool staged = span <= (uint64_t)kStageCap;
    if (staged) {
      block_stage<4>(span + 1, t, kJoinThreads,
                     [&](uint64_t x) { return make_ulonglong2(__ldg(a.off64 + i0 + x),
                                                              x < span ? __ldg(a.lb64 + i0 + x) : 0ull); },
                     [&](uint64_t x, ulonglong2 v) {
                       s_off[x] = v.x;
                       if (x < span) s_lb[x] = v.y;
                     });
      for (uint32_t x = t; x < (uint32_t)kExpTile; x += kJoinThreads) s_own[x] = 0;
    }
    __syncthreads();
    if (staged) {
      // each staged row with outputs marks its first output in the tile (row 0 owns the
      // tile's start); an inclusive max-scan then gives every output its row (the
      // load-balancing search of a merge-path join, without a search per output)
      for (uint64_t x = 1 + t; x < span; x += kJoinThreads)
        if (s_off[x] < k1 && s_off[x + 1] > s_off[x]) s_own[s_off[x] - k0] = (uint32_t)x;
      __syncthreads();
      constexpr uint32_t PER = kExpTile / kJoinThreads;
      uint32_t m = 0, v[PER];
#pragma unroll
      for (uint32_t j = 0; j < PER; ++j) {
        m = max(m, s_own[t * PER + j]);
        v[j] = m;
      }
      uint32_t inc = m;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= (uint32_t)o) inc = max(inc, y);
      }
      if (lane == 31) s_wmax[warp] = inc;
      uint32_t ex = __shfl_up_sync(0xffffffffu, inc, 1);
      if (lane == 0) ex = 0;
      __syncthreads();
      for (uint32_t w = 0; w < warp; ++w) ex = max(ex, s_wmax[w]);
#pragma unroll
      for (uint32_t j = 0; j < PER; ++j) s_own[t * PER + j] = max(v[j], ex);
    }
    __syncthreads();
    // outputs striped over the block: consecutive threads write consecutive rows
#pragma unroll 2
    for (int v = 0; v < kExpVT; ++v) {
      const uint64_t k = k0 + (uint64_t)v * kJoinThreads + t;
      if (k >= k1) break;
      uint64_t i, offi, lbi;
      if (staged) {
        const uint32_t x = s_own[k - k0];
        i = i0 + x;
        offi = s_off[x];
        lbi = s_lb[x];
      } else {
        i = owner_global(a.off64, a.nl, k);
        offi = __ldg(a.off64 + i);
        lbi = __ldg(a.lb64 + i);
      }
      const uint64_t j = lbi + (k - offi);
      if (j < a.nr)  // guards a timed-out scan
        store_u128<OE>(a.out, k, (load_u128<LE>(a.left, i) << a.rv_bits) | (load_u128<RE>(a.right, j) & rmask));
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ staged emit
// The emit with every operand of a tile in shared memory.  Per tile of kExpTile outputs:
// the owners of its first and last output come from the count pass (tile_owner), the
// offsets and lower bounds of the left rows in between are staged, each output finds its
// row by the mark + max-scan, and the tile's left rows and the window of right rows it
// touches (rows [jlo, jhi) of the right relation: right runs of equal keys are revisited
// by every left row with that key) are brought into shared memory by bulk copies
// (cp.async.bulk, this GPU's memory; an mbarrier counts the bytes; a range that is not
// 16-byte aligned or would read past the array is copied by the threads instead).  The
// outputs are then assembled from shared memory and stored in order, so the tile's
// global traffic is its output rows plus one pass over its input windows.
constexpr int kJsSpan = 1024;              // left rows staged per tile
constexpr int kJsLeftBytes = kJsSpan * 16;
constexpr int kJsRightBytes = 16384;       // right window staged per tile

struct JsLayout {
  static constexpr size_t OFF = 0;                                        // u64[kJsSpan + 1]
  static constexpr size_t LB = OFF + 8 * (kJsSpan + 1);                   // u64[kJsSpan]
  static constexpr size_t OWN = LB + 8 * kJsSpan;                         // u16[kExpTile]
  static constexpr size_t LEFT = (OWN + 2 * kExpTile + 127) / 128 * 128;  // left rows (+16 slack)
  static constexpr size_t RIGHT = LEFT + kJsLeftBytes + 128;              // right window (+16 slack)
  static constexpr size_t BYTES = RIGHT + kJsRightBytes + 128;
};

template <int E>
__device__ __forceinline__ u128 smem_row(const uint8_t* p) {
  if constexpr (E == 4) return (u128)*reinterpret_cast<const uint32_t*>(p);
  else if constexpr (E == 8) return (u128)*reinterpret_cast<const unsigned long long*>(p);
  else {
    const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(p);
    return ((u128)v.y << 64) | (u128)v.x;
  }
}

// Stages bytes [b0, b1) of `src` (an array of `limit` bytes) into `dst`: returns the first
// byte copied (16-byte aligned) when one bulk copy was issued on `bar` (*tx += its bytes),
// or copies with all threads when `bulk` is false.  Called by thread 0 (bulk) or by all
// threads (plain) -- see the caller.
__device__ __forceinline__ uint64_t js_align_lo(uint64_t b0) { return b0 & ~15ull; }
__device__ __forceinline__ uint64_t js_align_hi(uint64_t b1) { return (b1 + 15) & ~15ull; }

template <int LE, int RE, int OE>
__global__ void __launch_bounds__(kJoinThreads) tuple_join_staged_kernel(const TupleJoinArgs a) {
  extern __shared__ __align__(128) uint8_t js[];
  uint64_t* s_off = reinterpret_cast<uint64_t*>(js + JsLayout::OFF);
  uint64_t* s_lb = reinterpret_cast<uint64_t*>(js + JsLayout::LB);
  uint16_t* s_own = reinterpret_cast<uint16_t*>(js + JsLayout::OWN);
  uint8_t* s_left = js + JsLayout::LEFT;
  uint8_t* s_right = js + JsLayout::RIGHT;
  __shared__ uint64_t s_i0, s_i1, s_lbase, s_rbase;
  __shared__ unsigned long long s_jlo, s_jhi;
  __shared__ uint32_t s_mode;          // bit 0 left staged, 1 right staged, 2 bulk copies issued
  __shared__ uint32_t s_wmax[kJoinThreads / 32];
  __shared__ __align__(8) uint64_t s_bar;
  const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const uint64_t total = a.off64[a.nl];
  const uint64_t nout = total < a.cap ? total : a.cap;
  const u128 rmask = a.rv_bits >= 128 ? ~(u128)0 : (((u128)1 << a.rv_bits) - 1);
  const bool bulk_ok = ((reinterpret_cast<uintptr_t>(a.left) | reinterpret_cast<uintptr_t>(a.right)) & 15u) == 0;
  if (t == 0) {
    mbar_init(&s_bar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  uint32_t phase = 0;
  for (uint64_t k0 = (uint64_t)blockIdx.x * kExpTile; k0 < nout; k0 += (uint64_t)gridDim.x * kExpTile) {
    const uint64_t tile = k0 / kExpTile;
    const uint64_t k1 = min(k0 + (uint64_t)kExpTile, nout);
    // owners of the first and last output
    const bool rec0 = a.tile_owner && tile < a.n_owner;
    const bool rec1 = a.tile_owner && tile + 1 < a.n_owner && k1 < total;
    if (t < 32) {
      const uint64_t i0 = rec0 ? __ldg(a.tile_owner + tile) : owner_warp(a.off64, a.nl, k0);
      if (t == 0) s_i0 = i0;
    } else if (t < 64) {
      const uint64_t i1 = rec1 ? __ldg(a.tile_owner + tile + 1) : owner_warp(a.off64, a.nl, k1 - 1);
      if (t == 32) s_i1 = i1;
    }
    if (t == 64) {
      s_jlo = ~0ull;
      s_jhi = 0;
    }
    __syncthreads();
    const uint64_t i0 = s_i0, span = s_i1 - i0 + 1;
    if (span > (uint64_t)kJsSpan) {
      // more left rows than the stage holds (rows with very few outputs): search per output
#pragma unroll 2
      for (int v = 0; v < kExpVT; ++v) {
        const uint64_t k = k0 + (uint64_t)v * kJoinThreads + t;
        if (k >= k1) break;
        const uint64_t i = owner_global(a.off64, a.nl, k);
        const uint64_t j = __ldg(a.lb64 + i) + (k - __ldg(a.off64 + i));
        if (j < a.nr)
          store_u128<OE>(a.out, k, (load_u128<LE>(a.left, i) << a.rv_bits) | (load_u128<RE>(a.right, j) & rmask));
      }
      __syncthreads();
      continue;
    }
    block_stage<4>(span + 1, t, kJoinThreads,
                   [&](uint64_t x) { return make_ulonglong2(__ldg(a.off64 + i0 + x),
                                                            x < span ? __ldg(a.lb64 + i0 + x) : 0ull); },
                   [&](uint64_t x, ulonglong2 v) {
                     s_off[x] = v.x;
                     if (x < span) s_lb[x] = v.y;
                   });
    for (uint32_t x = t; x < (uint32_t)kExpTile; x += kJoinThreads) s_own[x] = 0;
    __syncthreads();
    // marks (each row's first output in the tile) and the right rows the tile touches
    {
      unsigned long long jlo = ~0ull, jhi = 0;
      for (uint32_t x = t; x < (uint32_t)span; x += kJoinThreads) {
        const uint64_t o0 = s_off[x], o1 = s_off[x + 1];
        const uint64_t a0 = o0 > k0 ? o0 : k0, a1 = o1 < k1 ? o1 : k1;
        if (a0 >= a1) continue;
        if (x > 0) s_own[a0 - k0] = (uint16_t)x;
        jlo = min(jlo, (unsigned long long)(s_lb[x] + (a0 - o0)));
        jhi = max(jhi, (unsigned long long)(s_lb[x] + (a1 - o0)));
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        jlo = min(jlo, __shfl_xor_sync(0xffffffffu, jlo, o));
        jhi = max(jhi, __shfl_xor_sync(0xffffffffu, jhi, o));
      }
      if (lane == 0) {
        atomicMin(&s_jlo, jlo);
        atomicMax(&s_jhi, jhi);
      }
    }
    __syncthreads();
    // stage the left rows [i0, i0 + span) and the right window [jlo, jhi)
    if (t == 0) {
      uint32_t mode = 0, tx = 0;
      const uint64_t lb0 = js_align_lo(i0 * LE), lb1 = js_align_hi((i0 + span) * LE);
      const uint64_t jlo = s_jlo, jhi = s_jhi > a.nr ? a.nr : s_jhi;
      const uint64_t rb0 = js_align_lo(jlo * RE), rb1 = js_align_hi(jhi * RE);
      if (lb1 - lb0 <= (uint64_t)kJsLeftBytes + 16) mode |= 1;
      if (jlo < jhi && rb1 - rb0 <= (uint64_t)kJsRightBytes + 16) mode |= 2;
      s_lbase = lb0;
      s_rbase = rb0;
      const bool lbulk = (mode & 1) && bulk_ok && lb1 <= a.nl * LE;
      const bool rbulk = (mode & 2) && bulk_ok && rb1 <= a.nr * RE;
      if (lbulk || rbulk) {
        fence_proxy_async_smem();
        tx = (lbulk ? (uint32_t)(lb1 - lb0) : 0u) + (rbulk ? (uint32_t)(rb1 - rb0) : 0u);
        mbar_arrive_tx(&s_bar, tx);
        if (lbulk) bulk_copy_g2s(s_left, a.left + lb0, (uint32_t)(lb1 - lb0), &s_bar);
        if (rbulk) bulk_copy_g2s(s_right, a.right + rb0, (uint32_t)(rb1 - rb0), &s_bar);
        mode |= 4 | (lbulk ? 8u : 0u) | (rbulk ? 16u : 0u);
      }
      s_mode = mode;
    }
    // every output's row by an inclusive max-scan of the marks (row 0 owns the start)
    {
      constexpr uint32_t PER = kExpTile / kJoinThreads;
      __syncthreads();
      uint32_t m = 0, v[PER];
#pragma unroll
      for (uint32_t j = 0; j < PER; ++j) {
        m = max(m, (uint32_t)s_own[t * PER + j]);
        v[j] = m;
      }
      uint32_t inc = m;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= (uint32_t)o) inc = max(inc, y);
      }
      if (lane == 31) s_wmax[warp] = inc;
      uint32_t ex = __shfl_up_sync(0xffffffffu, inc, 1);
      if (lane == 0) ex = 0;
      __syncthreads();
      for (uint32_t w = 0; w < warp; ++w) ex = max(ex, s_wmax[w]);
#pragma unroll
      for (uint32_t j = 0; j < PER; ++j) s_own[t * PER + j] = (uint16_t)max(v[j], ex);
    }
    const uint32_t mode = s_mode;
    // the parts the bulk copies did not take: plain loads by all threads (4-byte words;
    // row sizes and the window bases are multiples of 4, the aligned ends stay inside
    // the arrays)
    if ((mode & 1) && !(mode & 8)) {
      const uint64_t b0 = i0 * LE, b1 = (i0 + span) * LE;
      for (uint64_t b = b0 + 4ull * t; b < b1; b += 4ull * kJoinThreads)
        *reinterpret_cast<uint32_t*>(s_left + (b - s_lbase)) = *reinterpret_cast<const uint32_t*>(a.left + b);
    }
    if ((mode & 2) && !(mode & 16)) {
      const uint64_t jhi = s_jhi > a.nr ? a.nr : s_jhi;
      const uint64_t b0 = (uint64_t)s_jlo * RE, b1 = jhi * RE;
      for (uint64_t b = b0 + 4ull * t; b < b1; b += 4ull * kJoinThreads)
        *reinterpret_cast<uint32_t*>(s_right + (b - s_rbase)) = *reinterpret_cast<const uint32_t*>(a.right + b);
    }
    if (mode & 4) {
      if (!mbar_wait(&s_bar, phase)) raise_error(a.err, kErrTimeout);
      phase ^= 1u;
    }
    __syncthreads();
    // outputs in order: consecutive threads write consecutive rows
#pragma unroll
    for (int v = 0; v < kExpVT; ++v) {
      const uint64_t k = k0 + (uint64_t)v * kJoinThreads + t;
      if (k >= k1) break;
      const uint32_t x = s_own[k - k0];
      const uint64_t i = i0 + x;
      const uint64_t j = s_lb[x] + (k - s_off[x]);
      if (j >= a.nr) continue;   // guards a timed-out scan
      const u128 L = (mode & 1) ? smem_row<LE>(s_left + (i * LE - s_lbase)) : load_u128<LE>(a.left, i);
      const bool rin = (mode & 2) && (uint64_t)j >= (uint64_t)s_jlo && j < (uint64_t)s_jhi;
      const u128 Rv = rin ? smem_row<RE>(s_right + (j * RE - s_rbase)) : load_u128<RE>(a.right, j);
      store_u128<OE>(a.out, k, (L << a.rv_bits) | (Rv & rmask));
    }
    __syncthreads();
  }
}

}  // namespace rfx
