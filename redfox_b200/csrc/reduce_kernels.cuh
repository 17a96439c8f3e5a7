// reduce_kernels.cuh -- reduce-by-key over runs of equal keys in one pass.
//
// Every item contributes the pair (head, value), head = 1 where a new run of equal keys
// starts.  The pairs are scanned with the segmented operator
//   (f1, v1) . (f2, v2) = (f1 + f2, f2 ? v2 : v1 + v2)
// within each thread, across the block, and across tiles by decoupled look-back; the
// inclusive pair at the last item of a run gives the run's output index (f - 1) and its
// total.  This is thrust::reduce_by_key with equal_to / plus (Reduce.cu:175-1536):
// output keys are the run keys in input order.
#pragma once

#include "lookback.cuh"
#include "rfx_device.cuh"
#include "search.cuh"
#include "sort_kernels.cuh"
#include "tile_ring.cuh"

namespace rfx {

constexpr int kRedThreads = 256;
constexpr int kRedIPT = 8;
constexpr int kRedTile = kRedThreads * kRedIPT;

enum ValKind : int { VAL_NONE = 0, VAL_U32 = 1, VAL_I64 = 2 };

// (f, v, h): run heads, running total since the last head (u64 arithmetic, wraps),
// position of the last head (max); a run's length at its last item i is i - h + 1.
using SegPair = SegPayload;

__device__ __forceinline__ SegPair seg_op(const SegPair& a, const SegPair& b) { return lb_combine(a, b); }

template <int K>
__device__ __forceinline__ bool elem_eq(const Elem<K>& a, const Elem<K>& b) {
  bool e = true;
#pragma unroll
  for (int k = 0; k < Elem<K>::NW; ++k) e = e && a.w[k] == b.w[k];
  return e;
}

struct ReduceArgs {
  const uint8_t* keys;
  const void* vals;
  uint64_t n_max;
  const uint64_t* d_n;   // optional device-resident count (<= n_max)
  uint64_t n_div;        // divide *d_n by this (byte sizes -> elements), 1 otherwise
  uint8_t* out_keys;
  void* out_vals;        // sums (type of the values), may be null
  uint32_t* out_counts;  // run lengths, may be null
  uint64_t* d_groups;
  uint64_t* d_groups_bytes_k;  // optional: groups * key bytes (reference byte sizes)
  uint64_t* d_groups_bytes_v;  // optional: groups * value bytes
  uint32_t* flags;       // [tiles] look-back flags
  SegPair* agg;          // [tiles]
  SegPair* inc;          // [tiles]
  uint32_t* tile_counter;
  uint32_t* err;
};

// Warp 0: exclusive prefix of this tile by look-back (flags released after payloads).
__device__ __forceinline__ void seg_lookback(const ReduceArgs& a, uint32_t tile, SegPair agg, SegPair* pre) {
  const uint32_t lane = threadIdx.x & 31;
  if (tile == 0) {
    if (lane == 0) {
      a.inc[0] = agg;
      st_release_u32(&a.flags[0], 2u);
    }
    *pre = SegPair{0, 0, 0};
    return;
  }
  if (lane == 0) {
    a.agg[tile] = agg;
    st_release_u32(&a.flags[tile], 1u);
  }
  SegPair run{0, 0, 0};
  int64_t base = (int64_t)tile - 1;
  uint32_t spins = 0;
  while (true) {
    const int64_t idx = base - (int64_t)lane;
    uint32_t fl = 2u;
    SegPair e{0, 0, 0};
    if (idx >= 0) {
      fl = ld_acquire_u32(&a.flags[idx]);
      if (fl == 1u) e = a.agg[idx];
      else if (fl == 2u) e = a.inc[idx];
    }
    const unsigned not_ready = __ballot_sync(0xffffffffu, fl == 0u);
    const unsigned inc = __ballot_sync(0xffffffffu, fl == 2u);
    const unsigned upto = inc ? ((inc & (0u - inc)) << 1) - 1 : 0xffffffffu;
    if (not_ready & upto) {
      if (++spins > kSpinLimit) {
        raise_error(a.err, kErrTimeout);
        break;
      }
      __nanosleep(spins < 64 ? 20 : 200);
      continue;
    }
    const bool in = (upto >> lane) & 1u;
    // fold lanes 0 (nearest) .. last usable (farthest) in sequence order
    const unsigned heads = __ballot_sync(0xffffffffu, in && e.f > 0);
    const unsigned vcut = heads ? ((heads & (0u - heads)) << 1) - 1 : upto;
    uint64_t f = in ? e.f : 0, v = ((vcut & upto) >> lane) & 1u ? e.v : 0, h = in ? e.h : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      f += __shfl_xor_sync(0xffffffffu, f, o);
      v += __shfl_xor_sync(0xffffffffu, v, o);
      const uint64_t ho = __shfl_xor_sync(0xffffffffu, h, o);
      h = h > ho ? h : ho;
    }
    run = seg_op(SegPair{f, v, h}, run);  // the window is older than what is folded so far
    if (inc) break;
    base -= 32;
  }
  if (lane == 0) {
    a.inc[tile] = seg_op(run, agg);
    st_release_u32(&a.flags[tile], 2u);
  }
  *pre = run;
}

// Block-wide exclusive scan with the segmented operator.
template <int NT>
__device__ __forceinline__ SegPair block_seg_exclusive(SegPair x, SegPair* s_warp, SegPair* total) {
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  SegPair incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    SegPair y;
    y.f = __shfl_up_sync(0xffffffffu, incl.f, o);
    y.v = __shfl_up_sync(0xffffffffu, incl.v, o);
    y.h = __shfl_up_sync(0xffffffffu, incl.h, o);
    if (lane >= (uint32_t)o) incl = seg_op(y, incl);
  }
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  SegPair wpre{0, 0, 0};
  for (uint32_t w = 0; w < warp; ++w) wpre = seg_op(wpre, s_warp[w]);
  SegPair tot{0, 0, 0};
  for (uint32_t w = 0; w < NT / 32; ++w) tot = seg_op(tot, s_warp[w]);
  *total = tot;
  SegPair ex;
  ex.f = __shfl_up_sync(0xffffffffu, incl.f, 1);
  ex.v = __shfl_up_sync(0xffffffffu, incl.v, 1);
  ex.h = __shfl_up_sync(0xffffffffu, incl.h, 1);
  if (lane == 0) ex = SegPair{0, 0, 0};
  return seg_op(wpre, ex);
}

// The same scan with the warp totals combined by a W-lane shuffle scan in every warp
// (constant work per thread instead of a loop over the warps).
template <int NT>
__device__ __forceinline__ SegPair block_seg_exclusive_fast(SegPair x, SegPair* s_warp, SegPair* total) {
  constexpr uint32_t W = NT / 32;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  SegPair incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    SegPair y;
    y.f = __shfl_up_sync(0xffffffffu, incl.f, o);
    y.v = __shfl_up_sync(0xffffffffu, incl.v, o);
    y.h = __shfl_up_sync(0xffffffffu, incl.h, o);
    if (lane >= (uint32_t)o) incl = seg_op(y, incl);
  }
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  SegPair wt = lane < W ? s_warp[lane] : SegPair{0, 0, 0};
#pragma unroll
  for (uint32_t o = 1; o < W; o <<= 1) {
    SegPair y;
    y.f = __shfl_up_sync(0xffffffffu, wt.f, o);
    y.v = __shfl_up_sync(0xffffffffu, wt.v, o);
    y.h = __shfl_up_sync(0xffffffffu, wt.h, o);
    if (lane >= o) wt = seg_op(y, wt);
  }
  const uint32_t src = warp ? warp - 1 : 0;
  SegPair wpre{__shfl_sync(0xffffffffu, wt.f, src), __shfl_sync(0xffffffffu, wt.v, src),
               __shfl_sync(0xffffffffu, wt.h, src)};
  if (warp == 0) wpre = SegPair{0, 0, 0};
  *total = SegPair{__shfl_sync(0xffffffffu, wt.f, W - 1), __shfl_sync(0xffffffffu, wt.v, W - 1),
                   __shfl_sync(0xffffffffu, wt.h, W - 1)};
  SegPair ex;
  ex.f = __shfl_up_sync(0xffffffffu, incl.f, 1);
  ex.v = __shfl_up_sync(0xffffffffu, incl.v, 1);
  ex.h = __shfl_up_sync(0xffffffffu, incl.h, 1);
  if (lane == 0) ex = SegPair{0, 0, 0};
  return seg_op(wpre, ex);
}

template <int K, int VK>
__global__ void __launch_bounds__(kRedThreads, 3)
reduce_by_key_kernel(const ReduceArgs a) {
  __shared__ SegPair s_warp[kRedThreads / 32];
  __shared__ SegPair s_pre;
  __shared__ uint32_t s_tile;
  const uint32_t t = threadIdx.x, warp = t >> 5;
  uint64_t n = a.n_max;
  if (a.d_n) n = min(n, *a.d_n / a.n_div);
  const uint64_t num_tiles = (n + kRedTile - 1) / kRedTile;
  while (true) {
    if (t == 0) s_tile = atomicAdd(a.tile_counter, 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    if (tile >= num_tiles) break;
    const uint64_t first = tile * kRedTile + (uint64_t)t * kRedIPT;  // blocked items
    Elem<K> key[kRedIPT];
    uint64_t val[kRedIPT];
    bool head[kRedIPT], tail[kRedIPT], valid[kRedIPT];
    Elem<K> prev;
    if (first > 0 && first < n) prev = load_elem<K>(a.keys, first - 1);
#pragma unroll
    for (int j = 0; j < kRedIPT; ++j) {
      const uint64_t i = first + j;
      valid[j] = i < n;
      if (valid[j]) {
        key[j] = load_elem<K>(a.keys, i);
        if constexpr (VK == VAL_I64) val[j] = (uint64_t)reinterpret_cast<const int64_t*>(a.vals)[i];
        else if constexpr (VK == VAL_U32) val[j] = reinterpret_cast<const uint32_t*>(a.vals)[i];
        else val[j] = 1;
      }
    }
#pragma unroll
    for (int j = 0; j < kRedIPT; ++j) {
      const uint64_t i = first + j;
      if (!valid[j]) {
        head[j] = false;
        continue;
      }
      if (i == 0) head[j] = true;
      else if (j == 0) head[j] = !elem_eq<K>(prev, key[0]);
      else head[j] = !elem_eq<K>(key[j - 1], key[j]);
    }
    // a run ends at i when i is the last item or item i+1 starts a new run
#pragma unroll
    for (int j = 0; j < kRedIPT; ++j) {
      const uint64_t i = first + j;
      if (!valid[j]) {
        tail[j] = false;
      } else if (i + 1 >= n) {
        tail[j] = true;
      } else if (j + 1 < kRedIPT) {
        tail[j] = head[j + 1];
      } else {
        const Elem<K> nx = load_elem<K>(a.keys, i + 1);
        tail[j] = !elem_eq<K>(key[j], nx);
      }
    }
    // thread aggregates
    SegPair tp{0, 0, 0};
#pragma unroll
    for (int j = 0; j < kRedIPT; ++j) {
      if (!valid[j]) continue;
      tp = seg_op(tp, SegPair{head[j] ? 1ull : 0ull, val[j], head[j] ? first + j : 0ull});
    }
    SegPair btot;
    SegPair ex = block_seg_exclusive<kRedThreads>(tp, s_warp, &btot);
    if (warp == 0) {
      SegPair pre;
      seg_lookback(a, (uint32_t)tile, btot, &pre);
      if (t == 0) {
        s_pre = pre;
        if (tile == num_tiles - 1) {
          const uint64_t groups = pre.f + btot.f;
          *a.d_groups = groups;
          if (a.d_groups_bytes_k) *a.d_groups_bytes_k = groups * (uint64_t)K;
          if (a.d_groups_bytes_v) *a.d_groups_bytes_v = groups * (VK == VAL_I64 ? 8ull : 4ull);
        }
      }
    }
    __syncthreads();
    SegPair run = seg_op(s_pre, ex);
#pragma unroll
    for (int j = 0; j < kRedIPT; ++j) {
      if (!valid[j]) continue;
      run = seg_op(run, SegPair{head[j] ? 1ull : 0ull, val[j], head[j] ? first + j : 0ull});
      if (tail[j]) {
        const uint64_t g = run.f - 1;
        if (g < n) {
          store_elem<K>(a.out_keys, g, key[j]);
          if (a.out_vals) {
            if constexpr (VK == VAL_I64) reinterpret_cast<int64_t*>(a.out_vals)[g] = (int64_t)run.v;
            else reinterpret_cast<uint32_t*>(a.out_vals)[g] = (uint32_t)run.v;
          }
          if (a.out_counts) a.out_counts[g] = (uint32_t)(first + j - run.h + 1);
        }
      }
    }
    __syncthreads();
  }
  if (n == 0 && blockIdx.x == 0 && t == 0) {
    *a.d_groups = 0;
    if (a.d_groups_bytes_k) *a.d_groups_bytes_k = 0;
    if (a.d_groups_bytes_v) *a.d_groups_bytes_v = 0;
  }
}

// ------------------------------------------------------------------ packed-tuple reduce
// The same segmented reduction over packed tuples of RB <= 16 bytes: the key is the row
// shifted right by key_shift (the high key fields), the value a field of the row
// (int64 sum), and the run key is written in OKB bytes.  Reduces a sorted join output
// without splitting it into key and value arrays (the split / set_split step of addAgg,
// RelationalAlgebraCompiler.cpp:7852-8643, fused away).

struct TupleReduceArgs {
  ReduceArgs r;
  uint32_t key_shift;
  uint32_t val_shift;
  uint64_t val_mask;
};

template <int RB, int OKB>
__global__ void __launch_bounds__(kRedThreads, 3)
reduce_tuples_kernel(const TupleReduceArgs ta) {
  const ReduceArgs& a = ta.r;
  __shared__ SegPair s_warp[kRedThreads / 32];
  __shared__ SegPair s_pre;
  __shared__ uint32_t s_tile;
  const uint32_t t = threadIdx.x, warp = t >> 5;
  uint64_t n = a.n_max;
  if (a.d_n) n = min(n, *a.d_n / a.n_div);
  const uint64_t num_tiles = (n + kRedTile - 1) / kRedTile;
  while (true) {
    if (t == 0) s_tile = atomicAdd(a.tile_counter, 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    if (tile >= num_tiles) break;
    const uint64_t first = tile * kRedTile + (uint64_t)t * kRedIPT;
    u128 key[kRedIPT];
    uint64_t val[kRedIPT];
    bool head[kRedIPT], tail[kRedIPT], valid[kRedIPT];
    u128 prev = 0;
    if (first > 0 && first < n) prev = load_u128<RB>(a.keys, first - 1) >> ta.key_shift;
#pragma unroll
    for (int j = 0; j < kRedIPT; ++j) {
      const uint64_t i = first + j;
      valid[j] = i < n;
      if (valid[j]) {
        const u128 row = load_u128<RB>(a.keys, i);
        key[j] = row >> ta.key_shift;
        val[j] = (uint64_t)(row >> ta.val_shift) & ta.val_mask;
      }
    }
#pragma unroll
    for (int j = 0; j < kRedIPT; ++j) {
      const uint64_t i = first + j;
      if (!valid[j]) {
        head[j] = false;
        continue;
      }
      head[j] = i == 0 || (j == 0 ? prev != key[0] : key[j - 1] != key[j]);
    }
#pragma unroll
    for (int j = 0; j < kRedIPT; ++j) {
      const uint64_t i = first + j;
      if (!valid[j]) tail[j] = false;
      else if (i + 1 >= n) tail[j] = true;
      else if (j + 1 < kRedIPT) tail[j] = head[j + 1];
      else tail[j] = key[j] != (load_u128<RB>(a.keys, i + 1) >> ta.key_shift);
    }
    SegPair tp{0, 0, 0};
#pragma unroll
    for (int j = 0; j < kRedIPT; ++j) {
      if (!valid[j]) continue;
      tp = seg_op(tp, SegPair{head[j] ? 1ull : 0ull, val[j], head[j] ? first + j : 0ull});
    }
    SegPair btot;
    SegPair ex = block_seg_exclusive<kRedThreads>(tp, s_warp, &btot);
    if (warp == 0) {
      SegPair pre;
      seg_lookback(a, (uint32_t)tile, btot, &pre);
      if (t == 0) {
        s_pre = pre;
        if (tile == num_tiles - 1) *a.d_groups = pre.f + btot.f;
      }
    }
    __syncthreads();
    SegPair run = seg_op(s_pre, ex);
#pragma unroll
    for (int j = 0; j < kRedIPT; ++j) {
      if (!valid[j]) continue;
      run = seg_op(run, SegPair{head[j] ? 1ull : 0ull, val[j], head[j] ? first + j : 0ull});
      if (tail[j]) {
        const uint64_t g = run.f - 1;
        if (g < n) {
          store_u128<OKB>(a.out_keys, g, key[j]);
          if (a.out_vals) reinterpret_cast<int64_t*>(a.out_vals)[g] = (int64_t)run.v;
          if (a.out_counts) a.out_counts[g] = (uint32_t)(first + j - run.h + 1);
        }
      }
    }
    __syncthreads();
  }
  if (n == 0 && blockIdx.x == 0 && t == 0) *a.d_groups = 0;
}

// ------------------------------------------------------------------ TMA-staged row reduce
// The same reduction with every 32 KB tile of rows brought into shared memory by the
// tile ring (tile_ring.cuh) and tile prefixes resolved by the block-wide look-back
// (lookback.cuh).  Thread t owns the 128-byte line t of the tile (128 / RB rows).
//   pass 1: head bits of the thread's rows and the running sum since its last head give
//           the thread's (f, v, h) = (popc(heads), sum, last head); block scan; the tile
//           aggregate is published;
//   pass 2: after the look-back, the rows are read again from shared memory; at each
//           run end the group index is the carried f plus the heads so far.
// Pipeline of one block over three stages.  Step k: claim tile k+2 and start its copy;
// resolve the prefix of tile k (warp 0) and run its pass 2; wait for tile k+2's rows,
// run its pass 1 and publish its aggregate.  A tile is therefore resolved one full step
// after its aggregate was published, when its predecessors have published theirs too,
// and only the copy (never a waiting look-back of another tile) lies between a tile's
// claim and its aggregate: a slow look-back cannot hold up the aggregates that other
// blocks' look-backs wait for.
//
// Row shapes: SHAPE 0 takes key = row >> key_shift and value = (row >> value_shift) &
// mask at run time; SHAPE 1 / 2 are 16-byte rows with the key in the top 32 / 64 bits
// and a 64-bit value in the low 64 bits (the join outputs the plans reduce).

enum RowShape : int { ROW_GENERIC = 0, ROW16_K32_V64 = 1, ROW16_K64_V64 = 2 };

template <int RB>
struct RowWord;
template <>
struct RowWord<4> { typedef uint32_t T; };
template <>
struct RowWord<8> { typedef uint64_t T; };
template <>
struct RowWord<16> { typedef u128 T; };

template <int RB, int SHAPE>
struct RowAccess {
  typedef typename RowWord<RB>::T Key;
  __device__ __forceinline__ static void read(const uint8_t* st, uint32_t r, uint32_t ks, uint32_t vs,
                                              uint64_t vmask, Key& k, uint64_t& v) {
    typename RowWord<RB>::T row;
    if constexpr (RB == 16) {
      const uint4 w = ring_read<uint4>(st, r * 16u);
      row = ((u128)(((uint64_t)w.w << 32) | w.z) << 64) | (((uint64_t)w.y << 32) | w.x);
    } else {
      row = ring_read<typename RowWord<RB>::T>(st, r * (uint32_t)RB);
    }
    k = row >> ks;
    v = (uint64_t)(row >> vs) & vmask;
  }
  __device__ __forceinline__ static Key global_key(const uint8_t* rows, uint64_t i, uint32_t ks) {
    return (Key)(load_u128<RB>(rows, i) >> ks);
  }
};
template <>
struct RowAccess<16, ROW16_K32_V64> {
  typedef uint32_t Key;
  __device__ __forceinline__ static void read(const uint8_t* st, uint32_t r, uint32_t, uint32_t, uint64_t, Key& k,
                                              uint64_t& v) {
    const uint4 w = ring_read<uint4>(st, r * 16u);
    k = w.w;
    v = ((uint64_t)w.y << 32) | w.x;
  }
  __device__ __forceinline__ static Key global_key(const uint8_t* rows, uint64_t i, uint32_t) {
    return __ldg(reinterpret_cast<const uint32_t*>(rows + i * 16) + 3);
  }
};
template <>
struct RowAccess<16, ROW16_K64_V64> {
  typedef uint64_t Key;
  __device__ __forceinline__ static void read(const uint8_t* st, uint32_t r, uint32_t, uint32_t, uint64_t, Key& k,
                                              uint64_t& v) {
    const uint4 w = ring_read<uint4>(st, r * 16u);
    k = ((uint64_t)w.w << 32) | w.z;
    v = ((uint64_t)w.y << 32) | w.x;
  }
  __device__ __forceinline__ static Key global_key(const uint8_t* rows, uint64_t i, uint32_t) {
    return __ldg(reinterpret_cast<const unsigned long long*>(rows + i * 16) + 1);
  }
};

struct RowReduceArgs {
  const uint8_t* rows;
  uint64_t n_max;
  const uint64_t* d_n;
  uint64_t full_lines;   // 128-byte lines covered by the tensor map
  uint32_t key_shift;
  uint32_t val_shift;
  uint64_t val_mask;
  uint32_t out_key_bytes;
  uint8_t* out_keys;
  int64_t* out_sums;
  uint32_t* out_counts;
  uint64_t* d_groups;
  SegRecord* records;
  uint32_t* tile_counter;
  uint32_t* err;
};

constexpr int kRowRedStages = 3;

__device__ __forceinline__ uint8_t* align1024(uint8_t* p) {
  const uint32_t a = smem_u32(p);
  return p + ((1024u - (a & 1023u)) & 1023u);
}

template <typename K>
__device__ __forceinline__ void store_key(uint8_t* out, uint64_t g, uint32_t okb, K k) {
  if (okb == 4) reinterpret_cast<uint32_t*>(out)[g] = (uint32_t)k;
  else if (okb == 8) reinterpret_cast<uint64_t*>(out)[g] = (uint64_t)k;
  else store_u128<16>(out, g, (u128)k);
}

// State of an aggregated, not yet resolved tile.
struct RowTileState {
  uint64_t tile;
  SegPair ex, btot;
  uint32_t heads, nvalid;
};

template <int RB, int SHAPE, int S, int NT>
__global__ void __launch_bounds__(NT, 512 / NT) reduce_rows_kernel(const __grid_constant__ CUtensorMap map,
                                                                     const RowReduceArgs a) {
  constexpr uint32_t TILE_BYTES = NT * kRingLineBytes;
  constexpr uint32_t TR = TILE_BYTES / RB;
  constexpr uint32_t IPT = TR / NT;
  static_assert(IPT * RB == kRingLineBytes && IPT <= 32, "one 128-byte line per thread");
  static_assert(S == 3, "stages: the tile in pass 2, the aggregated tile, the tile being copied");
  typedef RowAccess<RB, SHAPE> RA;
  typedef typename RA::Key Key;
  extern __shared__ uint8_t dyn_smem[];
  uint8_t* stages = align1024(dyn_smem);
  __shared__ TileRing<S> ring;
  __shared__ SegPair s_warp[NT / 32];
  __shared__ SegPair s_pre;
  const uint32_t t = threadIdx.x;
  uint64_t n = a.n_max;
  if (a.d_n) n = min(n, *a.d_n);
  const uint64_t num_tiles = (n + TR - 1) / TR;
  const uint64_t covered = a.full_lines * kRingLineBytes;
  const uint32_t ks = a.key_shift, vs = a.val_shift;
  const uint64_t vmask = a.val_mask;
  const uint32_t tb = t * IPT;
  if (t == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&ring.bar[s], 1);
    mbar_fence_init();
    if (a.full_lines) prefetch_map(&map);
  }
  __syncthreads();

  // claim the next tile into stage s and start its copy (thread 0)
  auto claim = [&](int s) {
    const uint32_t tl = atomicAdd(a.tile_counter, 1u);
    ring.tile[s] = tl;
    if (tl >= num_tiles) return;
    const uint64_t line0 = (uint64_t)tl * NT;
    const bool copy = line0 < a.full_lines;
    mbar_arrive_tx(&ring.bar[s], copy ? TILE_BYTES : 0u);
    if (copy) tma_load_lines(stages + (size_t)s * TILE_BYTES, &map, (uint32_t)line0, &ring.bar[s]);
  };
  // pass 1 of the tile in stage s (its u-th use); tile = ~0 when the claim ran out or a
  // copy timed out (ok = false)
  bool ok = true;
  auto pass1 = [&](int s, uint32_t u) -> RowTileState {
    RowTileState r;
    r.tile = ring.tile[s];
    r.heads = 0;
    r.nvalid = 0;
    r.ex = r.btot = SegPair{0, 0, 0};
    if (r.tile >= num_tiles) return r;
    uint8_t* st = stages + (size_t)s * TILE_BYTES;
    bool w = true;
    if (t == 0) w = mbar_wait(&ring.bar[s], u & 1u);
    if (!__syncthreads_and(w)) {
      ok = false;
      r.tile = ~0ull;
      return r;
    }
    if ((r.tile + 1) * TILE_BYTES > covered) {
      ring_fill_tail(st, a.rows, r.tile, covered, n * RB, TILE_BYTES);
      __syncthreads();
    }
    const uint64_t first = r.tile * TR + tb;
    r.nvalid = first >= n ? 0u : (uint32_t)min((uint64_t)IPT, n - first);
    Key pk = 0;
    uint64_t v = 0;
    if (t > 0) RA::read(st, tb - 1, ks, vs, vmask, pk, v);
    else if (first > 0) pk = RA::global_key(a.rows, first - 1, ks);
    uint64_t acc = 0;
#pragma unroll
    for (uint32_t j = 0; j < IPT; ++j) {
      if (j < r.nvalid) {
        Key key;
        RA::read(st, tb + j, ks, vs, vmask, key, v);
        const bool h = key != pk || (j == 0 && first == 0);
        pk = key;
        r.heads |= (uint32_t)h << j;
        acc = h ? v : acc + v;
      }
    }
    const SegPair tp{(uint64_t)__popc(r.heads), acc, r.heads ? first + (31u - __clz(r.heads)) : 0ull};
    r.ex = block_seg_exclusive_fast<NT>(tp, s_warp, &r.btot);
    lb_publish(a.records, r.tile, r.btot);
    return r;
  };

  if (t == 0) {
    claim(0);
    claim(1);
  }
  __syncthreads();
  RowTileState cur = pass1(0, 0);
  RowTileState nxt = pass1(1, 0);
  for (uint32_t k = 0; ok && cur.tile < num_tiles; ++k) {
    const int s = (int)(k % S);
    if (t < 32) {
      if (t == 0) {
        // stage of tile k-1: its pass 2 ended before the barriers of the last pass 1
        fence_proxy_async_smem();
        claim((int)((k + 2) % S));
      }
      const SegPair p = warp_lookback_resolve<4>(a.records, cur.tile, cur.btot, a.err);
      if (t == 0) s_pre = p;
    }
    __syncthreads();
    const SegPair pre = s_pre;
    if (t == 0 && cur.tile == num_tiles - 1) *a.d_groups = pre.f + cur.btot.f;
    // pass 2: one output per run end
    const uint8_t* st = stages + (size_t)s * TILE_BYTES;
    const uint64_t first = cur.tile * TR + tb;
    const SegPair carry = seg_op(pre, cur.ex);
    const uint32_t heads = cur.heads, nvalid = cur.nvalid;
    uint64_t acc = carry.v, hpos = carry.h;
    Key nk = 0;
    const bool next_valid = first + IPT < n;
    if (next_valid) {
      if (t + 1 < (uint32_t)NT) {
        uint64_t dv;
        RA::read(st, tb + IPT, ks, vs, vmask, nk, dv);
      } else {
        nk = RA::global_key(a.rows, first + IPT, ks);
      }
    }
#pragma unroll
    for (uint32_t j = 0; j < IPT; ++j) {
      if (j < nvalid) {
        Key key;
        uint64_t v;
        RA::read(st, tb + j, ks, vs, vmask, key, v);
        const bool h = (heads >> j) & 1u;
        acc = h ? v : acc + v;
        if (h) hpos = first + j;
        bool tail;
        if (j + 1 < nvalid) tail = (heads >> (j + 1)) & 1u;
        else if (j + 1 < IPT) tail = true;            // last valid row of the relation
        else tail = !next_valid || key != nk;
        if (tail) {
          const uint64_t g = carry.f + (uint64_t)__popc(heads & ((2u << j) - 1u)) - 1;
          if (g < n) {
            store_key(a.out_keys, g, a.out_key_bytes, key);
            if (a.out_sums) a.out_sums[g] = (int64_t)acc;
            if (a.out_counts) a.out_counts[g] = (uint32_t)(first + j - hpos + 1);
          }
        }
      }
    }
    __syncthreads();
    cur = nxt;
    const int s2 = (int)((k + 2) % S);
    nxt = pass1(s2, (k + 2) / S);
  }
  if (!ok && t == 0) raise_error(a.err, kErrTimeout);
  if (n == 0 && blockIdx.x == 0 && t == 0) *a.d_groups = 0;
}

// A key from lane `src` of the warp (32-, 64- or 128-bit keys).
template <typename K>
__device__ __forceinline__ K shfl_key(K k, uint32_t src) {
  if constexpr (sizeof(K) <= 4) {
    return (K)__shfl_sync(0xffffffffu, (uint32_t)k, src);
  } else if constexpr (sizeof(K) == 8) {
    return (K)__shfl_sync(0xffffffffu, (unsigned long long)k, src);
  } else {
    const unsigned long long lo = __shfl_sync(0xffffffffu, (unsigned long long)k, src);
    const unsigned long long hi = __shfl_sync(0xffffffffu, (unsigned long long)(k >> 64), src);
    return ((K)hi << 64) | (K)lo;
  }
}

// ------------------------------------------------------------------ chunked variant
// Each block claims a contiguous chunk of tiles and streams it through the three-stage
// TMA ring, carrying the open run from tile to tile in registers, so no tile waits for
// another block.  Runs that start and end inside the chunk are written to the chunk's
// scratch area at their chunk-local index (the heads before them in the chunk).  After
// its last tile the block publishes the chunk's aggregate and resolves the exclusive
// prefix over chunks (one look-back per chunk): its f is the chunk's base group index and
// (v, h) the run left open when the chunk began.  The block then closes that run (its end
// lies in this chunk: total = carried v plus the chunk's first partial) and copies its
// scratch groups to base + local index.  A chunk with more groups than its scratch holds
// runs its tiles a second time, writing straight to base + local index.  Traffic: the
// rows once, the groups twice (scratch and final) -- the groups are few where a reduce
// follows a join.
struct ChunkReduceArgs {
  RowReduceArgs r;          // records: one per chunk; tile_counter: the chunk counter
  uint64_t tiles_per_chunk;
  uint32_t cap;             // scratch groups per chunk
  uint8_t* s_keys;          // [chunks * cap] keys of out_key_bytes
  int64_t* s_sums;          // [chunks * cap]
  uint32_t* s_counts;       // [chunks * cap]
};

template <int RB, int SHAPE, int S, int NT>
__global__ void __launch_bounds__(NT, (S <= 2 ? 768 : 512) / NT) reduce_chunks_kernel(const __grid_constant__ CUtensorMap map,
                                                                       const ChunkReduceArgs ca) {
  constexpr uint32_t TILE_BYTES = NT * kRingLineBytes;
  constexpr uint32_t TR = TILE_BYTES / RB;
  constexpr uint32_t IPT = TR / NT;
  static_assert(IPT * RB == kRingLineBytes && IPT <= 32, "one 128-byte line per thread");
  typedef RowAccess<RB, SHAPE> RA;
  typedef typename RA::Key Key;
  const RowReduceArgs& a = ca.r;
  extern __shared__ uint8_t dyn_smem[];
  uint8_t* stages = align1024(dyn_smem);
  __shared__ TileRing<S> ring;
  __shared__ SegPair s_warp[NT / 32];
  __shared__ SegPair s_pre;
  __shared__ uint32_t s_chunk, s_nlocal, s_overflow, s_has_first;
  __shared__ uint64_t s_first_sum, s_first_tail;
  __shared__ Key s_first_key;
  const uint32_t t = threadIdx.x;
  uint64_t n = a.n_max;
  if (a.d_n) n = min(n, *a.d_n);
  const uint64_t num_tiles = (n + TR - 1) / TR;
  const uint64_t covered = a.full_lines * kRingLineBytes;
  const uint32_t ks = a.key_shift, vs = a.val_shift;
  const uint64_t vmask = a.val_mask;
  const uint32_t tb = t * IPT;
  if (t == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&ring.bar[s], 1);
    mbar_fence_init();
    if (a.full_lines) prefetch_map(&map);
    s_chunk = atomicAdd(a.tile_counter, 1u);   // claim order = the look-back order
    s_nlocal = 0;
    s_overflow = 0;
    s_has_first = 0;
  }
  __syncthreads();
  const uint64_t c = s_chunk;
  const uint64_t t0 = c * ca.tiles_per_chunk;
  const uint64_t t1 = min(t0 + ca.tiles_per_chunk, num_tiles);
  const uint64_t ntiles = t0 < t1 ? t1 - t0 : 0;
  uint32_t uses[S];
#pragma unroll
  for (int s = 0; s < S; ++s) uses[s] = 0;
  bool ok = true;

  // start the copy of chunk tile i into its stage (thread 0)
  auto issue = [&](uint64_t i) {
    const int s = (int)(i % S);
    const uint64_t tl = t0 + i;
    const uint64_t line0 = tl * NT;
    const bool copy = line0 < a.full_lines;
    mbar_arrive_tx(&ring.bar[s], copy ? TILE_BYTES : 0u);
    if (copy) tma_load_lines(stages + (size_t)s * TILE_BYTES, &map, (uint32_t)line0, &ring.bar[s]);
  };

  // one pass over the chunk's tiles; direct: write to base + local index, else scratch
  auto run_chunk = [&](bool direct, uint64_t base) -> SegPair {
    SegPair run{0, 0, 0};
    if (t == 0) {
      fence_proxy_async_smem();   // a second pass reuses stages the first one read
      for (uint64_t i = 0; i < (uint64_t)S && i < ntiles; ++i) issue(i);
    }
    for (uint64_t i = 0; i < ntiles && ok; ++i) {
      const int s = (int)(i % S);
      const uint64_t tile = t0 + i;
      uint8_t* st = stages + (size_t)s * TILE_BYTES;
      bool w = true;
      if (t == 0) w = mbar_wait(&ring.bar[s], uses[s] & 1u);
      ++uses[s];
      if (!__syncthreads_and(w)) {
        ok = false;
        break;
      }
      if ((tile + 1) * TILE_BYTES > covered) {
        ring_fill_tail(st, a.rows, tile, covered, n * RB, TILE_BYTES);
        __syncthreads();
      }
      // pass 1: this thread's rows into registers, heads, this thread's (f, v, h); the
      // neighbouring keys come from the adjacent lanes
      const uint64_t first = tile * TR + tb;
      const uint32_t nvalid = first >= n ? 0u : (uint32_t)min((uint64_t)IPT, n - first);
      Key key[IPT];
      uint64_t val[IPT];
#pragma unroll
      for (uint32_t j = 0; j < IPT; ++j) {
        key[j] = 0;
        val[j] = 0;
        if (j < nvalid) RA::read(st, tb + j, ks, vs, vmask, key[j], val[j]);
      }
      const uint32_t lane = t & 31;
      Key pk = shfl_key(key[IPT - 1], lane ? lane - 1 : 0);
      Key nk = shfl_key(key[0], lane < 31 ? lane + 1 : 31);
      uint64_t v = 0;
      if (lane == 0) {
        if (t > 0) RA::read(st, tb - 1, ks, vs, vmask, pk, v);
        else if (first > 0) pk = RA::global_key(a.rows, first - 1, ks);
      }
      const bool next_valid = first + IPT < n;
      if (lane == 31 && next_valid) {
        if (t + 1 < (uint32_t)NT) RA::read(st, tb + IPT, ks, vs, vmask, nk, v);
        else nk = RA::global_key(a.rows, first + IPT, ks);
      }
      uint32_t heads = 0;
      uint64_t acc = 0;
#pragma unroll
      for (uint32_t j = 0; j < IPT; ++j) {
        if (j < nvalid) {
          const bool h = key[j] != (j ? key[j - 1] : pk) || (j == 0 && first == 0);
          heads |= (uint32_t)h << j;
          acc = h ? val[j] : acc + val[j];
        }
      }
      const SegPair tp{(uint64_t)__popc(heads), acc, heads ? first + (31u - __clz(heads)) : 0ull};
      SegPair btot;
      const SegPair ex = block_seg_exclusive_fast<NT>(tp, s_warp, &btot);
      // pass 2: one output per run end; the carry is chunk-local
      const SegPair carry = seg_op(run, ex);
      uint64_t racc = carry.v, hpos = carry.h;
#pragma unroll
      for (uint32_t j = 0; j < IPT; ++j) {
        if (j < nvalid) {
          const bool h = (heads >> j) & 1u;
          racc = h ? val[j] : racc + val[j];
          if (h) hpos = first + j;
          bool tail;
          if (j + 1 < nvalid) tail = (heads >> (j + 1)) & 1u;
          else if (j + 1 < IPT) tail = true;            // last row of the relation
          else tail = !next_valid || key[j] != nk;
          if (tail) {
            const uint64_t lf = carry.f + (uint64_t)__popc(heads & ((2u << j) - 1u));
            if (lf == 0) {
              // the run that was open when the chunk began ends here
              if (!direct) {
                s_first_sum = racc;
                s_first_tail = first + j;
                s_first_key = key[j];
                s_has_first = 1;
              }
            } else if (direct) {
              const uint64_t g = base + lf - 1;
              if (g < n) {
                store_key(a.out_keys, g, a.out_key_bytes, key[j]);
                if (a.out_sums) a.out_sums[g] = (int64_t)racc;
                if (a.out_counts) a.out_counts[g] = (uint32_t)(first + j - hpos + 1);
              }
            } else if (lf - 1 < ca.cap) {
              const uint64_t g = c * ca.cap + lf - 1;
              store_key(ca.s_keys, g, a.out_key_bytes, key[j]);
              ca.s_sums[g] = (int64_t)racc;
              ca.s_counts[g] = (uint32_t)(first + j - hpos + 1);
              atomicMax(&s_nlocal, (uint32_t)lf);
            } else {
              s_overflow = 1;
            }
          }
        }
      }
      run = seg_op(run, btot);
      __syncthreads();
      if (t == 0 && i + S < ntiles) {
        fence_proxy_async_smem();
        issue(i + S);
      }
    }
    return run;
  };

  const SegPair agg = run_chunk(false, 0);
  // the chunk's base and the run open at its start (look-back over chunks)
  lb_publish(a.records, c, agg);
  if (t < 32) {
    const SegPair p = warp_lookback_resolve<4>(a.records, c, agg, a.err);
    if (t == 0) s_pre = p;
  }
  __syncthreads();
  const SegPair pre = s_pre;
  if (t == 0 && ntiles && t1 == num_tiles) *a.d_groups = pre.f + agg.f;
  if (t == 0 && n == 0 && c == 0) *a.d_groups = 0;
  if (t == 0 && s_has_first && pre.f > 0) {
    const uint64_t g = pre.f - 1;
    store_key(a.out_keys, g, a.out_key_bytes, s_first_key);
    if (a.out_sums) a.out_sums[g] = (int64_t)(pre.v + s_first_sum);
    if (a.out_counts) a.out_counts[g] = (uint32_t)(s_first_tail - pre.h + 1);
  }
  if (s_overflow) {
    __syncthreads();
    run_chunk(true, pre.f);
  } else {
    const uint32_t nl = s_nlocal;
    for (uint32_t l = t; l < nl; l += NT) {
      const uint64_t src = c * ca.cap + l, g = pre.f + l;
      if (a.out_key_bytes == 4) reinterpret_cast<uint32_t*>(a.out_keys)[g] = reinterpret_cast<const uint32_t*>(ca.s_keys)[src];
      else if (a.out_key_bytes == 8) reinterpret_cast<uint64_t*>(a.out_keys)[g] = reinterpret_cast<const uint64_t*>(ca.s_keys)[src];
      else reinterpret_cast<uint4*>(a.out_keys)[g] = reinterpret_cast<const uint4*>(ca.s_keys)[src];
      if (a.out_sums) a.out_sums[g] = ca.s_sums[src];
      if (a.out_counts) a.out_counts[g] = ca.s_counts[src];
    }
  }
  if (!ok && t == 0) raise_error(a.err, kErrTimeout);
}

// ------------------------------------------------------------------ warp-chunked variant
// The chunked form with the block taken out of the per-tile path: a block claims a chunk,
// and each of its warps streams its own contiguous sub-chunk through a private TMA ring
// of 4 KB boxes (32 lines, one per lane), scans within the warp (shuffles only) and
// carries the open run in registers.  No barrier and no look-back lies on the per-tile
// path.  At the end the block folds its warps' aggregates in order, resolves one prefix
// for the chunk, and each warp closes the run open at its sub-chunk's start and copies its
// scratch groups (or runs its sub-chunk again, writing directly, if they overflowed).

template <int WARPS>
__device__ __forceinline__ void warp_fill_tail(uint8_t* stage, const uint8_t* src, uint64_t tile, uint64_t covered,
                                               uint64_t limit, uint32_t tile_bytes, uint32_t lane) {
  const uint64_t t0 = tile * tile_bytes;
  const uint64_t lo = covered > t0 ? covered : t0;
  const uint64_t hi = limit < t0 + tile_bytes ? limit : t0 + tile_bytes;
  if (lo >= hi) return;
  const uint64_t hi4 = lo + ((hi - lo) & ~3ull);
  for (uint64_t b = lo + 4ull * lane; b < hi4; b += 128ull) {
    const uint32_t w = *reinterpret_cast<const uint32_t*>(src + b);
    *reinterpret_cast<uint32_t*>(stage + swz((uint32_t)(b - t0))) = w;
  }
  if (lane == 0)
    for (uint64_t b = hi4; b < hi; ++b) stage[swz((uint32_t)(b - t0))] = src[b];
}

__device__ __forceinline__ SegPair shfl_seg(const SegPair& x, uint32_t src) {
  return SegPair{__shfl_sync(0xffffffffu, x.f, src), __shfl_sync(0xffffffffu, x.v, src),
                 __shfl_sync(0xffffffffu, x.h, src)};
}

template <int RB, int SHAPE, int S, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 2) reduce_warps_kernel(const __grid_constant__ CUtensorMap map,
                                                                       const ChunkReduceArgs ca) {
  constexpr uint32_t LINES = 32;
  constexpr uint32_t TILE_BYTES = LINES * kRingLineBytes;
  constexpr uint32_t TR = TILE_BYTES / RB;
  constexpr uint32_t IPT = TR / 32;
  static_assert(IPT * RB == kRingLineBytes && IPT <= 32, "one 128-byte line per lane");
  typedef RowAccess<RB, SHAPE> RA;
  typedef typename RA::Key Key;
  const RowReduceArgs& a = ca.r;
  extern __shared__ uint8_t dyn_smem[];
  uint8_t* stages = align1024(dyn_smem);
  __shared__ uint64_t bars[WARPS][S];
  __shared__ SegPair s_wagg[WARPS];
  __shared__ SegPair s_pre;
  __shared__ uint32_t s_chunk;
  const uint32_t t = threadIdx.x, lane = t & 31, w = t >> 5;
  uint64_t n = a.n_max;
  if (a.d_n) n = min(n, *a.d_n);
  const uint64_t num_tiles = (n + TR - 1) / TR;
  const uint64_t covered = a.full_lines * kRingLineBytes;
  const uint32_t ks = a.key_shift, vs = a.val_shift;
  const uint64_t vmask = a.val_mask;
  if (t == 0) {
    s_chunk = atomicAdd(a.tile_counter, 1u);   // claim order = the look-back order
    if (a.full_lines) prefetch_map(&map);
  }
  if (lane == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&bars[w][s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  const uint64_t bc = s_chunk;
  const uint64_t sub = bc * WARPS + w;
  const uint64_t tpc = ca.tiles_per_chunk;     // tiles per warp sub-chunk
  const uint64_t t0 = sub * tpc;
  const uint64_t t1 = min(t0 + tpc, num_tiles);
  const uint64_t ntiles = t0 < t1 ? t1 - t0 : 0;
  uint8_t* wst = stages + (size_t)w * S * TILE_BYTES;
  uint32_t uses[S];
#pragma unroll
  for (int s = 0; s < S; ++s) uses[s] = 0;
  bool ok = true;
  // this lane's record of the run open at the sub-chunk's start, if it ends here
  bool has_first = false, overflow = false;
  uint64_t first_sum = 0, first_tail = 0;
  Key first_key = 0;
  uint32_t max_lf = 0;

  auto issue = [&](uint64_t i) {
    const int s = (int)(i % S);
    const uint64_t line0 = (t0 + i) * LINES;
    const bool copy = line0 < a.full_lines;
    mbar_arrive_tx(&bars[w][s], copy ? TILE_BYTES : 0u);
    if (copy) tma_load_lines(wst + (size_t)s * TILE_BYTES, &map, (uint32_t)line0, &bars[w][s]);
  };

  // a group that ends at row `tail` with index lf (1-based, 0: the run open at the
  // sub-chunk's start), total `sum`, head at `hpos`
  auto emit = [&](bool direct, uint64_t base, uint64_t lf, Key key, uint64_t sum, uint64_t tail, uint64_t hpos) {
    if (lf == 0) {
      if (!direct) {
        has_first = true;
        first_sum = sum;
        first_tail = tail;
        first_key = key;
      }
    } else if (direct) {
      const uint64_t g = base + lf - 1;
      if (g < n) {
        store_key(a.out_keys, g, a.out_key_bytes, key);
        if (a.out_sums) a.out_sums[g] = (int64_t)sum;
        if (a.out_counts) a.out_counts[g] = (uint32_t)(tail - hpos + 1);
      }
    } else if (lf - 1 < ca.cap) {
      const uint64_t g = sub * ca.cap + lf - 1;
      store_key(ca.s_keys, g, a.out_key_bytes, key);
      ca.s_sums[g] = (int64_t)sum;
      ca.s_counts[g] = (uint32_t)(tail - hpos + 1);
      max_lf = max(max_lf, (uint32_t)lf);
    } else {
      overflow = true;
    }
  };

  auto run_sub = [&](bool direct, uint64_t base) -> SegPair {
    SegPair run{0, 0, 0};
    if (lane == 0) {
      fence_proxy_async_smem();   // a second pass reuses stages the first one read
      for (uint64_t i = 0; i < (uint64_t)S && i < ntiles; ++i) issue(i);
    }
    __syncwarp();
    // the key of the row before the current tile, and whether that row's run end is
    // still undecided (it is the last row of the previous tile)
    Key last_key = 0;
    bool pending = false;
    if (ntiles && t0 * TR > 0 && t0 * TR <= n) last_key = RA::global_key(a.rows, t0 * TR - 1, ks);
    for (uint64_t i = 0; i < ntiles && ok; ++i) {
      const int s = (int)(i % S);
      const uint64_t tile = t0 + i;
      uint8_t* st = wst + (size_t)s * TILE_BYTES;
      const bool wok = mbar_wait(&bars[w][s], uses[s] & 1u);
      ++uses[s];
      if (!__all_sync(0xffffffffu, wok)) {
        ok = false;
        break;
      }
      if ((tile + 1) * TILE_BYTES > covered) {
        warp_fill_tail<WARPS>(st, a.rows, tile, covered, n * RB, TILE_BYTES, lane);
        __syncwarp();
      }
      const uint64_t first = tile * TR + lane * IPT;
      if (IPT <= 16 && (tile + 1) * TR <= n) {
        // a full tile: every lane holds IPT rows; the scan carries (heads << 16 | position
        // of the last head within the tile) in one word and the sum in another
        const uint64_t tile_row = tile * TR;
        Key key[IPT];
        uint64_t val[IPT], racc[IPT];
#pragma unroll
        for (uint32_t j = 0; j < IPT; ++j) RA::read(st, lane * IPT + j, ks, vs, vmask, key[j], val[j]);
        // the rows are in registers: refill the stage now
        __syncwarp();
        if (lane == 0 && i + S < ntiles) {
          fence_proxy_async_smem();
          issue(i + S);
        }
        Key pk = shfl_key(key[IPT - 1], lane ? lane - 1 : 0);
        const Key nk = shfl_key(key[0], lane < 31 ? lane + 1 : 31);
        if (lane == 0) pk = last_key;
        uint32_t heads = 0;
        uint64_t acc = 0;
#pragma unroll
        for (uint32_t j = 0; j < IPT; ++j) {
          const bool h = key[j] != (j ? key[j - 1] : pk) || (j == 0 && first == 0);
          heads |= (uint32_t)h << j;
          acc = h ? val[j] : acc + val[j];
          racc[j] = acc;
        }
        if (lane == 0 && pending && (heads & 1u)) emit(direct, base, run.f, last_key, run.v, first - 1, run.h);
        uint32_t fh = heads ? ((uint32_t)__popc(heads) << 16) | (lane * IPT + 31u - __clz(heads)) : 0u;
        uint64_t fv = acc;
#pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1) {
          const uint32_t yfh = __shfl_up_sync(0xffffffffu, fh, o);
          const uint64_t yv = __shfl_up_sync(0xffffffffu, fv, o);
          if (lane >= o) {
            if (fh >> 16) {
              fh += yfh & 0xffff0000u;
            } else {
              fh = yfh;
              fv += yv;
            }
          }
        }
        const uint32_t tfh = __shfl_sync(0xffffffffu, fh, 31);
        const uint64_t tv = __shfl_sync(0xffffffffu, fv, 31);
        uint32_t efh = __shfl_up_sync(0xffffffffu, fh, 1);
        uint64_t ev = __shfl_up_sync(0xffffffffu, fv, 1);
        if (lane == 0) {
          efh = 0;
          ev = 0;
        }
        const uint64_t cf = run.f + (efh >> 16);
        const uint64_t cv = (efh >> 16) ? ev : run.v + ev;
        const uint64_t ch = (efh >> 16) ? tile_row + (efh & 0xffffu) : run.h;
        // run ends: the row before each head, and the last row when the next key differs
        uint32_t tails = heads >> 1;
        if (lane < 31) {
          if (key[IPT - 1] != nk) tails |= 1u << (IPT - 1);
        } else if ((tile + 1) * TR >= n) {
          tails |= 1u << (IPT - 1);                      // the relation's last row
        }
        // one round per run end of the lane with the most: each lane takes its lowest
        // remaining end (the row's key and running sum picked by compare-select)
        while (__any_sync(0xffffffffu, tails != 0)) {
          if (tails) {
            const uint32_t j = (uint32_t)__ffs(tails) - 1u;
            tails &= tails - 1u;
            Key kj = key[0];
            uint64_t rj = racc[0];
#pragma unroll
            for (uint32_t jj = 1; jj < IPT; ++jj)
              if (jj == j) {
                kj = key[jj];
                rj = racc[jj];
              }
            const uint32_t hb = heads & ((2u << j) - 1u);
            emit(direct, base, cf + (uint64_t)__popc(hb), kj, hb ? rj : cv + rj, first + j,
                 hb ? first + (31u - __clz(hb)) : ch);
          }
        }
        run.f += tfh >> 16;
        run.v = (tfh >> 16) ? tv : run.v + tv;
        run.h = (tfh >> 16) ? tile_row + (tfh & 0xffffu) : run.h;
        last_key = shfl_key(key[IPT - 1], 31);
        pending = (tile + 1) * TR < n;
        continue;
      }
      const uint32_t nvalid = first >= n ? 0u : (uint32_t)min((uint64_t)IPT, n - first);
      Key key[IPT];
      uint64_t val[IPT];
#pragma unroll
      for (uint32_t j = 0; j < IPT; ++j) {
        key[j] = 0;
        val[j] = 0;
        if (j < nvalid) RA::read(st, lane * IPT + j, ks, vs, vmask, key[j], val[j]);
      }
      Key pk = shfl_key(key[IPT - 1], lane ? lane - 1 : 0);
      const Key nk = shfl_key(key[0], lane < 31 ? lane + 1 : 31);
      if (lane == 0) pk = last_key;
      const bool next_valid = first + IPT < n;
      uint32_t heads = 0;
      uint64_t acc = 0;
#pragma unroll
      for (uint32_t j = 0; j < IPT; ++j) {
        if (j < nvalid) {
          const bool h = key[j] != (j ? key[j - 1] : pk) || (j == 0 && first == 0);
          heads |= (uint32_t)h << j;
          acc = h ? val[j] : acc + val[j];
        }
      }
      // the previous tile's last row ends its run when this tile starts a new one
      if (lane == 0 && pending && (heads & 1u)) emit(direct, base, run.f, last_key, run.v, first - 1, run.h);
      // warp segmented scan of (f, v, h)
      SegPair incl{(uint64_t)__popc(heads), acc, heads ? first + (31u - __clz(heads)) : 0ull};
#pragma unroll
      for (uint32_t o = 1; o < 32; o <<= 1) {
        SegPair y;
        y.f = __shfl_up_sync(0xffffffffu, incl.f, o);
        y.v = __shfl_up_sync(0xffffffffu, incl.v, o);
        y.h = __shfl_up_sync(0xffffffffu, incl.h, o);
        if (lane >= o) incl = seg_op(y, incl);
      }
      const SegPair wtot = shfl_seg(incl, 31);
      SegPair ex;
      ex.f = __shfl_up_sync(0xffffffffu, incl.f, 1);
      ex.v = __shfl_up_sync(0xffffffffu, incl.v, 1);
      ex.h = __shfl_up_sync(0xffffffffu, incl.h, 1);
      if (lane == 0) ex = SegPair{0, 0, 0};
      const SegPair carry = seg_op(run, ex);
      uint64_t racc = carry.v, hpos = carry.h;
#pragma unroll
      for (uint32_t j = 0; j < IPT; ++j) {
        if (j < nvalid) {
          const bool h = (heads >> j) & 1u;
          racc = h ? val[j] : racc + val[j];
          if (h) hpos = first + j;
          bool tail;
          if (j + 1 < nvalid) tail = (heads >> (j + 1)) & 1u;
          else if (j + 1 < IPT) tail = true;            // last row of the relation
          else if (!next_valid) tail = true;
          else if (lane < 31) tail = key[j] != nk;
          else tail = false;                            // decided with the next tile
          if (tail) emit(direct, base, carry.f + (uint64_t)__popc(heads & ((2u << j) - 1u)), key[j], racc, first + j, hpos);
        }
      }
      run = seg_op(run, wtot);
      last_key = shfl_key(key[IPT - 1], 31);
      pending = __shfl_sync(0xffffffffu, (uint32_t)(nvalid == IPT && next_valid), 31) != 0;
      __syncwarp();
      if (lane == 0 && i + S < ntiles) {
        fence_proxy_async_smem();
        issue(i + S);
      }
    }
    // the sub-chunk's last row: its run ends here unless the next row continues it
    if (lane == 0 && pending && ok) {
      const uint64_t nx = t1 * TR;   // first row after the sub-chunk (< n since pending)
      if (RA::global_key(a.rows, nx, ks) != last_key) emit(direct, base, run.f, last_key, run.v, nx - 1, run.h);
    }
    return run;
  };

  const SegPair wagg = run_sub(false, 0);
  const unsigned fb = __ballot_sync(0xffffffffu, has_first);
  const uint32_t src = fb ? (uint32_t)(__ffs(fb) - 1) : 0u;
  first_sum = __shfl_sync(0xffffffffu, first_sum, src);
  first_tail = __shfl_sync(0xffffffffu, first_tail, src);
  first_key = shfl_key(first_key, src);
  const bool wover = __any_sync(0xffffffffu, overflow);
  const uint32_t nloc = __reduce_max_sync(0xffffffffu, max_lf);
  if (lane == 0) s_wagg[w] = wagg;
  __syncthreads();
  if (t < 32) {
    SegPair bagg{0, 0, 0};
    for (int v = 0; v < WARPS; ++v) bagg = seg_op(bagg, s_wagg[v]);
    lb_publish(a.records, bc, bagg);
    const SegPair p = warp_lookback_resolve<4>(a.records, bc, bagg, a.err);
    if (t == 0) {
      s_pre = p;
      const uint64_t c0 = bc * WARPS * tpc;
      if (c0 < num_tiles && num_tiles <= c0 + WARPS * tpc) *a.d_groups = p.f + bagg.f;
      if (n == 0 && bc == 0) *a.d_groups = 0;
    }
  }
  __syncthreads();
  SegPair pw = s_pre;
  for (uint32_t v = 0; v < w; ++v) pw = seg_op(pw, s_wagg[v]);
  if (fb && pw.f > 0 && lane == 0) {
    const uint64_t g = pw.f - 1;
    store_key(a.out_keys, g, a.out_key_bytes, first_key);
    if (a.out_sums) a.out_sums[g] = (int64_t)(pw.v + first_sum);
    if (a.out_counts) a.out_counts[g] = (uint32_t)(first_tail - pw.h + 1);
  }
  if (wover) {
    run_sub(true, pw.f);
  } else {
    for (uint32_t l = lane; l < nloc; l += 32) {
      const uint64_t sidx = sub * ca.cap + l, g = pw.f + l;
      if (a.out_key_bytes == 4) reinterpret_cast<uint32_t*>(a.out_keys)[g] = reinterpret_cast<const uint32_t*>(ca.s_keys)[sidx];
      else if (a.out_key_bytes == 8) reinterpret_cast<uint64_t*>(a.out_keys)[g] = reinterpret_cast<const uint64_t*>(ca.s_keys)[sidx];
      else reinterpret_cast<uint4*>(a.out_keys)[g] = reinterpret_cast<const uint4*>(ca.s_keys)[sidx];
      if (a.out_sums) a.out_sums[g] = ca.s_sums[sidx];
      if (a.out_counts) a.out_counts[g] = ca.s_counts[sidx];
    }
  }
  if (!ok && lane == 0) raise_error(a.err, kErrTimeout);
}

}  // namespace rfx
