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

#include "rfx_device.cuh"
#include "search.cuh"
#include "sort_kernels.cuh"

namespace rfx {

constexpr int kRedThreads = 256;
constexpr int kRedIPT = 8;
constexpr int kRedTile = kRedThreads * kRedIPT;

enum ValKind : int { VAL_NONE = 0, VAL_U32 = 1, VAL_I64 = 2 };

struct SegPair {
  uint64_t f;  // heads
  uint64_t v;  // running total since the last head (u64 arithmetic, wraps)
  uint64_t h;  // position of the last head (max); a run's length at its last item i is i - h + 1
};

__device__ __forceinline__ SegPair seg_op(const SegPair& a, const SegPair& b) {
  return SegPair{a.f + b.f, b.f ? b.v : a.v + b.v, a.h > b.h ? a.h : b.h};
}

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

}  // namespace rfx
