// sort_kernels.cuh -- stable LSD radix sort of packed keys (with optional values):
// one histogram pass over the keys for every digit, then one "onesweep" kernel per 8-bit
// digit that ranks a tile with warp match/ballot, publishes per-digit tile counts through
// decoupled look-back, and scatters through shared memory so that global writes go out
// in digit runs.
//
// Keys are containers of K bytes (1..64), sorted on bits [begin_bit, end_bit) as
// unsigned integers, values V bytes (0 = keys only).  The sort is stable, so it orders
// exactly like b40c's LSD sort on bits [0, key_bits) (b40cSort.cu:58-1022) and like
// moderngpu's stable merge sort when the range covers the whole key (ModernGPUSort.cu).
#pragma once

#include "rfx_device.cuh"

namespace rfx {

constexpr int kSortThreads = 256;   // the histogram pass
constexpr int kRadix = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kMaxSortPasses = 16;  // up to 128 key bits per call
constexpr int kSortLookWindow = 8;  // predecessors examined per look-back round trip

// Items per thread by the bytes moved per item: tiles of 24-48 KB (as large as 128
// registers allow without spills), so the per-tile fixed costs (barriers, the look-back)
// are spread over enough keys.
template <int K, int V>
struct SortTuning {
  static constexpr int B = K + V;
  // a digit pass: 8 warps per block for elements up to 8 bytes, 12 above (two blocks per SM
  // either way; the larger elements' passes gain from the extra warps, the smaller lose)
  static constexpr int THREADS = B <= 8 ? 256 : 384;
  static constexpr int WARPS = THREADS / 32;
  static constexpr int IPT = B <= 4 ? 24 : B <= 8 ? 20 : B <= 16 ? 8 : B <= 32 ? 5 : B <= 64 ? 3 : 1;
  static constexpr int TILE = THREADS * IPT;
  static constexpr int SBYTES = (K > V ? K : V);
};

// A K-byte element as 32-bit words (1- and 2-byte elements zero-extended into w[0]).
template <int B>
struct Elem {
  static constexpr int NW = B <= 4 ? 1 : B / 4;
  uint32_t w[NW];
};

template <int B>
__device__ __forceinline__ Elem<B> load_elem(const uint8_t* base, uint64_t i) {
  Elem<B> e;
  if constexpr (B == 1) {
    e.w[0] = base[i];
  } else if constexpr (B == 2) {
    e.w[0] = reinterpret_cast<const uint16_t*>(base)[i];
  } else if constexpr (B == 4) {
    e.w[0] = reinterpret_cast<const uint32_t*>(base)[i];
  } else if constexpr (B == 8) {
    uint2 v = reinterpret_cast<const uint2*>(base)[i];
    e.w[0] = v.x;
    e.w[1] = v.y;
  } else {
    const uint4* p = reinterpret_cast<const uint4*>(base + i * B);
#pragma unroll
    for (int k = 0; k < B / 16; ++k) {
      uint4 v = p[k];
      e.w[4 * k] = v.x;
      e.w[4 * k + 1] = v.y;
      e.w[4 * k + 2] = v.z;
      e.w[4 * k + 3] = v.w;
    }
  }
  return e;
}

template <int B>
__device__ __forceinline__ void store_elem(uint8_t* base, uint64_t i, const Elem<B>& e) {
  if constexpr (B == 1) {
    base[i] = (uint8_t)e.w[0];
  } else if constexpr (B == 2) {
    reinterpret_cast<uint16_t*>(base)[i] = (uint16_t)e.w[0];
  } else if constexpr (B == 4) {
    reinterpret_cast<uint32_t*>(base)[i] = e.w[0];
  } else if constexpr (B == 8) {
    reinterpret_cast<uint2*>(base)[i] = make_uint2(e.w[0], e.w[1]);
  } else {
    uint4* p = reinterpret_cast<uint4*>(base + i * B);
#pragma unroll
    for (int k = 0; k < B / 16; ++k) p[k] = make_uint4(e.w[4 * k], e.w[4 * k + 1], e.w[4 * k + 2], e.w[4 * k + 3]);
  }
}

// Bits [shift, shift + 8) of the element (the caller masks to the digit width).
template <int K>
__device__ __forceinline__ uint32_t elem_bits(const Elem<K>& e, uint32_t shift) {
  if constexpr (Elem<K>::NW == 1) {
    return e.w[0] >> shift;
  } else {
    const uint32_t q = shift >> 5;
    uint32_t lo = e.w[0], hi = e.w[1];
#pragma unroll
    for (int k = 1; k < Elem<K>::NW; ++k) {
      if ((int)q == k) {
        lo = e.w[k];
        hi = k + 1 < Elem<K>::NW ? e.w[k + 1] : 0u;
      }
    }
    return __funnelshift_r(lo, hi, shift & 31);
  }
}

struct SortPassArgs {
  const uint8_t* keys_in;
  uint8_t* keys_out;
  const uint8_t* vals_in;
  uint8_t* vals_out;
  uint64_t n;
  uint32_t shift;       // first bit of this digit
  uint32_t mask;        // digit mask (0xff, or fewer bits for the last digit)
  const uint32_t* gexcl;  // exclusive global digit offsets of this pass [256]
  uint32_t* status;     // [tiles][256] look-back words of this pass
  uint32_t* tile_counter;
  uint32_t* err;
};

// 32-bit look-back words: bits 31..30 flag (1 aggregate, 2 inclusive), 29..0 value.
constexpr uint32_t kSFlagAgg = 1u << 30;
constexpr uint32_t kSFlagInc = 2u << 30;
constexpr uint32_t kSValMask = (1u << 30) - 1;

__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint4 ld_volatile_v4(const uint32_t* p) {
  uint4 v;
  asm volatile("ld.volatile.global.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p)
               : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ------------------------------------------------------------------ histogram
// Counts every pass's digits in one read of the keys (warp-aggregated shared atomics),
// then the last block turns the counts into exclusive offsets and flags trivial passes.
template <int K>
__global__ void __launch_bounds__(kSortThreads)
sort_histogram_kernel(const uint8_t* __restrict__ keys, uint64_t n, uint32_t begin_bit, uint32_t end_bit,
                      uint32_t passes, uint32_t* __restrict__ ghist, uint32_t* __restrict__ trivial,
                      uint32_t* __restrict__ done_counter) {
  __shared__ uint32_t h[kMaxSortPasses][kRadix];
  __shared__ bool s_last;
  const uint32_t t = threadIdx.x, lane = t & 31;
  for (uint32_t k = t; k < passes * kRadix; k += kSortThreads) (&h[0][0])[k] = 0;
  __syncthreads();
  // R elements per thread per iteration, all loaded before any is counted (a read-only
  // stream needs several loads in flight per thread to approach HBM bandwidth)
  constexpr int R = K <= 16 ? 4 : 2;
  const uint64_t stride = (uint64_t)gridDim.x * kSortThreads;
  const uint64_t nround = (n + R * stride - 1) / (R * stride) * (R * stride);  // warps stay converged
  for (uint64_t i0 = (uint64_t)blockIdx.x * kSortThreads + t; i0 < nround; i0 += R * stride) {
    Elem<K> e[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const uint64_t i = i0 + (uint64_t)r * stride;
      if (i < n) e[r] = load_elem<K>(keys, i);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const bool valid = i0 + (uint64_t)r * stride < n;
      const unsigned vmask = __ballot_sync(0xffffffffu, valid);
      for (uint32_t p = 0; p < passes; ++p) {
        const uint32_t shift = begin_bit + 8 * p;
        const uint32_t w = end_bit - shift < 8 ? end_bit - shift : 8;
        const uint32_t d = valid ? (elem_bits<K>(e[r], shift) & ((1u << w) - 1)) : kRadix;
        // a digit shared by the whole warp (constant high digits) is one add, not 32
        // conflicting atomics; otherwise plain shared atomics
        const uint32_t d0 = __shfl_sync(0xffffffffu, d, 0);
        if (__all_sync(0xffffffffu, d == d0 || !valid) && vmask == 0xffffffffu) {
          if (lane == 0) atomicAdd(&h[p][d0], 32u);
        } else if (valid) {
          atomicAdd(&h[p][d], 1u);
        }
      }
    }
  }
  __syncthreads();
  for (uint32_t k = t; k < passes * kRadix; k += kSortThreads) {
    const uint32_t c = (&h[0][0])[k];
    if (c) atomicAdd(&ghist[k], c);
  }
  __threadfence();
  __syncthreads();
  if (t == 0) s_last = atomicAdd(done_counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // exclusive scan per pass (one warp per pass)
  const uint32_t warp = t >> 5;
  for (uint32_t p = warp; p < passes; p += kSortWarps) {
    uint32_t run = 0, maxc = 0;
    for (uint32_t d0 = 0; d0 < kRadix; d0 += 32) {
      const uint32_t c = atomicAdd(&ghist[p * kRadix + d0 + lane], 0u);
      maxc = max(maxc, c);
      uint32_t incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += v;
      }
      ghist[p * kRadix + d0 + lane] = run + incl - c;
      run += __shfl_sync(0xffffffffu, incl, 31);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) maxc = max(maxc, __shfl_xor_sync(0xffffffffu, maxc, o));
    if (lane == 0) trivial[p] = (uint64_t)maxc == n ? 1u : 0u;
  }
}

// ------------------------------------------------------------------ per-tile pass
// Two blocks per SM: the per-item keys and ranks must fit 128 registers, so digits and
// tile positions are recomputed where needed instead of being kept live.
//
// A block claims its next tile one ahead and, where the keys are 16-byte aligned and two
// tile buffers fit, copies that tile's keys into shared memory with cp.async while it
// ranks, resolves and writes the current one, so the load of a tile never waits on the
// memory system.  Per tile: rank in registers, count digits and publish the tile's
// aggregate, scatter the keys into the tile's own buffer in digit order, resolve the
// global digit offsets by decoupled look-back (after the scatter, so the predecessors
// have had that long to publish), then write the buffer out in digit runs.
template <int K, int V>
struct SortBuffers {
  static constexpr int EB = (int)sizeof(Elem<K>) > (V > 0 ? (int)sizeof(Elem<V>) : 0) ? (int)sizeof(Elem<K>)
                                                                                        : (int)sizeof(Elem<V>);
  static constexpr int TILE = SortTuning<K, V>::TILE;
  // prefetch when the raw keys are whole 16-byte chunks and two buffers fit two blocks
  static constexpr bool PF = K >= 4 && 2 * TILE * EB <= 100 * 1024;
  static constexpr size_t SMEM = (size_t)(PF ? 2 : 1) * TILE * EB;
};

// The raw keys of tile `tile` (tcount keys) into `dst`, in 16-byte chunks (the last one
// zero-filled past the array).
template <int K>
__device__ __forceinline__ void sort_prefetch(uint8_t* dst, const uint8_t* keys, uint64_t tile, uint32_t tile_keys,
                                              uint64_t n, uint32_t nthreads) {
  block_prefetch16(dst, keys, tile * (uint64_t)tile_keys * K, (uint64_t)tile_keys * K, n * K, nthreads);
}

// The lanes of a warp whose digit equals this lane's (within `valid`): the intersection
// over the digit's bits of the ballot of lanes sharing that bit (lop3-friendly form), or
// the hardware match.
template <bool MATCH>
__device__ __forceinline__ unsigned digit_peers(uint32_t d, bool valid, uint32_t bits) {
  if constexpr (MATCH) {
    const unsigned m = __match_any_sync(0xffffffffu, valid ? d : 0xffffffffu);
    return valid ? m : 0u;
  } else {
    unsigned peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      if ((uint32_t)b < bits) {
        const unsigned bb = __ballot_sync(0xffffffffu, (d >> b) & 1u);
        const unsigned mb = 0u - ((d >> b) & 1u);   // all ones where this lane's bit is set
        peers &= ~(bb ^ mb);
      }
    }
    return peers;
  }
}

template <int K, int V, bool MATCH = false>
__global__ void __launch_bounds__((SortTuning<K, V>::THREADS), 2)
sort_pass_kernel(const SortPassArgs a) {
  using T = SortTuning<K, V>;
  using SB = SortBuffers<K, V>;
  constexpr int IPT = T::IPT;
  constexpr int TILE = T::TILE;
  extern __shared__ __align__(16) uint8_t sbuf[];              // 1 or 2 buffers of TILE * EB
  __shared__ uint16_t whist[T::WARPS][kRadix];               // per-warp digit counts (a tile's fit 16 bits)
  __shared__ uint32_t s_local[kRadix];                         // tile-local digit start
  __shared__ unsigned long long s_gb[kRadix];                  // output index of slot i = s_gb[digit] + i
  __shared__ uint8_t s_dig[TILE];                              // digit of each sorted slot
  __shared__ uint32_t s_scan[T::WARPS];
  __shared__ uint32_t s_tile[2];
  const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const uint64_t num_tiles = (a.n + TILE - 1) / TILE;
  const bool pf = SB::PF && (reinterpret_cast<uintptr_t>(a.keys_in) & 15u) == 0;
  const uint32_t dbits = 32 - __clz(a.mask);   // bits in this pass's digit (ballots needed)
  if (t == 0) s_tile[0] = atomicAdd(a.tile_counter, 1u);
  __syncthreads();
  if (pf && s_tile[0] < num_tiles) sort_prefetch<K>(sbuf, a.keys_in, s_tile[0], TILE, a.n, T::THREADS);
  cp_async_commit();

  for (uint32_t it = 0;; ++it) {
    const uint64_t tile = s_tile[it & 1];
    uint8_t* stage = sbuf + (pf ? (size_t)(it & 1) * TILE * SB::EB : 0);
    if (t == 0) s_tile[(it + 1) & 1] = atomicAdd(a.tile_counter, 1u);   // the next tile, one ahead
    for (uint32_t k = t; k < T::WARPS * kRadix / 2; k += T::THREADS) reinterpret_cast<uint32_t*>(&whist[0][0])[k] = 0;
    __syncthreads();
    if (tile >= num_tiles) break;   // the tile claimed next is larger still: no copy in flight
    const uint64_t next = s_tile[(it + 1) & 1];
    if (pf) {
      if (next < num_tiles) sort_prefetch<K>(sbuf + (size_t)((it + 1) & 1) * TILE * SB::EB, a.keys_in, next, TILE, a.n, T::THREADS);
      cp_async_commit();
      cp_async_wait<1>();          // this tile's copy (the next one may stay in flight)
      __syncthreads();
    }
    const uint64_t tbase = tile * TILE;
    const uint32_t tcount = (uint32_t)min((uint64_t)TILE, a.n - tbase);
    // warp w owns items [w*32*IPT, (w+1)*32*IPT) of the tile, item j of lane l at j*32+l
    const uint32_t wbase = warp * 32 * IPT;
    Elem<K> key[IPT];
    uint32_t rank[IPT];
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
      const uint32_t li = wbase + j * 32 + lane;
      if (li < tcount) key[j] = pf ? load_elem<K>(stage, li) : load_elem<K>(a.keys_in, tbase + li);
    }
    // the lanes of a warp whose key has this lane's digit: every key's bit goes into its
    // digit's mask with one shared-memory atomic OR (the warp's 256 masks sit in the tile
    // buffer, which is free from here until the scatter: every key is in registers), or the
    // hardware match in the MATCH variant
    uint32_t* s_peer = reinterpret_cast<uint32_t*>(stage) + warp * kRadix;
    if constexpr (!MATCH) {
      __syncthreads();   // all warps hold their keys
      for (uint32_t k = lane; k < kRadix; k += 32) s_peer[k] = 0u;
      __syncwarp();
    }
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
      const uint32_t li = wbase + j * 32 + lane;
      const bool valid = li < tcount;
      const uint32_t d = valid ? (elem_bits<K>(key[j], a.shift) & a.mask) : 0u;
      unsigned peers;
      if constexpr (MATCH) {
        peers = digit_peers<true>(d, valid, dbits);
      } else {
        if (valid) atomicOr(&s_peer[d], 1u << lane);
        __syncwarp();
        peers = valid ? s_peer[d] : 0u;
      }
      const unsigned lower = peers & ((1u << lane) - 1);
      uint32_t base = 0;
      if (valid) base = whist[warp][d];
      rank[j] = (base + __popc(lower)) | (d << 16);   // the digit rides along: extracted once
      __syncwarp();
      if (valid && lower == 0) {
        whist[warp][d] = (uint16_t)(base + __popc(peers));
        if constexpr (!MATCH) s_peer[d] = 0u;   // cleared for the next key by its group's first lane
      }
      __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive over warps, the tile's count (published at once), tile-local start
    uint32_t count = 0;
    if (t < kRadix) {
#pragma unroll
      for (int w = 0; w < T::WARPS; ++w) {
        const uint32_t c = whist[w][t];
        whist[w][t] = (uint16_t)count;
        count += c;
      }
      st_relaxed_u32(a.status + tile * kRadix + t, (tile == 0 ? kSFlagInc : kSFlagAgg) | count);
    }
    // block exclusive scan of count over the 256 digits
    uint32_t incl = count;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o) incl += v;
    }
    if (lane == 31) s_scan[warp] = incl;
    __syncthreads();
    if (t < kRadix) {
      uint32_t wpre = 0;
      for (uint32_t w = 0; w < warp; ++w) wpre += s_scan[w];
      s_local[t] = wpre + incl - count;
    }
    __syncthreads();
    // keys: scatter into tile order in shared memory (every thread's keys are in registers),
    // each slot's digit beside it
    Elem<K>* skeys = reinterpret_cast<Elem<K>*>(stage);
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
      const uint32_t li = wbase + j * 32 + lane;
      if (li < tcount) {
        const uint32_t d = rank[j] >> 16;
        const uint32_t slot = s_local[d] + whist[warp][d] + (rank[j] & 0xffffu);
        skeys[slot] = key[j];
        s_dig[slot] = (uint8_t)d;
      }
    }
    // decoupled look-back for digit t, kSortLookWindow predecessors per round trip
    // (independent loads, all in flight at once)
    if (t < kRadix) {
      uint32_t prefix = 0;
      if (tile > 0) {
        int64_t base = (int64_t)tile - 1;
        uint32_t spins = 0;
        while (base >= 0) {
          uint32_t w[kSortLookWindow];
          // predecessor base - r sits r * kRadix words below base's word: constant offsets
          // from one pointer (a window reaching past tile 0 reads "inclusive 0" there)
          const uint32_t* pb = a.status + (uint64_t)base * kRadix + t;
          if (base >= kSortLookWindow - 1) {
#pragma unroll
            for (int r = 0; r < kSortLookWindow; ++r) w[r] = ld_relaxed_u32(pb - r * kRadix);
          } else {
#pragma unroll
            for (int r = 0; r < kSortLookWindow; ++r) w[r] = r <= base ? ld_relaxed_u32(pb - r * kRadix) : kSFlagInc;
          }
          int r_inc = kSortLookWindow;
#pragma unroll
          for (int r = kSortLookWindow - 1; r >= 0; --r)
            if (w[r] & kSFlagInc) r_inc = r;
          bool busy = false;
          uint32_t sum = 0;
#pragma unroll
          for (int r = 0; r < kSortLookWindow; ++r) {
            if (r <= r_inc) {
              busy = busy || (w[r] & ~kSValMask) == 0;
              sum += w[r] & kSValMask;
            }
          }
          if (busy) {
            if (++spins > kSpinLimit) {
              raise_error(a.err, kErrTimeout);
              break;
            }
            __nanosleep(spins < 16 ? 32 : 128);
            continue;
          }
          prefix += sum;
          if (r_inc < kSortLookWindow) break;
          base -= kSortLookWindow;
        }
        st_relaxed_u32(a.status + tile * kRadix + t, kSFlagInc | ((prefix + count) & kSValMask));
      }
      // (global start of the digit's run) - (its tile-local start), modulo 2^64
      s_gb[t] = (unsigned long long)a.gexcl[t] + prefix - s_local[t];
    }
    __syncthreads();
    for (uint32_t i = t; i < tcount; i += T::THREADS) {
      const uint64_t pos = s_gb[s_dig[i]] + i;
      if (pos < a.n) store_elem<K>(a.keys_out, pos, skeys[i]);
    }
    if constexpr (V > 0) {
      __syncthreads();
      Elem<V>* svals = reinterpret_cast<Elem<V>*>(stage);
#pragma unroll
      for (int j = 0; j < IPT; ++j) {
        const uint32_t li = wbase + j * 32 + lane;
        if (li < tcount) {
          const uint32_t d = rank[j] >> 16;
          svals[s_local[d] + whist[warp][d] + (rank[j] & 0xffffu)] = load_elem<V>(a.vals_in, tbase + li);
        }
      }
      __syncthreads();
      for (uint32_t i = t; i < tcount; i += T::THREADS) {
        const uint64_t pos = s_gb[s_dig[i]] + i;
        if (pos < a.n) store_elem<V>(a.vals_out, pos, svals[i]);
      }
    }
    __syncthreads();
  }
  cp_async_wait<0>();
}

}  // namespace rfx
