// sort_onesweep.cuh -- the pipelined onesweep pass of the LSD radix sort (keys without
// separate values, 4 / 8 / 16-byte containers, 16-byte aligned buffers).
//
// One block per SM: eight compute warps and one look-back warp.  Tiles are claimed from a
// device counter in order and move through three shared-memory stages:
//
//   TMA      a 1-D bulk copy (cp.async.bulk, this GPU's memory only) brings tile i+2 into
//            a free stage while tile i is being worked on;
//   rank     the compute warps read tile i from its stage, rank every key within its
//            warp by digit (eight bit ballots) and count digits per warp;
//   count    per digit: the tile's count (published at once as the tile's aggregate for
//            the decoupled look-back) and its tile-local start;
//   look-back  the look-back warp resolves tile i's global digit offsets -- a window of
//            predecessors per round trip, each lane owning 8 digits -- while the compute
//            warps write tile i-1 out and rank tile i+1;
//   write    the compute warps scatter tile i into its own stage in digit order and, one
//            tile later, copy the stage to the output in digit runs.
//
// The look-back of a tile therefore overlaps the next tile's ranking, and the loads of
// the next two tiles are in flight the whole time, so HBM sees a continuous stream in
// both directions.  Hand-offs between the compute warps and the look-back warp are named
// barriers (bar.arrive / bar.sync), alternating by tile parity so that a fast side can
// never arrive twice at a barrier the other side has not passed.  Every wait is bounded:
// a stage that never fills or a predecessor that never publishes records kErrTimeout in
// the error word and the pass carries on (output unspecified, stores stay in bounds).
#pragma once

#include "sort_kernels.cuh"
#include "tile_ring.cuh"

namespace rfx {

constexpr int kOsCompute = 256;                 // 8 compute warps
constexpr int kOsThreads = kOsCompute + 32;     // + the look-back warp
constexpr int kOsStages = 3;
constexpr int kOsWindow = 16;                   // predecessors per look-back round trip

// Items per thread: the default and two tuner alternatives -- tiles of 48 / 32 / 64 KB for
// 16-byte keys, 48 / 32 / 40 KB for 8-byte keys, 32 / 16 / 24 KB for 4-byte keys (the
// look-back warp's window holds 128 registers, and every thread of the block gets the
// same allocation, so larger 8- and 4-byte tiles would spill).
template <int K>
struct OsIpt {
  static constexpr int DEF = K == 16 ? 12 : K == 8 ? 24 : 32;
  static constexpr int SMALL = K == 16 ? 8 : K == 8 ? 16 : 16;
  static constexpr int ALT = K == 16 ? 16 : K == 8 ? 20 : 24;
};

template <int K, int IPT_ = OsIpt<K>::DEF>
struct OsTuning {
  static constexpr int IPT = IPT_;
  static constexpr int TILE = kOsCompute * IPT;
  static constexpr uint32_t TILE_BYTES = (uint32_t)TILE * K;
  static constexpr size_t SMEM = (size_t)kOsStages * TILE_BYTES;
};

// Named barriers (0 is __syncthreads): the compute warps among themselves, and the two
// parities of "tile counted, look-back may start" / "look-back done".
constexpr int kBarCompute = 1;
constexpr int kBarGo0 = 2;
constexpr int kBarDone0 = 4;

__device__ __forceinline__ void nbar_sync(int id, int n) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}
__device__ __forceinline__ void nbar_arrive(int id, int n) {
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(n) : "memory");
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ uint4 ld_relaxed_v4(const uint32_t* p) {
  uint4 v;
  asm volatile("ld.relaxed.gpu.global.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p)
               : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_v4(uint32_t* p, uint4 v) {
  asm volatile("st.relaxed.gpu.global.v4.u32 [%0], {%1, %2, %3, %4};" ::"l"(p), "r"(v.x), "r"(v.y), "r"(v.z),
               "r"(v.w)
               : "memory");
}

__device__ __forceinline__ uint32_t v4_get(const uint4& v, int j) {
  return j == 0 ? v.x : j == 1 ? v.y : j == 2 ? v.z : v.w;
}

// The look-back of one tile by one warp: lane l owns digits 8l .. 8l+7.  Returns the
// exclusive prefixes in pre[] and publishes the tile's inclusive values.
__device__ __forceinline__ void os_lookback(uint32_t* status, uint64_t tile, const uint32_t cnt[8], uint32_t pre[8],
                                            uint32_t* err) {
  const uint32_t lane = threadIdx.x & 31;
#pragma unroll
  for (int j = 0; j < 8; ++j) pre[j] = 0;
  if (tile == 0) return;  // tile 0 published its counts as inclusive values
  uint32_t notdone = 0xffu;   // digits whose prefix is still open
  int64_t base = (int64_t)tile - 1;
  uint32_t spins = 0;
  while (__any_sync(0xffffffffu, notdone != 0)) {
    uint4 w[kOsWindow][2];
#pragma unroll
    for (int r = 0; r < kOsWindow; ++r) {
      const int64_t idx = base - r;
      if (idx >= 0) {
        const uint32_t* p = status + (uint64_t)idx * kRadix + 8 * lane;
        w[r][0] = ld_relaxed_v4(p);
        w[r][1] = ld_relaxed_v4(p + 4);
      } else {
        w[r][0] = make_uint4(kSFlagInc, kSFlagInc, kSFlagInc, kSFlagInc);
        w[r][1] = w[r][0];
      }
    }
    // per open digit: the values from the nearest predecessor back to (and including) the
    // first inclusive one; a predecessor that has published nothing yet means "retry"
    bool busy = false;
    uint32_t add[8];
    uint32_t fin = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      uint32_t sum = 0;
      bool stopped = false;
#pragma unroll
      for (int r = 0; r < kOsWindow; ++r) {
        const uint32_t v = v4_get(w[r][j >> 2], j & 3);
        if (!stopped) {
          busy = busy || (((notdone >> j) & 1u) && (v & ~kSValMask) == 0);
          sum += v & kSValMask;
          stopped = (v & kSFlagInc) != 0;
        }
      }
      add[j] = sum;
      if (stopped) fin |= 1u << j;
    }
    if (__any_sync(0xffffffffu, busy)) {
      if (++spins > kSpinLimit) {
        raise_error(err, kErrTimeout);
        break;
      }
      __nanosleep(spins < 8 ? 20 : 100);
      continue;
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if ((notdone >> j) & 1u) pre[j] += add[j];
    notdone &= ~fin;
    base -= kOsWindow;
  }
  uint32_t* st = status + tile * kRadix + 8 * lane;
  st_relaxed_v4(st, make_uint4(kSFlagInc | ((pre[0] + cnt[0]) & kSValMask), kSFlagInc | ((pre[1] + cnt[1]) & kSValMask),
                               kSFlagInc | ((pre[2] + cnt[2]) & kSValMask), kSFlagInc | ((pre[3] + cnt[3]) & kSValMask)));
  st_relaxed_v4(st + 4,
                make_uint4(kSFlagInc | ((pre[4] + cnt[4]) & kSValMask), kSFlagInc | ((pre[5] + cnt[5]) & kSValMask),
                           kSFlagInc | ((pre[6] + cnt[6]) & kSValMask), kSFlagInc | ((pre[7] + cnt[7]) & kSValMask)));
}

struct OsShared {
  uint32_t whist[kSortWarps][kRadix];   // per-warp digit counts, then exclusive over warps
  uint32_t count[2][kRadix];            // the tile's digit counts (by tile parity)
  uint32_t local[2][kRadix];            // tile-local digit starts
  uint64_t gbase[2][kRadix];            // output index of a stage slot = gbase[d] + slot
  uint32_t scan[kSortWarps];
  uint32_t tile[kOsStages];
  uint64_t bar[kOsStages];
};

template <int K, int IPT_>
__global__ void __launch_bounds__(kOsThreads, 1) sort_onesweep_kernel(const SortPassArgs a) {
  using T = OsTuning<K, IPT_>;
  constexpr int IPT = T::IPT;
  constexpr int TILE = T::TILE;
  extern __shared__ __align__(128) uint8_t os_stage[];   // kOsStages x TILE_BYTES
  __shared__ OsShared S;
  const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const uint64_t num_tiles = (a.n + TILE - 1) / TILE;
  const bool has_tail = (a.n % TILE) != 0;
  auto stage = [&](int b) { return os_stage + (size_t)b * T::TILE_BYTES; };
  auto is_tma_tile = [&](uint64_t tile) { return tile < num_tiles && !(has_tail && tile == num_tiles - 1); };

  // prologue: claim the first three tiles and start their copies
  if (t == 0) {
    for (int b = 0; b < kOsStages; ++b) mbar_init(&S.bar[b], 1);
    mbar_fence_init();
    for (int b = 0; b < kOsStages; ++b) {
      const uint32_t tile = atomicAdd(a.tile_counter, 1u);
      S.tile[b] = tile;
      if (is_tma_tile(tile)) {
        mbar_arrive_tx(&S.bar[b], T::TILE_BYTES);
        bulk_load(stage(b), a.keys_in + (uint64_t)tile * T::TILE_BYTES, T::TILE_BYTES, &S.bar[b]);
      }
    }
  }
  __syncthreads();

  if (warp == kSortWarps) {
    // ---------------------------------------------------------------- look-back warp
    uint32_t gex[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) gex[j] = a.gexcl[8 * lane + j];
    for (uint32_t i = 0;; ++i) {
      const int p = i & 1;
      nbar_sync(kBarGo0 + p, kOsThreads);
      const uint64_t tile = S.tile[i % kOsStages];
      if (tile >= num_tiles) break;
      uint32_t cnt[8], pre[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) cnt[j] = S.count[p][8 * lane + j];
      os_lookback(a.status, tile, cnt, pre, a.err);
#pragma unroll
      for (int j = 0; j < 8; ++j)
        S.gbase[p][8 * lane + j] = (uint64_t)gex[j] + pre[j] - S.local[p][8 * lane + j];
      nbar_arrive(kBarDone0 + p, kOsThreads);
    }
    return;
  }

  // ------------------------------------------------------------------ compute warps
  uint32_t phase = 0;           // bit b: parity of the next fill of stage b
  uint32_t prev_count = 0;      // keys in tile i-1
  const uint32_t wbase = warp * 32 * IPT;
  for (uint32_t i = 0;; ++i) {
    const int b = i % kOsStages;
    const int p = i & 1;
    const uint64_t tile = S.tile[b];
    if (tile >= num_tiles) {
      nbar_arrive(kBarGo0 + p, kOsThreads);            // lets the look-back warp stop
      if (i > 0) {
        nbar_sync(kBarDone0 + (p ^ 1), kOsThreads);
        const int bp = (i + kOsStages - 1) % kOsStages;
        const Elem<K>* src = reinterpret_cast<const Elem<K>*>(stage(bp));
        for (uint32_t x = t; x < prev_count; x += kOsCompute) {
          const Elem<K> k = src[x];
          const uint64_t pos = S.gbase[p ^ 1][elem_bits<K>(k, a.shift) & a.mask] + x;
          if (pos < a.n) store_elem<K>(a.keys_out, pos, k);
        }
      }
      break;
    }
    const uint64_t tbase = tile * TILE;
    const uint32_t tcount = (uint32_t)min((uint64_t)TILE, a.n - tbase);
    const bool tma = is_tma_tile(tile);
    // ---- rank tile i
#pragma unroll
    for (int j = 0; j < 8; ++j) S.whist[warp][8 * lane + j] = 0;
    if (tma) {
      if (!mbar_wait(&S.bar[b], (phase >> b) & 1u)) raise_error(a.err, kErrTimeout);
      phase ^= 1u << b;
    }
    __syncwarp();
    Elem<K> key[IPT];
    uint32_t rk[IPT];   // rank within the warp | digit << 16
    const Elem<K>* sk = reinterpret_cast<const Elem<K>*>(stage(b));
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
      const uint32_t li = wbase + j * 32 + lane;
      if (li < tcount) key[j] = tma ? sk[li] : load_elem<K>(a.keys_in, tbase + li);
    }
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
      const uint32_t li = wbase + j * 32 + lane;
      const bool valid = li < tcount;
      const uint32_t d = valid ? (elem_bits<K>(key[j], a.shift) & a.mask) : 0u;
      unsigned peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
      for (int bit = 0; bit < 8; ++bit) {
        const unsigned bb = __ballot_sync(0xffffffffu, (d >> bit) & 1u);
        peers &= ((d >> bit) & 1u) ? bb : ~bb;
      }
      const unsigned lower = peers & ((1u << lane) - 1);
      uint32_t base = 0;
      if (valid) base = S.whist[warp][d];
      rk[j] = (base + __popc(lower)) | (d << 16);
      __syncwarp();
      if (valid && lower == 0) S.whist[warp][d] = base + __popc(peers);
      __syncwarp();
    }
    nbar_sync(kBarCompute, kOsCompute);
    // ---- count: digit t of tile i
    {
      uint32_t count = 0;
#pragma unroll
      for (int w = 0; w < kSortWarps; ++w) {
        const uint32_t c = S.whist[w][t];
        S.whist[w][t] = count;
        count += c;
      }
      st_relaxed_u32(a.status + tile * kRadix + t, (tile == 0 ? kSFlagInc : kSFlagAgg) | count);
      S.count[p][t] = count;
      uint32_t incl = count;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += v;
      }
      if (lane == 31) S.scan[warp] = incl;
      nbar_sync(kBarCompute, kOsCompute);
      uint32_t wpre = 0;
      for (uint32_t w = 0; w < warp; ++w) wpre += S.scan[w];
      S.local[p][t] = wpre + incl - count;
    }
    nbar_sync(kBarCompute, kOsCompute);
    nbar_arrive(kBarGo0 + p, kOsThreads);               // tile i: look-back may start
    // ---- write tile i-1 out (its look-back ran while tile i was ranked)
    if (i > 0) {
      nbar_sync(kBarDone0 + (p ^ 1), kOsThreads);
      const int bp = (i + kOsStages - 1) % kOsStages;
      const Elem<K>* src = reinterpret_cast<const Elem<K>*>(stage(bp));
      for (uint32_t x = t; x < prev_count; x += kOsCompute) {
        const Elem<K> k = src[x];
        const uint64_t pos = S.gbase[p ^ 1][elem_bits<K>(k, a.shift) & a.mask] + x;
        if (pos < a.n) store_elem<K>(a.keys_out, pos, k);
      }
      nbar_sync(kBarCompute, kOsCompute);
      // stage of tile i-1 is free: claim tile i+2 and start its copy there
      if (t == 0) {
        const uint32_t nt = atomicAdd(a.tile_counter, 1u);
        S.tile[bp] = nt;
        if (is_tma_tile(nt)) {
          fence_proxy_async_smem();
          mbar_arrive_tx(&S.bar[bp], T::TILE_BYTES);
          bulk_load(stage(bp), a.keys_in + (uint64_t)nt * T::TILE_BYTES, T::TILE_BYTES, &S.bar[bp]);
        }
      }
    }
    // ---- scatter tile i into its own stage in digit order
    {
      Elem<K>* dst = reinterpret_cast<Elem<K>*>(stage(b));
#pragma unroll
      for (int j = 0; j < IPT; ++j) {
        const uint32_t li = wbase + j * 32 + lane;
        if (li < tcount) {
          const uint32_t d = rk[j] >> 16;
          const uint32_t slot = S.local[p][d] + S.whist[warp][d] + (rk[j] & 0xffffu);
          if (slot < (uint32_t)TILE) dst[slot] = key[j];
        }
      }
    }
    prev_count = tcount;
    nbar_sync(kBarCompute, kOsCompute);
  }
}

}  // namespace rfx
