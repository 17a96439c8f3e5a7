// lookback.cuh -- block-wide decoupled look-back.
//
// Every tile publishes its aggregate, then its inclusive prefix, in a status record of
// 64-bit words, each carrying the 2-bit state (1 aggregate, 2 inclusive) in its top
// bits, so that a record is read consistently word by word without fences: a record is
// usable only when all its words carry the same state.  The whole block examines
// predecessors, one per thread (a window of blockDim.x tiles per round trip), stops at
// the nearest inclusive one, and folds the window in sequence order.  With many tiles in
// flight the nearest inclusive predecessor can lie hundreds of tiles back; a window as
// wide as the block reaches it in one or two round trips where a warp-wide walk would
// need one per 32 tiles.  Waits are bounded (kSpinLimit) and record kErrTimeout.
#pragma once

#include "rfx_device.cuh"

namespace rfx {

__device__ __forceinline__ void st_relaxed_v2(uint64_t* p, uint64_t a, uint64_t b) {
  asm volatile("st.relaxed.gpu.global.v2.u64 [%0], {%1, %2};" ::"l"(p), "l"(a), "l"(b) : "memory");
}
__device__ __forceinline__ void ld_relaxed_v2(const uint64_t* p, uint64_t& a, uint64_t& b) {
  asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "l"(p) : "memory");
}

// ---- payloads: identity, combine(older, newer), record layout
struct CountPayload {           // plain sums (compaction offsets)
  uint64_t c;
};
struct CountRecord {
  uint64_t w;
};
__device__ __forceinline__ CountPayload lb_identity(CountPayload) { return CountPayload{0}; }
__device__ __forceinline__ CountPayload lb_combine(const CountPayload& o, const CountPayload& n) {
  return CountPayload{o.c + n.c};
}
__device__ __forceinline__ void lb_store(CountRecord* r, uint64_t flag, const CountPayload& x) {
  st_relaxed_u64(&r->w, flag | (x.c & kValMask));
}
__device__ __forceinline__ uint64_t lb_load(const CountRecord* r, CountPayload& x) {
  const uint64_t w = ld_relaxed_u64(&r->w);
  x.c = w & kValMask;
  return w & ~kValMask;
}

// Segmented-sum pair: f = run heads, v = total since the last head (wraps mod 2^64),
// h = position of the last head.
struct SegPayload {
  uint64_t f, v, h;
};
struct __align__(32) SegRecord {
  uint64_t w[4];   // f, h, v low 32 bits, v high 32 bits -- each with the state bits
};
__device__ __forceinline__ SegPayload lb_identity(SegPayload) { return SegPayload{0, 0, 0}; }
__device__ __forceinline__ SegPayload lb_combine(const SegPayload& a, const SegPayload& b) {
  return SegPayload{a.f + b.f, b.f ? b.v : a.v + b.v, a.h > b.h ? a.h : b.h};
}
__device__ __forceinline__ void lb_store(SegRecord* r, uint64_t flag, const SegPayload& x) {
  st_relaxed_v2(&r->w[0], flag | (x.f & kValMask), flag | (x.h & kValMask));
  st_relaxed_v2(&r->w[2], flag | (x.v & 0xffffffffull), flag | (x.v >> 32));
}
__device__ __forceinline__ uint64_t lb_load(const SegRecord* r, SegPayload& x) {
  uint64_t a, b, c, d;
  ld_relaxed_v2(&r->w[0], a, b);
  ld_relaxed_v2(&r->w[2], c, d);
  const uint64_t fa = a & ~kValMask;
  x.f = a & kValMask;
  x.h = b & kValMask;
  x.v = (c & 0xffffffffull) | ((d & 0xffffffffull) << 32);
  const bool same = fa == (b & ~kValMask) && fa == (c & ~kValMask) && fa == (d & ~kValMask);
  return same ? fa : 0;
}

__device__ __forceinline__ CountPayload lb_broadcast0(CountPayload x) {
  return CountPayload{__shfl_sync(0xffffffffu, x.c, 0)};
}
__device__ __forceinline__ SegPayload lb_broadcast0(SegPayload x) {
  return SegPayload{__shfl_sync(0xffffffffu, x.f, 0), __shfl_sync(0xffffffffu, x.v, 0),
                    __shfl_sync(0xffffffffu, x.h, 0)};
}

template <typename P>
struct LookbackSmem {
  uint32_t first[2][32];   // per warp: nearest inclusive predecessor (distance) or NT
  uint32_t busy[2][32];    // per warp: ballot of unpublished predecessors
  P part[2][32];           // per warp: folded window part
};

// Ordered warp fold: lane 0 receives combine(x[31], ..., x[1], x[0]) where lane l holds
// the record l steps back (higher lanes are older).
template <typename P>
__device__ __forceinline__ P warp_fold_older(P x);

template <>
__device__ __forceinline__ CountPayload warp_fold_older(CountPayload x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x.c += __shfl_xor_sync(0xffffffffu, x.c, o);
  return x;
}
template <>
__device__ __forceinline__ SegPayload warp_fold_older(SegPayload x) {
  const uint32_t lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    SegPayload y;
    y.f = __shfl_down_sync(0xffffffffu, x.f, o);
    y.v = __shfl_down_sync(0xffffffffu, x.v, o);
    y.h = __shfl_down_sync(0xffffffffu, x.h, o);
    if (lane + o < 32) x = lb_combine(y, x);
  }
  return x;
}

// Publishes a tile's aggregate (thread 0); tile 0 publishes its inclusive prefix.
template <typename P, typename R>
__device__ __forceinline__ void lb_publish(R* records, uint64_t tile, const P& agg) {
  if (threadIdx.x == 0) lb_store(&records[tile], tile == 0 ? kFlagInc : kFlagAgg, agg);
}

// Called by all NT threads of the block with the same `tile` and `agg`, after
// lb_publish of the aggregate.  Resolves the exclusive prefix (returned in every thread)
// and publishes the inclusive prefix.  Each thread reads one predecessor record; while
// some record below the nearest inclusive one is unpublished, only the threads holding
// such records poll them again (bounded), then the block re-evaluates.  Contains
// __syncthreads.
template <int NT, typename P, typename R>
__device__ __forceinline__ P block_lookback_resolve(R* records, uint64_t tile, const P& agg, uint32_t* err,
                                                    LookbackSmem<P>& sm) {
  const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
  constexpr uint32_t W = NT / 32;
  const P id = lb_identity(P{});
  if (tile == 0) return id;
  P run = id;
  int64_t base = (int64_t)tile - 1;
  uint32_t rc = 0;
  while (true) {
    const int64_t idx = base - (int64_t)t;
    P x = id;
    uint64_t flag = kFlagInc;
    if (idx >= 0) flag = lb_load(&records[idx], x);
    uint32_t dmin;
    while (true) {
      const uint32_t b = rc++ & 1;
      const unsigned inc = __ballot_sync(0xffffffffu, flag == kFlagInc);
      const unsigned busy = __ballot_sync(0xffffffffu, flag == 0);
      if (lane == 0) {
        sm.first[b][warp] = inc ? warp * 32 + (__ffs(inc) - 1) : NT;
        sm.busy[b][warp] = busy;
      }
      __syncthreads();
      dmin = NT;
#pragma unroll
      for (uint32_t w = 0; w < W; ++w) dmin = min(dmin, sm.first[b][w]);
      bool wait = false;
#pragma unroll
      for (uint32_t w = 0; w < W; ++w) {
        const uint32_t lo = w * 32;
        if (lo >= dmin) break;
        const uint32_t m = dmin - lo >= 32 ? 0xffffffffu : ((1u << (dmin - lo)) - 1u);
        wait = wait || (sm.busy[b][w] & m) != 0;
      }
      if (!wait) break;
      if (flag == 0 && t < dmin) {
        uint32_t spins = 0;
        do {
          __nanosleep(spins < 32 ? 32 : 256);
          flag = lb_load(&records[idx], x);
          if (++spins > kSpinLimit && flag == 0) {
            raise_error(err, kErrTimeout);
            flag = kFlagAgg;   // give up: carry on with whatever the record holds
          }
        } while (flag == 0);
      }
    }
    const uint32_t b = rc++ & 1;
    if (t > dmin || idx < 0) x = id;
    x = warp_fold_older(x);
    if (lane == 0) sm.part[b][warp] = x;
    __syncthreads();
    P win = id;
#pragma unroll
    for (int w = W - 1; w >= 0; --w) win = lb_combine(win, sm.part[b][w]);
    run = lb_combine(win, run);
    if (dmin < NT) break;
    base -= NT;
  }
  if (t == 0) lb_store(&records[tile], kFlagInc, lb_combine(run, agg));
  return run;
}

// Warp-level resolve (one warp, e.g. warp 0 of the block, all 32 lanes): lane l
// examines the PL predecessors at distances PL*l .. PL*l + PL-1 (a window of 32*PL per
// round trip), waits (bounded) only for unpublished ones below the nearest inclusive
// record, folds the window in sequence order and publishes the inclusive prefix.
// Returns the exclusive prefix in every lane; the other warps of the block do not take
// part (the caller broadcasts through shared memory).
template <int PL, typename P, typename R>
__device__ __forceinline__ P warp_lookback_resolve(R* records, uint64_t tile, const P& agg, uint32_t* err) {
  const uint32_t lane = threadIdx.x & 31;
  constexpr uint32_t WIN = 32u * PL;
  const P id = lb_identity(P{});
  if (tile == 0) return id;
  P run = id;
  int64_t base = (int64_t)tile - 1;
  while (true) {
    P x[PL];
    uint64_t fl[PL];
#pragma unroll
    for (int r = 0; r < PL; ++r) {
      const int64_t idx = base - (int64_t)(lane * PL + r);
      x[r] = id;
      fl[r] = kFlagInc;
      if (idx >= 0) fl[r] = lb_load(&records[idx], x[r]);
    }
    uint32_t dmin;
    while (true) {
      uint32_t first = WIN;
#pragma unroll
      for (int r = PL - 1; r >= 0; --r)
        if (fl[r] == kFlagInc) first = lane * PL + r;
      dmin = __reduce_min_sync(0xffffffffu, first);
      bool busy = false;
#pragma unroll
      for (int r = 0; r < PL; ++r) busy = busy || (fl[r] == 0 && lane * PL + r < dmin);
      if (!__any_sync(0xffffffffu, busy)) break;
#pragma unroll
      for (int r = 0; r < PL; ++r) {
        if (fl[r] == 0 && lane * PL + r < dmin) {
          const int64_t idx = base - (int64_t)(lane * PL + r);
          uint32_t spins = 0;
          do {
            __nanosleep(spins < 32 ? 32 : 256);
            fl[r] = lb_load(&records[idx], x[r]);
            if (++spins > kSpinLimit && fl[r] == 0) {
              raise_error(err, kErrTimeout);
              fl[r] = kFlagAgg;   // give up: carry on with whatever the record holds
            }
          } while (fl[r] == 0);
        }
      }
    }
    P acc = id;
#pragma unroll
    for (int r = PL - 1; r >= 0; --r)
      if (lane * PL + r <= dmin) acc = lb_combine(acc, x[r]);
    acc = warp_fold_older(acc);
    P win;
    win = acc;
    win = lb_broadcast0(win);
    run = lb_combine(win, run);
    if (dmin < WIN) break;
    base -= WIN;
  }
  if (lane == 0) lb_store(&records[tile], kFlagInc, lb_combine(run, agg));
  return run;
}

// Publish and resolve in one call.
template <int NT, typename P, typename R>
__device__ __forceinline__ P block_lookback(R* records, uint64_t tile, const P& agg, uint32_t* err,
                                            LookbackSmem<P>& sm) {
  lb_publish(records, tile, agg);
  return block_lookback_resolve<NT>(records, tile, agg, err, sm);
}

}  // namespace rfx
