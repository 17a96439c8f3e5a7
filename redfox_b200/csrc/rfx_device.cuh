// rfx_device.cuh -- device-side building blocks shared by every redfox_b200 kernel:
// packed-tuple limb access, vectorised row loads/stores, decoupled look-back with
// bounded waits, and the device error word.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "rfx/rfx.h"

namespace rfx {

// ------------------------------------------------------------------ errors
// Kernels never trap.  A bounded wait that gives up, or an input that violates a
// declared bound, records a code in the per-device error word and the kernel carries
// on (its output is then unspecified); the host reads the word with rfx_device_status.
enum : uint32_t {
  kErrNone = 0,
  kErrTimeout = RFX_ERR_TIMEOUT,
  kErrCapacity = RFX_ERR_CAPACITY,
  kErrInvalid = RFX_ERR_INVALID,
};

__device__ __forceinline__ void raise_error(uint32_t* err, uint32_t code) {
  if (err) atomicCAS(err, 0u, code);
}

// Upper bound on polls of a look-back predecessor before giving up (about 0.5 s with
// the back-off below); a healthy predecessor publishes within microseconds.
constexpr uint32_t kSpinLimit = 1u << 22;

// cp.async of one 16-byte chunk into shared memory; only `src_bytes` (<= 16) are read, the
// rest of the chunk is zero-filled.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
               "l"(src), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Up to `len` bytes of `src` from byte b0 (src + b0 16-byte aligned) into `dst`, block-
// strided 16-byte chunks; nothing at or past byte `bend` (the end of the array) is read.
__device__ __forceinline__ void block_prefetch16(uint8_t* dst, const uint8_t* src, uint64_t b0, uint64_t len,
                                                 uint64_t bend, uint32_t nthreads) {
  const uint64_t b1 = b0 + len < bend ? b0 + len : bend;
  const uint32_t chunks = b1 > b0 ? (uint32_t)((b1 - b0 + 15) / 16) : 0u;
  for (uint32_t c = threadIdx.x; c < chunks; c += nthreads) {
    const uint64_t at = b0 + 16ull * c;
    cp_async16(dst + 16u * c, src + at, (uint32_t)(bend - at < 16 ? bend - at : 16));
  }
}

// ------------------------------------------------------------------ memory order
__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(uint64_t* p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ------------------------------------------------------------------ look-back (64-bit)
// One status word per tile: bits 63..62 = 0 not ready, 1 aggregate, 2 inclusive prefix;
// bits 61..0 = the value.  Used for counts (compaction offsets, join output offsets).
constexpr uint64_t kFlagAgg = 1ull << 62;
constexpr uint64_t kFlagInc = 2ull << 62;
constexpr uint64_t kValMask = (1ull << 62) - 1;

// Called by the whole warp 0 of a tile.  Publishes `aggregate`, examines predecessors
// kLookLanes per lane (a window of 32 * kLookLanes tiles per round trip) and returns the
// exclusive prefix (same value in every lane).  A wider window pays when the nearest
// inclusive predecessor is far back (many short tiles in flight, as in the set filters);
// where it is usually near, the extra loads only add L2 traffic (the 60M-row select runs
// 2.36 ms with 1, 3.0 ms with 4).
template <int kLookLanes = 1>
__device__ __forceinline__ uint64_t lookback_exclusive(uint64_t* status, uint32_t tile,
                                                       uint64_t aggregate, uint32_t* err) {
  const uint32_t lane = threadIdx.x & 31;
  constexpr uint32_t WIN = 32u * kLookLanes;
  if (tile == 0) {
    if (lane == 0) st_relaxed_u64(&status[0], kFlagInc | (aggregate & kValMask));
    return 0;
  }
  if (lane == 0) st_relaxed_u64(&status[tile], kFlagAgg | (aggregate & kValMask));
  uint64_t prefix = 0;
  int64_t base = (int64_t)tile - 1;  // highest predecessor not yet folded in
  uint32_t spins = 0;
  while (true) {
    uint64_t w[kLookLanes];
#pragma unroll
    for (int r = 0; r < kLookLanes; ++r) {
      const int64_t idx = base - (int64_t)(lane * kLookLanes + r);
      w[r] = idx >= 0 ? ld_relaxed_u64(&status[idx]) : kFlagInc;
    }
    uint32_t first = WIN;
#pragma unroll
    for (int r = kLookLanes - 1; r >= 0; --r)
      if ((w[r] & ~kValMask) == kFlagInc) first = lane * kLookLanes + r;
    const uint32_t dmin = __reduce_min_sync(0xffffffffu, first);
    bool busy = false;
    uint64_t v = 0;
#pragma unroll
    for (int r = 0; r < kLookLanes; ++r) {
      if (lane * kLookLanes + r <= dmin) {
        busy = busy || (w[r] & ~kValMask) == 0;
        v += w[r] & kValMask;
      }
    }
    if (__any_sync(0xffffffffu, busy)) {
      if (++spins > kSpinLimit) {
        raise_error(err, kErrTimeout);
        break;
      }
      __nanosleep(spins < 64 ? 32 : 200);
      continue;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    prefix += v;
    if (dmin < WIN) break;
    base -= WIN;
  }
  if (lane == 0) st_relaxed_u64(&status[tile], kFlagInc | ((prefix + aggregate) & kValMask));
  return prefix;
}

}  // namespace rfx
