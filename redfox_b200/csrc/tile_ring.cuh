// tile_ring.cuh -- shared-memory stages filled by TMA tensor copies.
//
// A relation of packed rows is viewed as a 2-D byte tensor of 128-byte lines
// ([bytes / 128][128] u8).  One tile = a box of up to 256 lines (32 KB), copied by one
// cp.async.bulk.tensor into a 1024-byte aligned stage with the 128-byte swizzle: the
// 16-byte chunk c of line l lands at chunk c ^ (l & 7).  A thread that owns a
// contiguous span of a tile (a power of two of at least 8 bytes) then reads it from
// shared memory without bank conflicts.  The bytes after the last full line (< 128)
// are not covered by the tensor map; the consumer copies them with plain loads.
// Completion of a copy is counted on an mbarrier; every wait is bounded.
#pragma once

#include <cuda.h>

#include "rfx_device.cuh"

namespace rfx {

constexpr uint32_t kRingLineBytes = 128;
constexpr uint32_t kRingBoxLines = 256;
constexpr uint32_t kRingTileBytes = kRingLineBytes * kRingBoxLines;   // 32 KB
constexpr uint32_t kRingWaitLimit = 1u << 24;                         // polls of an mbarrier

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset within a stage after the 128-byte swizzle.
__device__ __forceinline__ uint32_t swz(uint32_t off) { return off ^ (((off >> 7) & 7u) << 4); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// Bounded wait for the phase with the given parity; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t i = 0; i < kRingWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (i > 64) __nanosleep(64);
  }
  return false;
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// One box of the line tensor (x = 0, y = first line) into shared memory; completion is
// counted on `bar`.  No multicast: the source is this GPU's own memory.
__device__ __forceinline__ void tma_load_lines(void* dst, const CUtensorMap* map, uint32_t line, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(line), "r"(smem_u32(bar))
      : "memory");
}
// A 1-D bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from this
// GPU's global memory into shared memory; completion counted on `bar`.  No multicast.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void prefetch_map(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// Per-stage mbarriers and the tile each stage holds.
template <int S>
struct TileRing {
  uint64_t bar[S];
  uint32_t tile[S];
};

// Copies the bytes of tile `tile` at or beyond byte `covered` (not in the tensor map)
// from global memory into the swizzled stage: 4-byte words, then single bytes.
// `limit` = total bytes; `src` is 16-byte aligned and `covered` a multiple of 128.
__device__ __forceinline__ void ring_fill_tail(uint8_t* stage, const uint8_t* src, uint64_t tile, uint64_t covered,
                                               uint64_t limit, uint32_t tile_bytes = kRingTileBytes) {
  const uint64_t t0 = tile * tile_bytes;
  const uint64_t lo = covered > t0 ? covered : t0;
  const uint64_t hi = limit < t0 + tile_bytes ? limit : t0 + tile_bytes;
  if (lo >= hi) return;
  const uint64_t hi4 = lo + ((hi - lo) & ~3ull);
  for (uint64_t b = lo + 4ull * threadIdx.x; b < hi4; b += 4ull * blockDim.x) {
    const uint32_t w = *reinterpret_cast<const uint32_t*>(src + b);
    *reinterpret_cast<uint32_t*>(stage + swz((uint32_t)(b - t0))) = w;
  }
  if (threadIdx.x == 0)
    for (uint64_t b = hi4; b < hi; ++b) stage[swz((uint32_t)(b - t0))] = src[b];
}

template <typename T>
__device__ __forceinline__ T ring_read(const uint8_t* stage, uint32_t off) {
  return *reinterpret_cast<const T*>(stage + swz(off));
}

}  // namespace rfx
