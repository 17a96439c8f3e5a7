// host_common.h -- host-side helpers shared by the entry points: CUDA error mapping,
// per-device properties and error word, workspace carving, launch sizing.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "rfx/rfx.h"

namespace rfx {

#define RFX_CUDA_TRY(expr)                              \
  do {                                                  \
    cudaError_t e_ = (expr);                            \
    if (e_ != cudaSuccess) return ::rfx::cuda_fail(e_); \
  } while (0)

rfx_status cuda_fail(cudaError_t e);

// Streaming multiprocessors of the current device (148 on B200).
int device_sms();
// The current device's error word (allocated once per device, zero when healthy).
uint32_t* device_error_word();

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Sequential carving of a workspace into 256-byte aligned pieces.
struct Carver {
  uint8_t* base;
  size_t used;
  explicit Carver(void* b) : base(static_cast<uint8_t*>(b)), used(0) {}
  template <typename T>
  T* take(size_t count) {
    used = align_up(used, 256);
    T* p = reinterpret_cast<T*>(base ? base + used : nullptr);
    used += count * sizeof(T);
    return p;
  }
};

inline cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

// Persistent grid: min(work blocks, SMs * resident blocks per SM).
int persistent_grid(const void* kernel, int threads, size_t dyn_smem, uint64_t work_blocks);
// Raise a kernel's dynamic shared memory limit once.
cudaError_t allow_smem(const void* kernel, size_t bytes);

// Tensor map of `lines` 128-byte lines at `base` (a [lines][128] u8 tensor, boxes of
// `box_lines` <= 256 lines, 128-byte swizzle) for the tile ring.  False when `base` is not 16-byte
// aligned, `lines` is 0 or above 2^31, or the driver rejects the map; *map is then
// zeroed and must not be used.
bool encode_line_map(CUtensorMap* map, const void* base, uint64_t lines, uint32_t box_lines = 256);

}  // namespace rfx
