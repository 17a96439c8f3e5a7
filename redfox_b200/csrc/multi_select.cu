// multi_select.cu -- one scan of a resident relation for many range selections at once
// (the serving form's shared scan): every row is tested against each query's range and
// emitted once per matching query, tagged with the query id, in (row, query) order.
//
// Output rows are 8 bytes: ((key << 8 | q) << val_width) | val, where key and val are bit
// fields of the input row.  Folding q into the key makes the queries of one batch sort,
// join and group together without mixing: the sort-merge join on (key, q) joins every
// query with itself only.  Compaction is one pass with decoupled look-back over tiles of
// 2048 rows (dynamic tile ids, bounded waits), as the select kernels do.
#include <cstring>

#include "host_common.h"
#include "search.cuh"

namespace rfx {

constexpr int kMsThreads = 256;
constexpr int kMsRows = 8;                         // rows per thread
constexpr int kMsTile = kMsThreads * kMsRows;
constexpr uint32_t kMsMaxQueries = 256;

struct MultiSelectArgs {
  const uint8_t* in;
  uint64_t n;
  uint8_t* out;          // 8-byte rows
  uint64_t cap;
  uint64_t* d_count;
  uint64_t* status;
  uint32_t* tile_counter;
  uint32_t* err;
  uint32_t fshift, fwidth, kshift, kwidth, vshift, vwidth, nq;
  uint32_t lo[kMsMaxQueries];
  uint32_t hi[kMsMaxQueries];
};

__device__ __forceinline__ uint64_t ms_field(u128 row, uint32_t shift, uint32_t width) {
  const u128 v = row >> shift;
  return width >= 64 ? (uint64_t)v : (uint64_t)v & ((1ull << width) - 1);
}

template <int W>
__global__ void __launch_bounds__(kMsThreads) multi_select_kernel(const MultiSelectArgs a) {
  __shared__ uint32_t s_lo[kMsMaxQueries], s_hi[kMsMaxQueries];
  __shared__ uint64_t s_warp[kMsThreads / 32];
  __shared__ uint64_t s_prefix;
  __shared__ uint32_t s_tile;
  const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
  for (uint32_t q = t; q < a.nq; q += kMsThreads) {
    s_lo[q] = a.lo[q];
    s_hi[q] = a.hi[q];
  }
  const uint64_t num_tiles = (a.n + kMsTile - 1) / kMsTile;
  while (true) {
    if (t == 0) s_tile = atomicAdd(a.tile_counter, 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    if (tile >= num_tiles) break;
    const uint64_t r0 = tile * kMsTile + (uint64_t)t * kMsRows;
    uint32_t f[kMsRows];
    uint64_t cnt = 0;
#pragma unroll
    for (int j = 0; j < kMsRows; ++j) {
      f[j] = 0xffffffffu;
      if (r0 + j < a.n) f[j] = (uint32_t)ms_field(load_u128<W>(a.in, r0 + j), a.fshift, a.fwidth);
    }
#pragma unroll
    for (int j = 0; j < kMsRows; ++j) {
      if (r0 + j >= a.n) continue;
      for (uint32_t q = 0; q < a.nq; ++q) cnt += (f[j] >= s_lo[q] && f[j] < s_hi[q]) ? 1u : 0u;
    }
    // block exclusive scan of the per-thread counts
    uint64_t incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    uint64_t wpre = 0, btot = 0;
    for (uint32_t w = 0; w < kMsThreads / 32; ++w) {
      if (w < warp) wpre += s_warp[w];
      btot += s_warp[w];
    }
    if (warp == 0) {
      const uint64_t pre = lookback_exclusive(a.status, (uint32_t)tile, btot, a.err);
      if (t == 0) {
        s_prefix = pre;
        if (tile == num_tiles - 1) *a.d_count = pre + btot;
      }
    }
    __syncthreads();
    uint64_t pos = s_prefix + wpre + incl - cnt;
    uint64_t* out = reinterpret_cast<uint64_t*>(a.out);
#pragma unroll
    for (int j = 0; j < kMsRows; ++j) {
      if (r0 + j >= a.n) continue;
      const u128 row = load_u128<W>(a.in, r0 + j);
      const uint64_t key = ms_field(row, a.kshift, a.kwidth);
      const uint64_t val = ms_field(row, a.vshift, a.vwidth);
      for (uint32_t q = 0; q < a.nq; ++q) {
        if (f[j] >= s_lo[q] && f[j] < s_hi[q]) {
          if (pos < a.cap) out[pos] = (((key << 8) | q) << a.vwidth) | val;
          ++pos;
        }
      }
    }
    __syncthreads();
  }
  if (a.n == 0 && blockIdx.x == 0 && t == 0) *a.d_count = 0;
}

namespace {

struct MsLayout {
  uint64_t* status;
  uint32_t* counter;
  size_t total;
};

MsLayout ms_layout(void* ws, uint64_t n) {
  MsLayout L;
  Carver c(ws);
  L.status = c.take<uint64_t>((n + kMsTile - 1) / kMsTile + 1);
  L.counter = c.take<uint32_t>(1);
  L.total = align_up(c.used, 256);
  return L;
}

template <int W>
rfx_status launch_ms(const MultiSelectArgs& a, cudaStream_t s) {
  const uint64_t tiles = (a.n + kMsTile - 1) / kMsTile;
  const int grid = persistent_grid((const void*)multi_select_kernel<W>, kMsThreads, 0, tiles ? tiles : 1);
  multi_select_kernel<W><<<grid, kMsThreads, 0, s>>>(a);
  RFX_CUDA_TRY(cudaGetLastError());
  return RFX_OK;
}

}  // namespace
}  // namespace rfx

using namespace rfx;

extern "C" size_t rfx_multi_select_workspace(uint64_t n) { return ms_layout(nullptr, n).total; }

extern "C" rfx_status rfx_multi_select(void* out, uint64_t capacity, uint64_t* d_count, const void* in, uint64_t n,
                                       uint32_t in_bytes, uint32_t field_shift, uint32_t field_width,
                                       const uint32_t* lo, const uint32_t* hi, uint32_t nq, uint32_t key_shift,
                                       uint32_t key_width, uint32_t val_shift, uint32_t val_width, void* workspace,
                                       size_t workspace_bytes, void* stream) {
  if (in_bytes != 4 && in_bytes != 8 && in_bytes != 16) return RFX_ERR_UNSUPPORTED;
  if (nq == 0 || nq > kMsMaxQueries || field_width == 0 || field_width > 32 || key_width == 0 ||
      key_width + 8 + val_width > 64 || field_shift + field_width > in_bytes * 8 ||
      key_shift + key_width > in_bytes * 8 || val_shift + val_width > in_bytes * 8)
    return RFX_ERR_UNSUPPORTED;
  if (!d_count || !lo || !hi || (n && !in) || (capacity && !out)) return RFX_ERR_INVALID;
  if ((n && reinterpret_cast<uintptr_t>(in) % (in_bytes < 16 ? in_bytes : 16)) ||
      (capacity && reinterpret_cast<uintptr_t>(out) % 8))
    return RFX_ERR_INVALID;
  MsLayout L = ms_layout(workspace, n);
  if (!workspace || workspace_bytes < L.total) return RFX_ERR_WORKSPACE;
  uint32_t* err = device_error_word();
  if (!err) return RFX_ERR_CUDA;
  cudaStream_t s = as_stream(stream);
  RFX_CUDA_TRY(cudaMemsetAsync(workspace, 0, L.total, s));
  MultiSelectArgs a;
  std::memset(&a, 0, sizeof(a));
  a.in = static_cast<const uint8_t*>(in);
  a.n = n;
  a.out = static_cast<uint8_t*>(out);
  a.cap = capacity;
  a.d_count = d_count;
  a.status = L.status;
  a.tile_counter = L.counter;
  a.err = err;
  a.fshift = field_shift;
  a.fwidth = field_width;
  a.kshift = key_shift;
  a.kwidth = key_width;
  a.vshift = val_shift;
  a.vwidth = val_width;
  a.nq = nq;
  for (uint32_t q = 0; q < nq; ++q) {
    a.lo[q] = lo[q];
    a.hi[q] = hi[q];
  }
  switch (in_bytes) {
    case 4: return launch_ms<4>(a, s);
    case 8: return launch_ms<8>(a, s);
    default: return launch_ms<16>(a, s);
  }
}
