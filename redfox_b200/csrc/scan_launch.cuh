// scan_launch.cuh -- launchers for the scan kernels, instantiated per input width in
// scan_w{1,2,4,8,16,32,64}.cu so the instantiations compile in parallel.
#pragma once

#include "host_common.h"
#include "scan_kernels.cuh"

namespace rfx {

struct ScanLaunch {
  const ScanProgram* prog;
  const void* in;
  uint64_t n;
  void* out;
  uint64_t* d_count;
  uint64_t* tile_status;
  uint32_t* tile_counter;
  uint32_t* err;
  cudaStream_t stream;
};

template <int WIN, int WOUT, int MODE>
rfx_status launch_compact_wo(const ScanLaunch& a) {
  using S = Slots<WIN, WOUT>;
  const size_t smem = (size_t)S::PER_THREAD * kScanThreads * sizeof(uint64_t);
  auto k = scan_compact_kernel<WIN, WOUT, MODE>;
  RFX_CUDA_TRY(allow_smem((const void*)k, smem));
  const uint64_t tiles = (a.n + kScanTile - 1) / kScanTile;
  const int grid = persistent_grid((const void*)k, kScanThreads, smem, tiles ? tiles : 1);
  k<<<grid, kScanThreads, smem, a.stream>>>(*a.prog, static_cast<const uint8_t*>(a.in), a.n,
                                             static_cast<uint8_t*>(a.out), a.d_count, a.tile_status,
                                             a.tile_counter, a.err);
  RFX_CUDA_TRY(cudaGetLastError());
  return RFX_OK;
}

// mode: 0 select (WOUT == WIN), 1 select+arith+project, 2 map (no predicate)
template <int WIN>
rfx_status launch_compact(int mode, uint32_t wout, const ScanLaunch& a) {
  if (mode == 0) return launch_compact_wo<WIN, WIN, 0>(a);
#define RFX_WOUT_CASE(WO)                                                             \
  case WO:                                                                            \
    return mode == 1 ? launch_compact_wo<WIN, WO, 1>(a) : launch_compact_wo<WIN, WO, 2>(a);
  switch (wout) {
    RFX_WOUT_CASE(1)
    RFX_WOUT_CASE(2)
    RFX_WOUT_CASE(4)
    RFX_WOUT_CASE(8)
    RFX_WOUT_CASE(16)
    RFX_WOUT_CASE(32)
    RFX_WOUT_CASE(64)
    default: return RFX_ERR_UNSUPPORTED;
  }
#undef RFX_WOUT_CASE
}

struct AggLaunch {
  const ScanProgram* prog;
  const void* in;
  uint64_t n;
  unsigned long long* gacc;
  uint32_t* done_counter;
  uint64_t* out_keys;
  int64_t* out_sums;
  uint64_t* out_counts;
  uint64_t* d_groups;
  uint32_t* err;
  cudaStream_t stream;
};

// Private per-thread accumulators are used while the table is this small.
constexpr uint32_t kPrivateAccLimit = 24;

template <int WIN>
rfx_status launch_aggregate(const AggLaunch& a) {
  constexpr int NIN = Limbs<WIN>::N;
  const uint32_t nacc = a.prog->ngroups_total * (a.prog->nsum + 1);
  const size_t slots = (size_t)(NIN + kMaxExt + kMaxRegs) * kScanThreads * sizeof(uint64_t);
  const bool priv = nacc <= kPrivateAccLimit;
  const size_t smem = slots + (priv ? (size_t)nacc * kScanThreads : (size_t)nacc) * sizeof(uint64_t);
  const void* k = priv ? (const void*)scan_aggregate_kernel<WIN, true> : (const void*)scan_aggregate_kernel<WIN, false>;
  RFX_CUDA_TRY(allow_smem(k, smem));
  const uint64_t blocks = (a.n + 2ull * kScanThreads - 1) / (2ull * kScanThreads);
  const int grid = persistent_grid(k, kScanThreads, smem, blocks ? blocks : 1);
  if (priv)
    scan_aggregate_kernel<WIN, true><<<grid, kScanThreads, smem, a.stream>>>(
        *a.prog, static_cast<const uint8_t*>(a.in), a.n, a.gacc, a.done_counter, a.out_keys,
        a.out_sums, a.out_counts, a.d_groups, a.err);
  else
    scan_aggregate_kernel<WIN, false><<<grid, kScanThreads, smem, a.stream>>>(
        *a.prog, static_cast<const uint8_t*>(a.in), a.n, a.gacc, a.done_counter, a.out_keys,
        a.out_sums, a.out_counts, a.d_groups, a.err);
  RFX_CUDA_TRY(cudaGetLastError());
  return RFX_OK;
}

// Loads both aggregate kernels of this row width (CUDA loads a kernel on its first launch
// by default, which takes device memory): a caller that must not allocate on later calls
// loads them up front.
template <int WIN>
rfx_status preload_aggregate() {
  cudaFuncAttributes attr;
  RFX_CUDA_TRY(cudaFuncGetAttributes(&attr, (const void*)scan_aggregate_kernel<WIN, true>));
  RFX_CUDA_TRY(cudaFuncGetAttributes(&attr, (const void*)scan_aggregate_kernel<WIN, false>));
  return RFX_OK;
}

#define RFX_INSTANTIATE_SCAN(W)                                              \
  template rfx_status launch_compact<W>(int, uint32_t, const ScanLaunch&); \
  template rfx_status launch_aggregate<W>(const AggLaunch&);               \
  template rfx_status preload_aggregate<W>();

}  // namespace rfx
