// noalloc_abi.cu -- rfx_filter_aggregate_noalloc: the fused filter -> arith -> group-by
// aggregate with its scratch in a fixed device array instead of a caller workspace.
//
// Who needs it: callers that cannot allocate device memory at call time -- a host runtime
// that has already handed all device memory out by liveness (as the reference's Harmony
// runtime plans its variables), or a serving loop that must not touch the allocator on its
// request path.
//
// The scratch is g_scratch below: kScratchWords 64-bit accumulators (room for the largest
// plan the aggregate accepts: 4096 groups x (4 sums + a count)) plus a completion counter,
// about 160 KiB, held by every GPU that loads the library until the process exits.  Every call uses the same array, so two
// calls whose kernels overlap on the GPU (different streams without ordering between
// them) race and produce wrong sums; calls on one stream are ordered and safe.  The array
// keeps the last call's contents; each call clears what must start at zero.
#include <mutex>

#include "scan_launch.cuh"

namespace rfx {

template <int W>
rfx_status launch_aggregate(const AggLaunch&);
template <int W>
rfx_status preload_aggregate();

namespace {

constexpr size_t kScratchWords = (size_t)kMaxGroups * (kMaxSum + 1);

// The scratch: the accumulators, then the completion counter (one more 64-bit word).
static __device__ __align__(256) unsigned long long g_scratch[kScratchWords + 1];

// In host code `g_scratch` only names a host-side stand-in; the device address comes from
// cudaGetSymbolAddress, taken once per device with that device current.  The same first
// call loads every kernel the entry can launch (CUDA otherwise loads each on its first
// launch, taking device memory then), so that later calls change nothing in device memory.
std::mutex g_mu;
unsigned long long* g_addr[128] = {nullptr};

rfx_status preload_kernels() {
  rfx_status st;
  if ((st = preload_aggregate<1>()) != RFX_OK || (st = preload_aggregate<2>()) != RFX_OK ||
      (st = preload_aggregate<4>()) != RFX_OK || (st = preload_aggregate<8>()) != RFX_OK ||
      (st = preload_aggregate<16>()) != RFX_OK || (st = preload_aggregate<32>()) != RFX_OK ||
      (st = preload_aggregate<64>()) != RFX_OK)
    return st;
  return RFX_OK;
}

rfx_status scratch_address(unsigned long long** out) {
  int dev = 0;
  RFX_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) return RFX_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p) {
      (void)cudaGetLastError();
      return RFX_ERR_CUDA;
    }
    const rfx_status st = preload_kernels();
    if (st != RFX_OK) return st;
    g_addr[dev] = static_cast<unsigned long long*>(p);
  }
  *out = g_addr[dev];
  return RFX_OK;
}

rfx_status dispatch(uint32_t win, const AggLaunch& a) {
  switch (win) {
    case 1: return launch_aggregate<1>(a);
    case 2: return launch_aggregate<2>(a);
    case 4: return launch_aggregate<4>(a);
    case 8: return launch_aggregate<8>(a);
    case 16: return launch_aggregate<16>(a);
    case 32: return launch_aggregate<32>(a);
    case 64: return launch_aggregate<64>(a);
    default: return RFX_ERR_UNSUPPORTED;
  }
}

}  // namespace
}  // namespace rfx

using namespace rfx;

extern "C" rfx_status rfx_filter_aggregate_noalloc(const void* in, uint64_t n, const rfx_tuple* in_type,
                                                   const rfx_cmp* cmps, uint32_t ncmp,
                                                   const rfx_arith_expr* ariths, uint32_t narith,
                                                   const uint32_t* group_fields, const uint32_t* group_domain,
                                                   uint32_t ngroup, const uint32_t* sum_fields, uint32_t nsum,
                                                   uint64_t* out_keys, int64_t* out_sums, uint64_t* out_counts,
                                                   uint64_t* d_groups, uint32_t* d_error, void* stream) {
  if ((!in && n) || !out_keys || !out_counts || !d_groups || (nsum && !out_sums)) return RFX_ERR_INVALID;
  // the plan is validated exactly as rfx_filter_aggregate validates it (same statuses);
  // every plan it accepts fits the fixed scratch, and the check below keeps that true
  ScanProgram p;
  rfx_status st = compile_scan(&p, in_type, cmps, ncmp, ariths, narith);
  if (st != RFX_OK) return st;
  st = compile_aggregate(&p, group_fields, group_domain, ngroup, sum_fields, nsum);
  if (st != RFX_OK) return st;
  const size_t nacc = (size_t)p.ngroups_total * (nsum + 1);
  if (nacc > kScratchWords) return RFX_ERR_CAPACITY;  // larger than the fixed scratch (not reachable
                                                      // while compile_aggregate caps the table)
  if (n && (reinterpret_cast<uintptr_t>(in) % (p.in_bytes < 16 ? p.in_bytes : 16)) != 0) return RFX_ERR_INVALID;
  unsigned long long* base = nullptr;
  st = scratch_address(&base);
  if (st != RFX_OK) return st;
  cudaStream_t s = as_stream(stream);
  unsigned long long* gacc = base;
  uint32_t* done = reinterpret_cast<uint32_t*>(base + kScratchWords);
  // zero this call's accumulators and the completion counter (the array keeps old values)
  RFX_CUDA_TRY(cudaMemsetAsync(gacc, 0, nacc * sizeof(unsigned long long), s));
  RFX_CUDA_TRY(cudaMemsetAsync(done, 0, sizeof(unsigned long long), s));
  AggLaunch a{&p, in, n, gacc, done, out_keys, out_sums, out_counts, d_groups, d_error, s};
  return dispatch(p.in_bytes, a);
}
