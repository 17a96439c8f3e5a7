// scan_abi.cu -- C ABI entries for select / arith / project / filter-aggregate and the
// synthetic row generator.
#include <cstring>

#include "scan_launch.cuh"
#include "tune.h"

namespace rfx {

rfx_status jit_aggregate(const ScanProgram& p, const void* in, uint64_t n, unsigned long long* gacc, uint32_t* done,
                         uint64_t* out_keys, int64_t* out_sums, uint64_t* out_counts, uint64_t* d_groups, uint32_t* err,
                         cudaStream_t stream, int variant = 0);
rfx_status jit_compact(const ScanProgram& p, int mode, const void* in, uint64_t n, void* out, uint64_t* d_count,
                       uint64_t* status, uint32_t* counter, uint32_t* err, cudaStream_t stream, uint64_t tile_rows, int variant = 0);

template <int W>
rfx_status launch_compact(int, uint32_t, const ScanLaunch&);
template <int W>
rfx_status launch_aggregate(const AggLaunch&);

namespace {

rfx_status dispatch_compact(uint32_t win, int mode, uint32_t wout, const ScanLaunch& a) {
  switch (win) {
    case 1: return launch_compact<1>(mode, wout, a);
    case 2: return launch_compact<2>(mode, wout, a);
    case 4: return launch_compact<4>(mode, wout, a);
    case 8: return launch_compact<8>(mode, wout, a);
    case 16: return launch_compact<16>(mode, wout, a);
    case 32: return launch_compact<32>(mode, wout, a);
    case 64: return launch_compact<64>(mode, wout, a);
    default: return RFX_ERR_UNSUPPORTED;
  }
}

rfx_status dispatch_aggregate(uint32_t win, const AggLaunch& a) {
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

// Rows of 16 bytes and more are moved with 16-byte vector accesses.
bool aligned(const void* p, uint32_t row_bytes) {
  const uintptr_t a = row_bytes < 16 ? row_bytes : 16;
  return (reinterpret_cast<uintptr_t>(p) % a) == 0;
}

size_t compact_workspace(uint64_t n) {
  Carver c(nullptr);
  c.take<uint64_t>((n + kScanTile - 1) / kScanTile + 1);
  c.take<uint32_t>(1);
  return align_up(c.used, 256);
}

rfx_status run_compact(int mode, const ScanProgram& p, void* out, uint64_t* d_count, const void* in,
                       uint64_t n, void* ws, size_t ws_bytes, void* stream) {
  if (!d_count) return RFX_ERR_INVALID;
  if (n == 0) {  // empty relation: nothing to read, the count is 0
    RFX_CUDA_TRY(cudaMemsetAsync(d_count, 0, sizeof(uint64_t), as_stream(stream)));
    return RFX_OK;
  }
  if (!out || !in) return RFX_ERR_INVALID;
  if (!aligned(in, p.in_bytes) || !aligned(out, mode == 0 ? p.in_bytes : p.out_bytes)) return RFX_ERR_INVALID;
  cudaStream_t s = as_stream(stream);
  uint32_t* err = device_error_word();
  if (!err) return RFX_ERR_CUDA;
  Carver c(ws);
  const uint64_t tiles = (n + kScanTile - 1) / kScanTile;
  uint64_t* status = c.take<uint64_t>(tiles + 1);
  uint32_t* counter = c.take<uint32_t>(1);
  if (!ws || ws_bytes < c.used) return RFX_ERR_WORKSPACE;
  // the plan-specialised kernel when runtime compilation is available; its rows per
  // thread are tuned per plan shape and size class when tuning is on
  const size_t clear = c.used;
  auto run = [&](int v) -> rfx_status {
    RFX_CUDA_TRY(cudaMemsetAsync(ws, 0, clear, s));
    return jit_compact(p, mode, in, n, out, d_count, status, counter, err, s, kScanTile, v);
  };
  const uint64_t shape = ((uint64_t)p.in_bytes << 40) | ((uint64_t)(mode == 0 ? p.in_bytes : p.out_bytes) << 24) |
                         ((uint64_t)mode << 16) | ((uint64_t)p.ncmp << 8) | p.ninstr;
  rfx_status st = run(tune_pick(TUNE_SCAN_COMPACT, shape, n, 3, run, s));
  if (st != RFX_ERR_UNSUPPORTED) return st;
  RFX_CUDA_TRY(cudaMemsetAsync(ws, 0, clear, s));
  ScanLaunch a{&p, in, n, out, d_count, status, counter, err, s};
  return dispatch_compact(p.in_bytes, mode, mode == 0 ? p.in_bytes : p.out_bytes, a);
}

}  // namespace
}  // namespace rfx

using namespace rfx;

extern "C" size_t rfx_select_workspace(uint64_t n, const rfx_tuple* in) {
  (void)in;
  return compact_workspace(n);
}

extern "C" rfx_status rfx_select(void* out, uint64_t* d_count, const void* in, uint64_t n,
                                 const rfx_tuple* in_type, const rfx_cmp* cmps, uint32_t ncmp,
                                 void* workspace, size_t workspace_bytes, void* stream) {
  ScanProgram p;
  rfx_status st = compile_scan(&p, in_type, cmps, ncmp, nullptr, 0);
  if (st != RFX_OK) return st;
  return run_compact(0, p, out, d_count, in, n, workspace, workspace_bytes, stream);
}

extern "C" rfx_status rfx_select_project(void* out, uint64_t* d_count, const void* in, uint64_t n,
                                         const rfx_tuple* in_type, const rfx_cmp* cmps, uint32_t ncmp,
                                         const rfx_arith_expr* ariths, uint32_t narith,
                                         const rfx_tuple* out_type, const uint32_t* map,
                                         void* workspace, size_t workspace_bytes, void* stream) {
  ScanProgram p;
  rfx_status st = compile_scan(&p, in_type, cmps, ncmp, ariths, narith);
  if (st != RFX_OK) return st;
  st = compile_projection(&p, out_type, map);
  if (st != RFX_OK) return st;
  return run_compact(1, p, out, d_count, in, n, workspace, workspace_bytes, stream);
}

namespace {
// Map mode (arith / project alone) assigns tiles statically and needs no workspace,
// matching the reference's set_arith / set_project signatures.
rfx_status run_map(const ScanProgram& p, void* out, const void* in, uint64_t n, void* stream) {
  if (n == 0) return RFX_OK;
  if (!out || !in) return RFX_ERR_INVALID;
  if (!aligned(in, p.in_bytes) || !aligned(out, p.out_bytes)) return RFX_ERR_INVALID;
  uint32_t* err = device_error_word();
  if (!err) return RFX_ERR_CUDA;
  rfx_status st = jit_compact(p, 2, in, n, out, nullptr, nullptr, nullptr, err, as_stream(stream), kScanTile);
  if (st != RFX_ERR_UNSUPPORTED) return st;
  ScanLaunch a{&p, in, n, out, nullptr, nullptr, nullptr, err, as_stream(stream)};
  return dispatch_compact(p.in_bytes, 2, p.out_bytes, a);
}
}  // namespace

extern "C" rfx_status rfx_arith(void* out, const void* in, uint64_t n, const rfx_tuple* in_type,
                                const rfx_arith_expr* arith, void* stream) {
  if (!in_type || !arith || in_type->nfields >= 16) return RFX_ERR_INVALID;
  ScanProgram p;
  rfx_status st = compile_scan(&p, in_type, nullptr, 0, arith, 1);
  if (st != RFX_OK) return st;
  // the result tuple: the source fields followed by the new one (set_arith)
  rfx_tuple ot = *in_type;
  ot.widths[ot.nfields++] = arith->dest_bits;
  uint32_t map[16];
  for (uint32_t k = 0; k < ot.nfields; ++k) map[k] = k;
  st = compile_projection(&p, &ot, map);
  if (st != RFX_OK) return st;
  return run_map(p, out, in, n, stream);
}

extern "C" rfx_status rfx_project(void* out, const void* in, uint64_t n, const rfx_tuple* in_type,
                                  const rfx_tuple* out_type, const uint32_t* map, void* stream) {
  ScanProgram p;
  rfx_status st = compile_scan(&p, in_type, nullptr, 0, nullptr, 0);
  if (st != RFX_OK) return st;
  st = compile_projection(&p, out_type, map);
  if (st != RFX_OK) return st;
  return run_map(p, out, in, n, stream);
}

extern "C" size_t rfx_filter_aggregate_workspace(uint64_t n, const rfx_tuple* in_type,
                                                 const uint32_t* group_domain, uint32_t ngroup,
                                                 uint32_t nsum) {
  (void)n;
  (void)in_type;
  uint64_t g = 1;
  for (uint32_t k = 0; k < ngroup && group_domain; ++k) g *= group_domain[k] ? group_domain[k] : 1;
  if (g > (uint64_t)kMaxGroups) g = kMaxGroups;
  Carver c(nullptr);
  c.take<unsigned long long>(g * (nsum + 1));
  c.take<uint32_t>(1);
  return align_up(c.used, 256);
}

extern "C" rfx_status rfx_filter_aggregate(const void* in, uint64_t n, const rfx_tuple* in_type,
                                           const rfx_cmp* cmps, uint32_t ncmp,
                                           const rfx_arith_expr* ariths, uint32_t narith,
                                           const uint32_t* group_fields, const uint32_t* group_domain,
                                           uint32_t ngroup, const uint32_t* sum_fields, uint32_t nsum,
                                           uint64_t* out_keys, int64_t* out_sums, uint64_t* out_counts,
                                           uint64_t* d_groups, void* workspace, size_t workspace_bytes,
                                           void* stream) {
  if ((!in && n) || !out_keys || !out_counts || !d_groups || (nsum && !out_sums)) return RFX_ERR_INVALID;
  ScanProgram p;
  rfx_status st = compile_scan(&p, in_type, cmps, ncmp, ariths, narith);
  if (st != RFX_OK) return st;
  st = compile_aggregate(&p, group_fields, group_domain, ngroup, sum_fields, nsum);
  if (st != RFX_OK) return st;
  if (n && !aligned(in, p.in_bytes)) return RFX_ERR_INVALID;
  cudaStream_t s = as_stream(stream);
  uint32_t* err = device_error_word();
  if (!err) return RFX_ERR_CUDA;
  Carver c(workspace);
  unsigned long long* gacc = c.take<unsigned long long>((size_t)p.ngroups_total * (nsum + 1));
  uint32_t* done = c.take<uint32_t>(1);
  if (!workspace || workspace_bytes < c.used) return RFX_ERR_WORKSPACE;
  // the plan-specialised kernel (rows per thread per iteration tuned per plan shape and
  // size class when tuning is on), else the interpreting kernel
  const size_t clear = c.used;
  auto run = [&](int v) -> rfx_status {
    RFX_CUDA_TRY(cudaMemsetAsync(workspace, 0, clear, s));
    return jit_aggregate(p, in, n, gacc, done, out_keys, out_sums, out_counts, d_groups, err, s, v);
  };
  const uint64_t shape = ((uint64_t)p.in_bytes << 40) | ((uint64_t)p.ngroups_total << 16) | ((uint64_t)nsum << 8) |
                         p.ncmp;
  st = run(tune_pick(TUNE_SCAN_AGGREGATE, shape, n, 3, run, s));
  if (st != RFX_ERR_UNSUPPORTED) return st;
  RFX_CUDA_TRY(cudaMemsetAsync(workspace, 0, clear, s));
  AggLaunch a{&p, in, n, gacc, done, out_keys, out_sums, out_counts, d_groups, err, s};
  return dispatch_aggregate(p.in_bytes, a);
}

// ------------------------------------------------------------------ synthetic rows
namespace rfx {
namespace {

struct GenDesc {
  uint32_t nfields;
  uint32_t bytes;
  FieldLoc loc[16];
  uint64_t lo[16];
  uint64_t span[16];
  uint64_t base[16];  // per-column stream base
};

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

template <int W>
__global__ void gen_rows_kernel(const __grid_constant__ GenDesc d, uint8_t* out, uint64_t n) {
  constexpr int NL = Limbs<W>::N;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t L[NL];
#pragma unroll
    for (int l = 0; l < NL; ++l) L[l] = 0;
    for (uint32_t f = 0; f < d.nfields; ++f) {
      const uint64_t r = mix64(d.base[f] + (i + 1) * 0x9E3779B97F4A7C15ull);
      const uint64_t v = d.lo[f] + __umul64hi(r, d.span[f]);
      const FieldLoc fl = d.loc[f];
      const uint64_t m = fl.width >= 64 ? ~0ull : ((1ull << fl.width) - 1);
#pragma unroll
      for (int l = 0; l < NL; ++l) {
        if (l == fl.limb) L[l] |= (v & m) << fl.off;
        if (l == fl.limb + 1 && fl.off && fl.off + fl.width > 64) L[l] |= (v & m) >> (64 - fl.off);
      }
    }
    store_row<W>(out, i, L);
  }
}

uint64_t host_mix64(uint64_t x) {
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

}  // namespace
}  // namespace rfx

extern "C" rfx_status rfx_gen_uniform_rows(void* out, uint64_t n, const rfx_tuple* type, uint64_t seed,
                                           const uint64_t* lo, const uint64_t* hi, void* stream) {
  if (!type || !lo || !hi || (!out && n)) return RFX_ERR_INVALID;
  if (n && (reinterpret_cast<uintptr_t>(out) % 16) != 0) return RFX_ERR_INVALID;
  GenDesc d;
  std::memset(&d, 0, sizeof(d));
  rfx_status st = compile_tuple(type, d.loc, &d.bytes, nullptr);
  if (st != RFX_OK) return st;
  d.nfields = type->nfields;
  for (uint32_t f = 0; f < d.nfields; ++f) {
    if (hi[f] < lo[f]) return RFX_ERR_INVALID;
    d.lo[f] = lo[f];
    d.span[f] = hi[f] - lo[f];
    // column f is SplitMix64 stream f of `seed`
    d.base[f] = host_mix64(seed ^ ((uint64_t)f * 0xD1B54A32D192ED03ull));
  }
  if (n == 0) return RFX_OK;
  cudaStream_t s = as_stream(stream);
  const int threads = 256;
  const uint64_t want = (n + threads - 1) / threads;
  const int grid = (int)(want < (uint64_t)device_sms() * 8 ? want : (uint64_t)device_sms() * 8);
  switch (d.bytes) {
    case 1: gen_rows_kernel<1><<<grid, threads, 0, s>>>(d, (uint8_t*)out, n); break;
    case 2: gen_rows_kernel<2><<<grid, threads, 0, s>>>(d, (uint8_t*)out, n); break;
    case 4: gen_rows_kernel<4><<<grid, threads, 0, s>>>(d, (uint8_t*)out, n); break;
    case 8: gen_rows_kernel<8><<<grid, threads, 0, s>>>(d, (uint8_t*)out, n); break;
    case 16: gen_rows_kernel<16><<<grid, threads, 0, s>>>(d, (uint8_t*)out, n); break;
    case 32: gen_rows_kernel<32><<<grid, threads, 0, s>>>(d, (uint8_t*)out, n); break;
    case 64: gen_rows_kernel<64><<<grid, threads, 0, s>>>(d, (uint8_t*)out, n); break;
    default: return RFX_ERR_UNSUPPORTED;
  }
  RFX_CUDA_TRY(cudaGetLastError());
  return RFX_OK;
}
