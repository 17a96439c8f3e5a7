// merge_abi.cu -- packs an aggregate's key and value columns back into tuples: the merge
// step that closes the reference's aggregation sequence (the merge kernel addAgg emits,
// RelationalAlgebraCompiler.cpp:8536-8643, i.e. ra::cuda::merge / mergeElement of
// Split_Merge.h:442-495), out[i] = key[i] << value_bits | (value[i] & mask(value_bits)).
#include "host_common.h"
#include "rfx_device.cuh"

namespace rfx {
namespace {

struct U128 {
  unsigned long long lo, hi;
};

template <int KB>
__device__ __forceinline__ U128 load_col(const uint8_t* p, uint64_t i) {
  if constexpr (KB == 4) return U128{reinterpret_cast<const uint32_t*>(p)[i], 0ull};
  if constexpr (KB == 8) return U128{reinterpret_cast<const unsigned long long*>(p)[i], 0ull};
  if constexpr (KB == 16) {
    const ulonglong2 v = reinterpret_cast<const ulonglong2*>(p)[i];
    return U128{v.x, v.y};
  }
  return U128{0ull, 0ull};
}

template <int OB, int KB, int VB>
__global__ void merge_kernel(uint8_t* out, uint64_t n, const uint64_t* d_n, const uint8_t* keys, const uint8_t* vals,
                             uint32_t value_bits) {
  const uint64_t m = d_n ? (*d_n < n ? *d_n : n) : n;
  const unsigned long long vmask = value_bits >= 64 ? ~0ull : ((1ull << value_bits) - 1);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
    const U128 k = load_col<KB>(keys, i);
    const unsigned long long v = value_bits ? load_col<VB>(vals, i).lo & vmask : 0ull;
    U128 r;
    if (value_bits == 0) {
      r = k;
    } else if (value_bits >= 64) {
      r.lo = v;
      r.hi = k.lo;
    } else {
      r.lo = (k.lo << value_bits) | v;
      r.hi = (k.hi << value_bits) | (k.lo >> (64 - value_bits));
    }
    if constexpr (OB == 4) reinterpret_cast<uint32_t*>(out)[i] = (uint32_t)r.lo;
    if constexpr (OB == 8) reinterpret_cast<unsigned long long*>(out)[i] = r.lo;
    if constexpr (OB == 16) reinterpret_cast<ulonglong2*>(out)[i] = make_ulonglong2(r.lo, r.hi);
  }
}

template <int OB, int KB>
rfx_status launch_v(uint32_t vb, uint8_t* out, uint64_t n, const uint64_t* d_n, const uint8_t* k, const uint8_t* v,
                    uint32_t bits, int grid, cudaStream_t s) {
  if (vb == 4)
    merge_kernel<OB, KB, 4><<<grid, 256, 0, s>>>(out, n, d_n, k, v, bits);
  else
    merge_kernel<OB, KB, 8><<<grid, 256, 0, s>>>(out, n, d_n, k, v, bits);
  RFX_CUDA_TRY(cudaGetLastError());
  return RFX_OK;
}

template <int OB>
rfx_status launch_k(uint32_t kb, uint32_t vb, uint8_t* out, uint64_t n, const uint64_t* d_n, const uint8_t* k,
                    const uint8_t* v, uint32_t bits, int grid, cudaStream_t s) {
  switch (kb) {
    case 4: return launch_v<OB, 4>(vb, out, n, d_n, k, v, bits, grid, s);
    case 8: return launch_v<OB, 8>(vb, out, n, d_n, k, v, bits, grid, s);
    default: return launch_v<OB, 16>(vb, out, n, d_n, k, v, bits, grid, s);
  }
}

bool ok_width(uint32_t b) { return b == 4 || b == 8 || b == 16; }

}  // namespace
}  // namespace rfx

using namespace rfx;

extern "C" rfx_status rfx_merge_columns(void* out, uint32_t out_bytes, uint64_t n, const uint64_t* d_n,
                                        const void* keys, uint32_t key_bytes, const void* values,
                                        uint32_t value_bytes, uint32_t value_bits, void* stream) {
  if (!ok_width(out_bytes) || !ok_width(key_bytes) || (value_bytes != 4 && value_bytes != 8) ||
      value_bits > value_bytes * 8u)
    return RFX_ERR_UNSUPPORTED;
  if (n == 0) return RFX_OK;
  if (!out || !keys || (value_bits && !values)) return RFX_ERR_INVALID;
  const uint64_t blocks = (n + 255) / 256, cap = (uint64_t)device_sms() * 8;
  const int grid = (int)(blocks < cap ? blocks : cap);
  uint8_t* o = static_cast<uint8_t*>(out);
  const uint8_t* k = static_cast<const uint8_t*>(keys);
  const uint8_t* v = static_cast<const uint8_t*>(values);
  cudaStream_t s = as_stream(stream);
  switch (out_bytes) {
    case 4: return launch_k<4>(key_bytes, value_bytes, o, n, d_n, k, v, value_bits, grid, s);
    case 8: return launch_k<8>(key_bytes, value_bytes, o, n, d_n, k, v, value_bits, grid, s);
    default: return launch_k<16>(key_bytes, value_bytes, o, n, d_n, k, v, value_bits, grid, s);
  }
}
