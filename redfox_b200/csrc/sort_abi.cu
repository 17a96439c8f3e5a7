// sort_abi.cu -- C ABI of the radix sort, including the reference-compatible
// b40c / moderngpu entries.
#include <algorithm>
#include <cstring>

#include "sort_launch.cuh"

namespace rfx {

template <int K>
rfx_status run_sort(SortPlan&, uint32_t);
template <int K>
uint64_t sort_tiles_for(uint64_t, uint32_t);

namespace {

bool valid_width(uint32_t k) { return k == 1 || k == 2 || k == 4 || k == 8 || k == 16 || k == 32 || k == 64; }
bool valid_vwidth(uint32_t v) { return v == 0 || v == 1 || v == 2 || v == 4 || v == 8 || v == 16; }

uint64_t tiles_for(uint32_t kb, uint64_t n, uint32_t vb) {
  switch (kb) {
    case 1: return sort_tiles_for<1>(n, vb);
    case 2: return sort_tiles_for<2>(n, vb);
    case 4: return sort_tiles_for<4>(n, vb);
    case 8: return sort_tiles_for<8>(n, vb);
    case 16: return sort_tiles_for<16>(n, vb);
    case 32: return sort_tiles_for<32>(n, vb);
    default: return sort_tiles_for<64>(n, vb);
  }
}

rfx_status dispatch(uint32_t kb, SortPlan& s, uint32_t vb) {
  switch (kb) {
    case 1: return run_sort<1>(s, vb);
    case 2: return run_sort<2>(s, vb);
    case 4: return run_sort<4>(s, vb);
    case 8: return run_sort<8>(s, vb);
    case 16: return run_sort<16>(s, vb);
    case 32: return run_sort<32>(s, vb);
    case 64: return run_sort<64>(s, vb);
    default: return RFX_ERR_UNSUPPORTED;
  }
}

struct SortLayout {
  uint8_t* alt_keys;
  uint8_t* alt_vals;
  uint8_t* alt2_keys;   // with 3 or more digit passes: lets an odd number of passes end in
  uint8_t* alt2_vals;   // the caller's buffers instead of being copied back
  uint32_t* ctrl;  // ghist | trivial | done | counters
  uint32_t* status;
  size_t ctrl_bytes;  // bytes to clear per chunk (ctrl + status)
  size_t total;
  uint64_t tiles;
  uint32_t passes;
};

SortLayout layout(void* ws, uint64_t n, uint32_t kb, uint32_t vb, uint32_t begin_bit, uint32_t end_bit) {
  SortLayout L;
  const uint32_t bits = end_bit - begin_bit;
  L.passes = std::min<uint32_t>((std::min<uint32_t>(bits, 128) + 7) / 8, kMaxSortPasses);
  L.tiles = tiles_for(kb, n, vb);
  Carver c(ws);
  L.alt_keys = c.take<uint8_t>(n * kb);
  L.alt_vals = c.take<uint8_t>(vb ? n * vb : 0);
  const bool second = L.passes >= 3;
  L.alt2_keys = second ? c.take<uint8_t>(n * kb) : nullptr;
  L.alt2_vals = second && vb ? c.take<uint8_t>(n * vb) : nullptr;
  c.used = align_up(c.used, 256);
  const size_t ctrl_start = c.used;
  L.ctrl = c.take<uint32_t>(kMaxSortPasses * kRadix + 2 * kMaxSortPasses + 1);
  L.status = c.take<uint32_t>((size_t)L.passes * L.tiles * kRadix);
  L.ctrl_bytes = c.used - ctrl_start;
  L.total = align_up(c.used, 256);
  return L;
}

thread_local uint32_t t_host_trivial[kMaxSortPasses];

}  // namespace

rfx_status sort_pairs_impl(void* keys, void* vals, uint64_t n, uint32_t kb, uint32_t vb, uint32_t begin_bit,
                           uint32_t end_bit, void* ws, size_t ws_bytes, cudaStream_t stream, bool skip_trivial,
                           int* passes_run, const void* src_keys = nullptr, const void* src_vals = nullptr) {
  if (passes_run) *passes_run = 0;
  if (!valid_width(kb) || !valid_vwidth(vb)) return RFX_ERR_UNSUPPORTED;
  if (end_bit > kb * 8 || begin_bit > end_bit) return RFX_ERR_INVALID;
  if (src_keys && (n == 0 || !keys || (vb && (!vals || !src_vals)))) return n == 0 ? RFX_OK : RFX_ERR_INVALID;
  if (src_keys && (n <= 1 || begin_bit == end_bit)) {
    // nothing to order: the output is a copy of the input
    RFX_CUDA_TRY(cudaMemcpyAsync(keys, src_keys, n * kb, cudaMemcpyDeviceToDevice, stream));
    if (vb) RFX_CUDA_TRY(cudaMemcpyAsync(vals, src_vals, n * vb, cudaMemcpyDeviceToDevice, stream));
    return RFX_OK;
  }
  if (n <= 1 || begin_bit == end_bit) return RFX_OK;
  if (n >= (1ull << 30)) return RFX_ERR_UNSUPPORTED;  // 30-bit look-back counts
  if (!keys || (vb && !vals)) return RFX_ERR_INVALID;
  if (reinterpret_cast<uintptr_t>(keys) % std::min<uint32_t>(kb, 16) ||
      (vb && reinterpret_cast<uintptr_t>(vals) % std::min<uint32_t>(vb, 16)))
    return RFX_ERR_INVALID;
  if (src_keys && (reinterpret_cast<uintptr_t>(src_keys) % std::min<uint32_t>(kb, 16) ||
                   (vb && reinterpret_cast<uintptr_t>(src_vals) % std::min<uint32_t>(vb, 16))))
    return RFX_ERR_INVALID;
  if (src_keys) {
    // source and destination must not overlap
    const uintptr_t a = reinterpret_cast<uintptr_t>(src_keys), b = reinterpret_cast<uintptr_t>(keys);
    if (a < b + n * kb && b < a + n * kb) return RFX_ERR_INVALID;
    if (vb) {
      const uintptr_t c = reinterpret_cast<uintptr_t>(src_vals), d = reinterpret_cast<uintptr_t>(vals);
      if (c < d + n * vb && d < c + n * vb) return RFX_ERR_INVALID;
    }
  }
  SortLayout L = layout(ws, n, kb, vb, begin_bit, end_bit);
  if (!ws || ws_bytes < L.total) return RFX_ERR_WORKSPACE;
  uint32_t* err = device_error_word();
  if (!err) return RFX_ERR_CUDA;
  uint8_t* cur_k = static_cast<uint8_t*>(keys);
  uint8_t* cur_v = static_cast<uint8_t*>(vals);
  uint8_t* oth_k = L.alt_keys;
  uint8_t* oth_v = vb ? L.alt_vals : nullptr;
  // LSD order across 128-bit chunks: each chunk is a stable sort on its bits
  for (uint32_t lo = begin_bit; lo < end_bit; lo += 128) {
    const uint32_t hi = std::min(end_bit, lo + 128);
    RFX_CUDA_TRY(cudaMemsetAsync(L.ctrl, 0, L.ctrl_bytes, stream));
    SortPlan s;
    std::memset(&s, 0, sizeof(s));
    s.keys = cur_k;
    s.vals = cur_v;
    const bool from_src = src_keys && lo == begin_bit;   // the first 128-bit chunk reads the source
    s.src_keys = from_src ? static_cast<const uint8_t*>(src_keys) : nullptr;
    s.src_vals = from_src && vb ? static_cast<const uint8_t*>(src_vals) : nullptr;
    s.alt_keys = oth_k;
    s.alt_vals = oth_v;
    s.alt2_keys = L.alt2_keys;
    s.alt2_vals = L.alt2_vals;
    s.n = n;
    s.begin_bit = lo;
    s.end_bit = hi;
    s.passes = (hi - lo + 7) / 8;
    s.ghist = L.ctrl;
    s.trivial = L.ctrl + kMaxSortPasses * kRadix;
    s.done = s.trivial + kMaxSortPasses;
    s.counters = s.done + 1;
    s.status = L.status;
    s.tiles = L.tiles;
    s.skip_trivial = skip_trivial;
    s.host_trivial = t_host_trivial;
    s.err = err;
    s.stream = stream;
    rfx_status st = dispatch(kb, s, vb);
    if (st != RFX_OK) return st;
    if (passes_run) *passes_run += s.executed;
    if (from_src && s.executed == 0) {
      // every pass was trivial: the output is a copy of the input
      RFX_CUDA_TRY(cudaMemcpyAsync(cur_k, src_keys, n * kb, cudaMemcpyDeviceToDevice, stream));
      if (vb) RFX_CUDA_TRY(cudaMemcpyAsync(cur_v, src_vals, n * vb, cudaMemcpyDeviceToDevice, stream));
    }
    if (s.in_alt) {
      std::swap(cur_k, oth_k);
      std::swap(cur_v, oth_v);
    }
  }
  if (cur_k != keys) {
    RFX_CUDA_TRY(cudaMemcpyAsync(keys, cur_k, n * kb, cudaMemcpyDeviceToDevice, stream));
    if (vb) RFX_CUDA_TRY(cudaMemcpyAsync(vals, cur_v, n * vb, cudaMemcpyDeviceToDevice, stream));
  }
  return RFX_OK;
}

size_t sort_workspace_impl(uint64_t n, uint32_t kb, uint32_t vb, uint32_t begin_bit, uint32_t end_bit) {
  if (!valid_width(kb) || !valid_vwidth(vb) || end_bit <= begin_bit) return 256;
  return layout(nullptr, n, kb, vb, begin_bit, end_bit).total;
}

namespace {

// Bytes of the element for a DataType code (RelationalAlgebraKernel.h:81-95).
uint32_t type_bytes(uint64_t type) {
  switch (type) {
    case RFX_I8: return 1;
    case RFX_I16: return 2;
    case RFX_I32: return 4;
    case RFX_I64: return 8;
    case RFX_I128: return 16;
    case RFX_I256: return 32;
    case RFX_I512: return 64;
    default: return 0;
  }
}

// The b40c entries pick the key container from the key bits (b40cSort.cu:85-1005).
uint32_t bits_container(uint64_t bits) { return bits <= 8 ? 1 : bits <= 16 ? 2 : bits <= 32 ? 4 : bits <= 64 ? 8 : 0; }

// The reference-compatible entries own their scratch and finish before returning,
// like the reference (which cudaMallocs its pong buffers and synchronises per call).
rfx_status sort_sync(void* keys, void* vals, uint64_t n, uint32_t kb, uint32_t vb, uint32_t begin, uint32_t end) {
  if (n <= 1) return RFX_OK;
  cudaStream_t s = 0;
  const size_t need = sort_workspace_impl(n, kb, vb, begin, end);
  void* ws = nullptr;
  RFX_CUDA_TRY(cudaMallocAsync(&ws, need, s));
  rfx_status st = sort_pairs_impl(keys, vals, n, kb, vb, begin, end, ws, need, s, true, nullptr);
  cudaError_t e = cudaFreeAsync(ws, s);
  if (st != RFX_OK) return st;
  RFX_CUDA_TRY(e);
  RFX_CUDA_TRY(cudaStreamSynchronize(s));
  return RFX_OK;
}

}  // namespace
}  // namespace rfx

using namespace rfx;

extern "C" size_t rfx_sort_workspace(uint64_t n, uint32_t key_bytes, uint32_t value_bytes, uint32_t begin_bit,
                                     uint32_t end_bit) {
  return sort_workspace_impl(n, key_bytes, value_bytes, begin_bit, end_bit);
}

extern "C" rfx_status rfx_sort_pairs(void* keys, void* values, uint64_t n, uint32_t key_bytes, uint32_t value_bytes,
                                     uint32_t begin_bit, uint32_t end_bit, uint32_t flags, void* workspace,
                                     size_t workspace_bytes, void* stream) {
  return sort_pairs_impl(keys, values, n, key_bytes, value_bytes, begin_bit, end_bit, workspace, workspace_bytes,
                         as_stream(stream), (flags & RFX_SORT_SKIP_TRIVIAL) != 0, nullptr);
}

extern "C" rfx_status rfx_sort_pairs_from(const void* keys_in, const void* values_in, void* keys, void* values,
                                          uint64_t n, uint32_t key_bytes, uint32_t value_bytes, uint32_t begin_bit,
                                          uint32_t end_bit, uint32_t flags, void* workspace, size_t workspace_bytes,
                                          void* stream) {
  if (n && !keys_in) return RFX_ERR_INVALID;
  return sort_pairs_impl(keys, values, n, key_bytes, value_bytes, begin_bit, end_bit, workspace, workspace_bytes,
                         as_stream(stream), (flags & RFX_SORT_SKIP_TRIVIAL) != 0, nullptr, keys_in, values_in);
}

extern "C" rfx_status rfx_b40c_sort_pair(void* keys, void* values, uint64_t n, uint64_t key_bits, uint64_t value_type) {
  const uint32_t kb = bits_container(key_bits), vb = type_bytes(value_type);
  if (!kb || !vb || vb > 16 || key_bits == 0) return RFX_ERR_UNSUPPORTED;
  return sort_sync(keys, values, n, kb, vb, 0, (uint32_t)key_bits);
}

extern "C" rfx_status rfx_b40c_sort_key(void* keys, uint64_t n, uint64_t bits) {
  const uint32_t kb = bits_container(bits);
  if (!kb || bits == 0) return RFX_ERR_UNSUPPORTED;
  return sort_sync(keys, nullptr, n, kb, 0, 0, (uint32_t)bits);
}

extern "C" rfx_status rfx_mgpu_sort_pair(void* keys, void* values, uint64_t n, uint64_t key_type, uint64_t value_type) {
  const uint32_t kb = type_bytes(key_type), vb = type_bytes(value_type);
  if (!kb || !vb || vb > 16) return RFX_ERR_UNSUPPORTED;
  return sort_sync(keys, values, n, kb, vb, 0, kb * 8);
}

extern "C" rfx_status rfx_mgpu_sort_key(void* keys, uint64_t n, uint64_t key_type) {
  const uint32_t kb = type_bytes(key_type);
  if (!kb) return RFX_ERR_UNSUPPORTED;
  return sort_sync(keys, nullptr, n, kb, 0, 0, kb * 8);
}
