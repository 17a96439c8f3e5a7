// strings_abi.cu -- string-keyed operators.  A string column is an array of 64-bit device
// pointers to NUL-terminated strings, as in the reference (ModernGPUSort.cu:44-67,
// ModernGPUJoin.cu:44-100, Reduce.cu:30-53).  Order: lexicographic on `char` (signed),
// a proper prefix first; equality: the same characters.
//
// Every operator works on dictionary codes.  string_codes gives each element the dense
// rank of its string among the distinct strings of the column (equal strings, equal codes;
// code order = string order) and the stable sorted permutation, by multikey refinement:
// each round reads the next 7 characters of every string not yet ended into a 63-bit
// chunk (9 bits per character: NUL -> 0, then the signed byte order), radix-sorts rows
// (code, chunk, index) on (code, chunk), and re-ranks the rows by (code, chunk).  Rounds
// stop when no group of equal codes holds a string that has not ended; such groups then
// hold equal strings only.  A string is never read past its terminator.  The integer
// kernels then do the work: the sort gathers by the permutation, find_bounds runs on the
// codes of both sides coded together, count reduces runs of equal codes.
#include <cstring>

#include "host_common.h"
#include "rfx_device.cuh"

namespace rfx {

size_t find_bounds_workspace_impl(uint64_t nl);
rfx_status find_bounds_impl(int32_t* lb, int32_t* scan, uint64_t* d_total, const void* left, uint64_t nl,
                            const void* right, uint64_t nr, uint32_t kb, void* ws, size_t wsb, cudaStream_t s);

namespace {

constexpr int kStrThreads = 256;
constexpr int kStrIPT = 4;
constexpr int kStrTile = kStrThreads * kStrIPT;
constexpr uint32_t kChunkBit = 33;  // rows sort on bits [33, 96 + code bits)

// A refinement row, 16 bytes, limb 0 low: bits 0..31 element index, 33..95 chunk (the
// next 7 characters), 96..127 code (rank of the string's prefix read so far).
struct StrRow {
  unsigned long long lo, hi;
};

__device__ __forceinline__ uint32_t row_idx(const StrRow& r) { return (uint32_t)r.lo; }
__device__ __forceinline__ bool row_key_eq(const StrRow& a, const StrRow& b) {
  return a.hi == b.hi && (a.lo >> kChunkBit) == (b.lo >> kChunkBit);
}

__device__ __forceinline__ uint64_t gtid() { return (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint64_t gstride() { return (uint64_t)gridDim.x * blockDim.x; }

__global__ void str_init(StrRow* rows, uint64_t n, uint8_t* ended) {
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    rows[i].lo = (unsigned long long)(uint32_t)i;
    rows[i].hi = 0;
    ended[i] = 0;
  }
}

// The characters [offset, offset + 7) of every row's string into its chunk; ended strings
// read nothing and get chunk 0.
__global__ void str_fill(StrRow* rows, uint64_t n, const unsigned long long* ptrs, uint8_t* ended, uint64_t offset) {
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    StrRow r = rows[i];
    const uint32_t idx = row_idx(r);
    unsigned long long chunk = 0;
    if (!ended[idx]) {
      const signed char* p = reinterpret_cast<const signed char*>(ptrs[idx]) + offset;
      bool done = false;
#pragma unroll
      for (int c = 0; c < 7; ++c) {
        unsigned long long rank = 0;
        if (!done) {
          const signed char ch = p[c];
          if (ch == 0)
            done = true;
          else
            rank = (unsigned long long)((int)ch + 129);  // -128..127 -> 1..256
        }
        chunk |= rank << (9 * (6 - c));
      }
      if (done) ended[idx] = 1;
    }
    r.lo = (r.lo & 0xffffffffull) | (chunk << kChunkBit);
    r.hi = (r.hi & 0xffffffff00000000ull) | (chunk >> (64 - kChunkBit));
    rows[i] = r;
  }
}

// heads[i] = 1 where row i's (code, chunk) differs from row i-1's.
__global__ void str_heads(const StrRow* rows, uint64_t n, uint8_t* heads) {
  for (uint64_t i = gtid(); i < n; i += gstride()) heads[i] = i == 0 || !row_key_eq(rows[i], rows[i - 1]);
}

// heads[i] = 1 where codes[i] differs from codes[i-1].
__global__ void code_heads(const uint32_t* codes, uint64_t n, uint8_t* heads) {
  for (uint64_t i = gtid(); i < n; i += gstride()) heads[i] = i == 0 || codes[i] != codes[i - 1];
}

// Writes the run index as the row's new code.
struct SetCode {
  StrRow* rows;
  __device__ void operator()(uint64_t i, uint64_t run, uint32_t) const {
    rows[i].hi = (rows[i].hi & 0xffffffffull) | ((unsigned long long)(uint32_t)run << 32);
  }
};

// Writes the first key pointer of every run.
struct FirstKey {
  const unsigned long long* keys;
  unsigned long long* out;
  __device__ void operator()(uint64_t i, uint64_t run, uint32_t head) const {
    if (head) out[run] = keys[i];
  }
};

// Run index of every element (inclusive scan of heads, minus one) by decoupled look-back
// over tiles of kStrTile; calls f(i, run, head) for each element and writes the number of
// runs to *d_runs.
template <typename F>
__global__ void __launch_bounds__(kStrThreads) head_scan(uint64_t n, const uint8_t* heads, uint64_t* status,
                                                          uint32_t* tile_counter, uint64_t* d_runs, uint32_t* err,
                                                          F f) {
  __shared__ uint32_t s_warp[kStrThreads / 32];
  __shared__ uint64_t s_pre;
  __shared__ uint32_t s_tile;
  const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const uint64_t tiles = (n + kStrTile - 1) / kStrTile;
  while (true) {
    if (t == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    if (tile >= tiles) break;
    const uint64_t first = tile * kStrTile + (uint64_t)t * kStrIPT;
    uint32_t h[kStrIPT], cnt = 0;
#pragma unroll
    for (int j = 0; j < kStrIPT; ++j) {
      h[j] = first + j < n ? heads[first + j] : 0u;
      cnt += h[j];
    }
    uint32_t incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o) incl += v;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    uint32_t wpre = 0, tot = 0;
#pragma unroll
    for (uint32_t w = 0; w < kStrThreads / 32; ++w) {
      if (w < warp) wpre += s_warp[w];
      tot += s_warp[w];
    }
    if (warp == 0) {
      const uint64_t pre = lookback_exclusive(status, (uint32_t)tile, tot, err);
      if (t == 0) {
        s_pre = pre;
        if (tile == tiles - 1) *d_runs = pre + tot;
      }
    }
    __syncthreads();
    uint64_t run = s_pre + wpre + incl - cnt;
#pragma unroll
    for (int j = 0; j < kStrIPT; ++j) {
      const uint64_t i = first + j;
      if (i < n) {
        run += h[j];
        f(i, run - 1, h[j]);
      }
    }
    __syncthreads();
  }
}

// *flag = 1 if a string that has not ended shares its (code, chunk) with another row.
__global__ void str_unresolved(const StrRow* rows, uint64_t n, const uint8_t* heads, const uint8_t* ended,
                               uint32_t* flag) {
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    if (ended[row_idx(rows[i])]) continue;
    if (!heads[i] || (i + 1 < n && !heads[i + 1])) *flag = 1;
  }
}

__global__ void str_scatter(const StrRow* rows, uint64_t n, uint32_t* codes, uint32_t* perm) {
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    const uint32_t idx = row_idx(rows[i]);
    if (codes) codes[idx] = (uint32_t)(rows[i].hi >> 32);
    if (perm) perm[i] = idx;
  }
}

// out[i] = in[perm[i]] for elements of W bytes (W a multiple of 8: limb copies).
template <int W>
__global__ void gather_limbs(unsigned long long* out, const unsigned long long* in, const uint32_t* perm, uint64_t n) {
  constexpr int L = W / 8;
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    const uint64_t src = (uint64_t)perm[i] * L;
#pragma unroll
    for (int l = 0; l < L; ++l) out[i * L + l] = in[src + l];
  }
}

template <typename T>
__global__ void gather_small(T* out, const T* in, const uint32_t* perm, uint64_t n) {
  for (uint64_t i = gtid(); i < n; i += gstride()) out[i] = in[perm[i]];
}

int grid_for(uint64_t n) {
  const uint64_t b = (n + 255) / 256;
  const uint64_t cap = (uint64_t)device_sms() * 8;
  return (int)(b < cap ? (b ? b : 1) : cap);
}

// Stream-ordered scratch freed on scope exit.
struct DevBuf {
  void* p = nullptr;
  cudaStream_t s = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (p) cudaFreeAsync(p, s);
  }
  rfx_status alloc(size_t bytes, cudaStream_t st) {
    s = st;
    RFX_CUDA_TRY(cudaMallocAsync(&p, bytes ? bytes : 16, st));
    return RFX_OK;
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// Look-back words for head_scan over n elements, plus its tile counter (zeroed).
struct ScanState {
  DevBuf buf;
  uint64_t tiles = 0;
  rfx_status init(uint64_t n, cudaStream_t s) {
    tiles = (n + kStrTile - 1) / kStrTile;
    rfx_status st = buf.alloc(tiles * 8 + 64, s);
    if (st != RFX_OK) return st;
    return reset(s);
  }
  rfx_status reset(cudaStream_t s) {
    RFX_CUDA_TRY(cudaMemsetAsync(buf.p, 0, tiles * 8 + 64, s));
    return RFX_OK;
  }
  uint64_t* status() const { return buf.as<uint64_t>(); }
  uint32_t* counter() const { return reinterpret_cast<uint32_t*>(buf.as<uint8_t>() + tiles * 8); }
};

template <typename F>
rfx_status launch_head_scan(uint64_t n, const uint8_t* heads, ScanState& ss, uint64_t* d_runs, uint32_t* err, F f,
                            cudaStream_t s) {
  const int grid = persistent_grid((const void*)head_scan<F>, kStrThreads, 0, ss.tiles);
  head_scan<F><<<grid, kStrThreads, 0, s>>>(n, heads, ss.status(), ss.counter(), d_runs, err, f);
  RFX_CUDA_TRY(cudaGetLastError());
  return RFX_OK;
}

uint32_t bit_length(uint64_t x) { return x ? 64u - (uint32_t)__builtin_clzll(x) : 0u; }

}  // namespace

// Dense codes of n strings (codes[i] for element i; may be null), the stable sorted
// permutation (perm[k] = the element at sorted position k; may be null) and the number of
// distinct strings (may be null).  Returns after the stream has drained (each round reads
// a flag back).
rfx_status string_codes(const unsigned long long* ptrs, uint64_t n, uint32_t* codes, uint32_t* perm,
                        uint64_t* ndistinct, cudaStream_t s) {
  if (ndistinct) *ndistinct = 0;
  if (n == 0) return RFX_OK;
  if (!ptrs) return RFX_ERR_INVALID;
  if (n >= (1ull << 30)) return RFX_ERR_UNSUPPORTED;  // radix sort limit
  uint32_t* err = device_error_word();
  if (!err) return RFX_ERR_CUDA;
  const size_t sws = rfx_sort_workspace(n, 16, 0, kChunkBit, 128);
  DevBuf rows, ended, heads, sortws, small;
  ScanState ss;
  rfx_status st;
  if ((st = rows.alloc(n * sizeof(StrRow), s)) != RFX_OK || (st = ended.alloc(n, s)) != RFX_OK ||
      (st = heads.alloc(n, s)) != RFX_OK || (st = sortws.alloc(sws, s)) != RFX_OK ||
      (st = small.alloc(64, s)) != RFX_OK || (st = ss.init(n, s)) != RFX_OK)
    return st;
  StrRow* R = rows.as<StrRow>();
  uint64_t* d_groups = small.as<uint64_t>();
  uint32_t* d_flag = reinterpret_cast<uint32_t*>(small.as<uint8_t>() + 16);
  const int g = grid_for(n);
  str_init<<<g, 256, 0, s>>>(R, n, ended.as<uint8_t>());
  RFX_CUDA_TRY(cudaGetLastError());
  uint64_t groups = 1;  // every code is 0 before the first round
  for (uint64_t offset = 0;; offset += 7) {
    str_fill<<<g, 256, 0, s>>>(R, n, ptrs, ended.as<uint8_t>(), offset);
    RFX_CUDA_TRY(cudaGetLastError());
    const uint32_t end_bit = 96 + bit_length(groups - 1);
    if ((st = rfx_sort_pairs(R, nullptr, n, 16, 0, kChunkBit, end_bit, 0, sortws.p, sws, s)) != RFX_OK) return st;
    str_heads<<<g, 256, 0, s>>>(R, n, heads.as<uint8_t>());
    RFX_CUDA_TRY(cudaGetLastError());
    if (offset && (st = ss.reset(s)) != RFX_OK) return st;
    if ((st = launch_head_scan(n, heads.as<uint8_t>(), ss, d_groups, err, SetCode{R}, s)) != RFX_OK) return st;
    RFX_CUDA_TRY(cudaMemsetAsync(d_flag, 0, sizeof(uint32_t), s));
    str_unresolved<<<g, 256, 0, s>>>(R, n, heads.as<uint8_t>(), ended.as<uint8_t>(), d_flag);
    RFX_CUDA_TRY(cudaGetLastError());
    uint32_t flag = 0;
    RFX_CUDA_TRY(cudaMemcpyAsync(&flag, d_flag, sizeof(flag), cudaMemcpyDeviceToHost, s));
    RFX_CUDA_TRY(cudaMemcpyAsync(&groups, d_groups, sizeof(groups), cudaMemcpyDeviceToHost, s));
    RFX_CUDA_TRY(cudaStreamSynchronize(s));
    uint32_t e = 0;
    RFX_CUDA_TRY(cudaMemcpy(&e, err, sizeof(e), cudaMemcpyDeviceToHost));
    if (e) return RFX_ERR_TIMEOUT;
    if (!flag) break;
  }
  str_scatter<<<g, 256, 0, s>>>(R, n, codes, perm);
  RFX_CUDA_TRY(cudaGetLastError());
  RFX_CUDA_TRY(cudaStreamSynchronize(s));
  if (ndistinct) *ndistinct = groups;
  return RFX_OK;
}

}  // namespace rfx

using namespace rfx;

extern "C" rfx_status rfx_string_codes(const void* ptrs, uint64_t n, uint32_t* codes, uint32_t* perm,
                                       uint64_t* ndistinct, void* stream) {
  return string_codes(static_cast<const unsigned long long*>(ptrs), n, codes, perm, ndistinct, as_stream(stream));
}

// redfox::sort_string_key / sort_string_pair (ModernGPUSort.cu:148-470, a stable merge
// sort by compare_sort_string) and redfox::sort_string (Sort.cu:176-195): the pointer
// column in string order, equal strings in input order; values (value_type, a DataType
// code I8..I512; 0 = no values) move with their keys.  Synchronous on the default stream.
extern "C" rfx_status rfx_sort_string_compat(void* keys, void* values, uint64_t n, uint64_t value_type) {
  if (n == 0) return RFX_OK;
  if (!keys) return RFX_ERR_INVALID;
  uint32_t vw = 0;
  if (value_type) {
    if (!values) return RFX_ERR_INVALID;
    switch (value_type) {
      case RFX_I8: vw = 1; break;
      case RFX_I16: vw = 2; break;
      case RFX_I32: vw = 4; break;
      case RFX_I64: vw = 8; break;
      case RFX_I128: vw = 16; break;
      case RFX_I256: vw = 32; break;
      case RFX_I512: vw = 64; break;
      default: return RFX_ERR_UNSUPPORTED;
    }
  }
  cudaStream_t s = 0;
  DevBuf perm, tmp;
  rfx_status st;
  if ((st = perm.alloc(n * 4, s)) != RFX_OK) return st;
  if ((st = string_codes(static_cast<const unsigned long long*>(keys), n, nullptr, perm.as<uint32_t>(), nullptr, s)) !=
      RFX_OK)
    return st;
  if ((st = tmp.alloc(n * (vw > 8 ? vw : 8), s)) != RFX_OK) return st;
  const int g = grid_for(n);
  const uint32_t* P = perm.as<uint32_t>();
  RFX_CUDA_TRY(cudaMemcpyAsync(tmp.p, keys, n * 8, cudaMemcpyDeviceToDevice, s));
  gather_limbs<8><<<g, 256, 0, s>>>(static_cast<unsigned long long*>(keys), tmp.as<unsigned long long>(), P, n);
  if (vw) {
    RFX_CUDA_TRY(cudaMemcpyAsync(tmp.p, values, n * vw, cudaMemcpyDeviceToDevice, s));
    auto* vo = static_cast<unsigned long long*>(values);
    const auto* vi = tmp.as<unsigned long long>();
    switch (vw) {
      case 1: gather_small<uint8_t><<<g, 256, 0, s>>>(static_cast<uint8_t*>(values), tmp.as<uint8_t>(), P, n); break;
      case 2: gather_small<uint16_t><<<g, 256, 0, s>>>(static_cast<uint16_t*>(values), tmp.as<uint16_t>(), P, n); break;
      case 4: gather_small<uint32_t><<<g, 256, 0, s>>>(static_cast<uint32_t*>(values), tmp.as<uint32_t>(), P, n); break;
      case 8: gather_limbs<8><<<g, 256, 0, s>>>(vo, vi, P, n); break;
      case 16: gather_limbs<16><<<g, 256, 0, s>>>(vo, vi, P, n); break;
      case 32: gather_limbs<32><<<g, 256, 0, s>>>(vo, vi, P, n); break;
      default: gather_limbs<64><<<g, 256, 0, s>>>(vo, vi, P, n); break;
    }
  }
  RFX_CUDA_TRY(cudaGetLastError());
  RFX_CUDA_TRY(cudaStreamSynchronize(s));
  return RFX_OK;
}

// redfox::find_bounds_string (ModernGPUJoin.cu:213-300): both pointer columns sorted by
// string; per left element the lower bound in the right column, the exclusive scan of
// the equal-string counts, and the total (*result_size, device), as the integer
// find_bounds_*.  Both columns are coded together so their codes compare.
extern "C" rfx_status rfx_find_bounds_string_compat(int32_t* lower_bound, int32_t* left_count, uint64_t* result_size,
                                                    const void* left_key, uint64_t left_size, const void* right_key,
                                                    uint64_t right_size) {
  if (!result_size || (left_size && (!lower_bound || !left_count || !left_key)) || (right_size && !right_key))
    return RFX_ERR_INVALID;
  if (left_size >= (1ull << 31) || right_size >= (1ull << 31)) return RFX_ERR_UNSUPPORTED;
  cudaStream_t s = 0;
  const uint64_t n = left_size + right_size;
  DevBuf both, codes, ws;
  rfx_status st;
  if ((st = both.alloc(n * 8, s)) != RFX_OK || (st = codes.alloc(n * 4, s)) != RFX_OK) return st;
  if (left_size) RFX_CUDA_TRY(cudaMemcpyAsync(both.p, left_key, left_size * 8, cudaMemcpyDeviceToDevice, s));
  if (right_size)
    RFX_CUDA_TRY(cudaMemcpyAsync(both.as<uint8_t>() + left_size * 8, right_key, right_size * 8,
                                 cudaMemcpyDeviceToDevice, s));
  if ((st = string_codes(both.as<unsigned long long>(), n, codes.as<uint32_t>(), nullptr, nullptr, s)) != RFX_OK)
    return st;
  const size_t need = find_bounds_workspace_impl(left_size);
  if ((st = ws.alloc(need, s)) != RFX_OK) return st;
  const uint32_t* c = codes.as<uint32_t>();
  if ((st = find_bounds_impl(lower_bound, left_count, result_size, c, left_size, c + left_size, right_size, 4, ws.p,
                             need, s)) != RFX_OK)
    return st;
  RFX_CUDA_TRY(cudaStreamSynchronize(s));
  return RFX_OK;
}

// redfox::count_string / total_string_32 (Reduce.cu:424-480, :665-740): runs of
// consecutive equal strings; per run the first key pointer and the u32 sum of its values.
// *key_size / *value_size are device-resident byte counts, read on entry and replaced by
// the output byte counts.  Synchronous on the default stream.
extern "C" rfx_status rfx_count_string_compat(const void* key_begin, const void* value_begin, void* result_key_begin,
                                              void* result_value_begin, uint64_t* key_size, uint64_t* value_size) {
  if (!key_size || !value_size) return RFX_ERR_INVALID;
  cudaStream_t s = 0;
  uint64_t kbytes = 0;
  RFX_CUDA_TRY(cudaMemcpy(&kbytes, key_size, sizeof(kbytes), cudaMemcpyDeviceToHost));
  const uint64_t n = kbytes / 8;
  uint64_t sizes[2] = {0, 0};
  if (n) {
    if (!key_begin || !value_begin || !result_key_begin || !result_value_begin) return RFX_ERR_INVALID;
    uint32_t* err = device_error_word();
    if (!err) return RFX_ERR_CUDA;
    DevBuf codes, heads, ws, okeys, small;
    ScanState ss;
    rfx_status st;
    if ((st = codes.alloc(n * 4, s)) != RFX_OK) return st;
    if ((st = string_codes(static_cast<const unsigned long long*>(key_begin), n, codes.as<uint32_t>(), nullptr,
                           nullptr, s)) != RFX_OK)
      return st;
    const size_t need = rfx_reduce_by_key_workspace(n);
    if ((st = ws.alloc(need, s)) != RFX_OK || (st = okeys.alloc(n * 4, s)) != RFX_OK ||
        (st = heads.alloc(n, s)) != RFX_OK || (st = small.alloc(64, s)) != RFX_OK || (st = ss.init(n, s)) != RFX_OK)
      return st;
    uint64_t* d_groups = small.as<uint64_t>();
    if ((st = rfx_reduce_by_key(codes.p, n, nullptr, 4, value_begin, RFX_VAL_U32, okeys.p, result_value_begin,
                                nullptr, d_groups, ws.p, need, s)) != RFX_OK)
      return st;
    code_heads<<<grid_for(n), 256, 0, s>>>(codes.as<uint32_t>(), n, heads.as<uint8_t>());
    RFX_CUDA_TRY(cudaGetLastError());
    FirstKey fk{static_cast<const unsigned long long*>(key_begin), static_cast<unsigned long long*>(result_key_begin)};
    if ((st = launch_head_scan(n, heads.as<uint8_t>(), ss, d_groups + 1, err, fk, s)) != RFX_OK) return st;
    uint64_t g[2] = {0, 0};
    RFX_CUDA_TRY(cudaMemcpyAsync(g, d_groups, sizeof(g), cudaMemcpyDeviceToHost, s));
    RFX_CUDA_TRY(cudaStreamSynchronize(s));
    uint32_t e = 0;
    RFX_CUDA_TRY(cudaMemcpy(&e, err, sizeof(e), cudaMemcpyDeviceToHost));
    if (e) return RFX_ERR_TIMEOUT;
    if (g[0] != g[1]) return RFX_ERR_INVALID;  // both count runs of equal codes
    sizes[0] = g[0] * 8;
    sizes[1] = g[0] * 4;
  }
  RFX_CUDA_TRY(cudaMemcpy(key_size, &sizes[0], sizeof(uint64_t), cudaMemcpyHostToDevice));
  RFX_CUDA_TRY(cudaMemcpy(value_size, &sizes[1], sizeof(uint64_t), cudaMemcpyHostToDevice));
  return RFX_OK;
}
