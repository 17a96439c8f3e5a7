// join_abi.cu -- C ABI of the sort-merge join: find_bounds, index expansion, gather, the
// fused tuple join, and the reference-compatible find_bounds_* / join entries.
#include <cstring>

#include "host_common.h"
#include "join_kernels.cuh"
#include "tune.h"

namespace rfx {
namespace {

bool key_width(uint32_t e) { return e == 1 || e == 2 || e == 4 || e == 8 || e == 16; }

struct FbLayout {
  uint64_t* status;
  uint32_t* counter;
  size_t clear;
  uint64_t* lb64;
  uint64_t* off64;
  uint64_t* tile_owner;   // fused join: first owner of each output tile (nl + 2 tiles)
  uint64_t n_owner;
  size_t total;
};

FbLayout fb_layout(void* ws, uint64_t nl, bool with_offsets) {
  FbLayout L;
  Carver c(ws);
  L.status = c.take<uint64_t>((nl + kFbTile - 1) / kFbTile + 1);
  L.counter = c.take<uint32_t>(1);
  L.clear = align_up(c.used, 256);
  c.used = L.clear;
  L.lb64 = with_offsets ? c.take<uint64_t>(nl + 1) : nullptr;
  L.off64 = with_offsets ? c.take<uint64_t>(nl + 1) : nullptr;
  L.n_owner = with_offsets ? nl + 2 : 0;
  L.tile_owner = with_offsets ? c.take<uint64_t>(nl + 2) : nullptr;
  L.total = align_up(c.used, 256);
  return L;
}

// The window of find_bounds: what a tile of kFbTile left rows is expected to need (nr / nl
// right keys per left row, 1.25x for variation, 512 more) at the width the kernel stores
// the keys in, between 8 and 64 KB.  Smaller windows leave room for more blocks per SM; a tile
// whose window does not fit searches in global memory instead.
uint32_t fb_window_bytes(uint64_t nl, uint64_t nr, uint32_t re, uint32_t rshift) {
  const uint32_t kbits = re * 8u > rshift ? re * 8u - rshift : 0u;
  const double kw = re <= 4 ? 4.0 : kbits <= 64 ? 8.0 : 16.0;
  double want = nl ? (1.25 * kFbTile * ((double)nr / (double)nl) + 512.0) * kw : 0.0;
  if (want < 8192.0) want = 8192.0;
  if (want > (double)kFbWindowBytes) want = kFbWindowBytes;
  return (uint32_t)align_up((uint64_t)want, 4096);
}

template <int LE, int RE>
rfx_status launch_fb(FindBoundsArgs& a, cudaStream_t s) {
  auto k = find_bounds_kernel<LE, RE>;
  RFX_CUDA_TRY(allow_smem((const void*)k, kFbWindowBytes));
  const uint64_t tiles = (a.nl + kFbTile - 1) / kFbTile;
  a.window_bytes = fb_window_bytes(a.nl, a.nr, RE, a.rshift);
  const int grid = persistent_grid((const void*)k, kJoinThreads, a.window_bytes, tiles ? tiles : 1);
  k<<<grid, kJoinThreads, a.window_bytes, s>>>(a);
  RFX_CUDA_TRY(cudaGetLastError());
  return RFX_OK;
}

rfx_status dispatch_fb(uint32_t le, uint32_t re, FindBoundsArgs& a, cudaStream_t s) {
#define RFX_FB(L, R) \
  if (le == L && re == R) return launch_fb<L, R>(a, s);
  RFX_FB(1, 1) RFX_FB(2, 2) RFX_FB(4, 4) RFX_FB(8, 8) RFX_FB(16, 16)
  RFX_FB(4, 8) RFX_FB(4, 16) RFX_FB(8, 4) RFX_FB(8, 16) RFX_FB(16, 4) RFX_FB(16, 8)
#undef RFX_FB
  return RFX_ERR_UNSUPPORTED;
}

template <int LE, int RE>
rfx_status launch_group(FindBoundsArgs& a, cudaStream_t s) {
  auto k = find_bounds_kernel<LE, RE, true>;
  RFX_CUDA_TRY(allow_smem((const void*)k, kFbWindowBytes));
  const uint64_t tiles = (a.nl + kFbTile - 1) / kFbTile;
  a.window_bytes = kFbWindowBytes;   // the group count is on the device: the largest window
  const int grid = persistent_grid((const void*)k, kJoinThreads, kFbWindowBytes, tiles ? tiles : 1);
  k<<<grid, kJoinThreads, kFbWindowBytes, s>>>(a);
  RFX_CUDA_TRY(cudaGetLastError());
  return RFX_OK;
}

rfx_status dispatch_group(uint32_t ke, uint32_t re, FindBoundsArgs& a, cudaStream_t s) {
#define RFX_GJ(L, R) \
  if (ke == L && re == R) return launch_group<L, R>(a, s);
  RFX_GJ(4, 4) RFX_GJ(4, 8) RFX_GJ(4, 16) RFX_GJ(8, 4) RFX_GJ(8, 8) RFX_GJ(8, 16)
#undef RFX_GJ
  return RFX_ERR_UNSUPPORTED;
}

// Workspace of rfx_join_aggregate: the right side's groups (keys, sums, counts, their
// number), the group join's tile status, then the reduce's own workspace.
struct JaLayout {
  uint8_t* gkeys;
  int64_t* gsum;
  uint32_t* gcnt;
  uint64_t* ngroups;
  uint64_t* status;
  uint32_t* counter;
  size_t clear_off, clear;   // status + counter
  void* rws;
  size_t rws_bytes;
  size_t total;
};

JaLayout ja_layout(void* ws, uint64_t nr, uint32_t kb) {
  JaLayout L;
  Carver c(ws);
  L.gkeys = c.take<uint8_t>(nr * kb);
  L.gsum = c.take<int64_t>(nr);
  L.gcnt = c.take<uint32_t>(nr);
  L.ngroups = c.take<uint64_t>(1);
  c.used = align_up(c.used, 256);
  L.clear_off = c.used;
  L.status = c.take<uint64_t>((nr + kFbTile - 1) / kFbTile + 1);
  L.counter = c.take<uint32_t>(1);
  L.clear = c.used - L.clear_off;
  L.rws_bytes = rfx_reduce_by_key_workspace(nr);
  L.rws = c.take<uint8_t>(L.rws_bytes);
  L.total = align_up(c.used, 256);
  return L;
}

// Emit variants: 0 = operands of each tile staged in shared memory by bulk copies,
// 1 = rows gathered from global memory per output.
template <int LE, int RE, int OE>
rfx_status launch_tj(TupleJoinArgs& a, cudaStream_t s) {
  const uint64_t tiles = (a.cap + kExpTile - 1) / kExpTile;
  auto run = [&](int v) -> rfx_status {
    if (v == 0) {
      auto k = tuple_join_staged_kernel<LE, RE, OE>;
      RFX_CUDA_TRY(allow_smem((const void*)k, JsLayout::BYTES));
      const int grid = persistent_grid((const void*)k, kJoinThreads, JsLayout::BYTES, tiles ? tiles : 1);
      k<<<grid, kJoinThreads, JsLayout::BYTES, s>>>(a);
    } else {
      auto k = tuple_join_kernel<LE, RE, OE>;
      const int grid = persistent_grid((const void*)k, kJoinThreads, 0, tiles ? tiles : 1);
      k<<<grid, kJoinThreads, 0, s>>>(a);
    }
    RFX_CUDA_TRY(cudaGetLastError());
    return RFX_OK;
  };
  // the emit writes only `out`, so candidates can be timed on the caller's call
  return run(tune_pick(TUNE_JOIN_EMIT, ((uint64_t)LE << 16) | ((uint64_t)RE << 8) | OE, a.cap, 2, run, s));
}

template <int LE, int RE>
rfx_status dispatch_tj_o(uint32_t oe, TupleJoinArgs& a, cudaStream_t s) {
  switch (oe) {
    case 4: return launch_tj<LE, RE, 4>(a, s);
    case 8: return launch_tj<LE, RE, 8>(a, s);
    case 16: return launch_tj<LE, RE, 16>(a, s);
    default: return RFX_ERR_UNSUPPORTED;
  }
}

rfx_status dispatch_tj(uint32_t le, uint32_t re, uint32_t oe, TupleJoinArgs& a, cudaStream_t s) {
#define RFX_TJ(L, R) \
  if (le == L && re == R) return dispatch_tj_o<L, R>(oe, a, s);
  RFX_TJ(4, 4) RFX_TJ(4, 8) RFX_TJ(4, 16) RFX_TJ(8, 4) RFX_TJ(8, 8) RFX_TJ(8, 16) RFX_TJ(16, 4) RFX_TJ(16, 8)
  RFX_TJ(16, 16)
#undef RFX_TJ
  return RFX_ERR_UNSUPPORTED;
}

bool aligned_to(const void* p, uint32_t b) { return (reinterpret_cast<uintptr_t>(p) % (b < 16 ? b : 16)) == 0; }

}  // namespace

size_t find_bounds_workspace_impl(uint64_t nl) { return fb_layout(nullptr, nl, false).total; }

rfx_status find_bounds_impl(int32_t* lb, int32_t* scan, uint64_t* d_total, const void* left, uint64_t nl,
                            const void* right, uint64_t nr, uint32_t kb, void* ws, size_t wsb, cudaStream_t s) {
  if (!key_width(kb)) return RFX_ERR_UNSUPPORTED;
  if (!d_total || (nl && (!left || !lb || !scan)) || (nr && !right)) return RFX_ERR_INVALID;
  if (nl >= (1ull << 31) || nr >= (1ull << 31)) return RFX_ERR_UNSUPPORTED;  // int32 outputs
  if ((nl && !aligned_to(left, kb)) || (nr && !aligned_to(right, kb))) return RFX_ERR_INVALID;
  FbLayout L = fb_layout(ws, nl, false);
  if (!ws || wsb < L.total) return RFX_ERR_WORKSPACE;
  uint32_t* err = device_error_word();
  if (!err) return RFX_ERR_CUDA;
  RFX_CUDA_TRY(cudaMemsetAsync(ws, 0, L.clear, s));
  FindBoundsArgs a;
  std::memset(&a, 0, sizeof(a));
  a.left = static_cast<const uint8_t*>(left);
  a.nl = nl;
  a.right = static_cast<const uint8_t*>(right);
  a.nr = nr;
  a.lb32 = lb;
  a.scan32 = scan;
  a.d_total = d_total;
  a.status = L.status;
  a.tile_counter = L.counter;
  a.err = err;
  return dispatch_fb(kb, kb, a, s);
}

rfx_status join_expand_impl(int32_t* li, int32_t* ri, uint64_t nout, const uint64_t* d_nout, const int32_t* lb,
                            const int32_t* scan, uint64_t nl, cudaStream_t s) {
  if (nout == 0) return RFX_OK;
  if (!li || !ri || !lb || !scan || nl == 0) return RFX_ERR_INVALID;
  const uint64_t tiles = (nout + kExpTile - 1) / kExpTile;
  const int grid = persistent_grid((const void*)join_expand_kernel, kJoinThreads, 0, tiles);
  join_expand_kernel<<<grid, kJoinThreads, 0, s>>>(li, ri, nout, d_nout, lb, scan, nl);
  RFX_CUDA_TRY(cudaGetLastError());
  return RFX_OK;
}

}  // namespace rfx

using namespace rfx;

extern "C" size_t rfx_join_find_bounds_workspace(uint64_t nl) { return find_bounds_workspace_impl(nl); }

extern "C" rfx_status rfx_join_find_bounds(int32_t* lower_bound, int32_t* left_count, uint64_t* d_total,
                                           const void* left_keys, uint64_t nl, const void* right_keys, uint64_t nr,
                                           uint32_t key_bytes, void* workspace, size_t workspace_bytes, void* stream) {
  return find_bounds_impl(lower_bound, left_count, d_total, left_keys, nl, right_keys, nr, key_bytes, workspace,
                          workspace_bytes, as_stream(stream));
}

extern "C" rfx_status rfx_join_expand(int32_t* left_idx, int32_t* right_idx, uint64_t nout, const uint64_t* d_nout,
                                      const int32_t* lower_bound, const int32_t* left_count_scan, uint64_t nl,
                                      void* stream) {
  return join_expand_impl(left_idx, right_idx, nout, d_nout, lower_bound, left_count_scan, nl, as_stream(stream));
}

extern "C" rfx_status rfx_join_gather(void* out, uint32_t out_bytes, uint64_t nout, const uint64_t* d_nout,
                                      const int32_t* left_idx, const int32_t* right_idx, const void* lkey,
                                      uint32_t lkey_bytes, const void* lval, uint32_t lval_bytes, uint32_t lval_bits,
                                      const void* rval, uint32_t rval_bytes, uint32_t rval_bits, void* stream) {
  auto ok_w = [](uint32_t b) { return b == 1 || b == 2 || b == 4 || b == 8 || b == 16 || b == 32 || b == 64; };
  if (!ok_w(out_bytes) || !ok_w(lkey_bytes) || (lval && !ok_w(lval_bytes)) || (rval && !ok_w(rval_bytes)))
    return RFX_ERR_UNSUPPORTED;
  if (nout == 0) return RFX_OK;
  if (!out || !left_idx || !lkey || (rval && !right_idx)) return RFX_ERR_INVALID;
  GatherArgs a;
  a.out = static_cast<uint8_t*>(out);
  a.ob = out_bytes;
  a.nout_max = nout;
  a.d_nout = d_nout;
  a.li = left_idx;
  a.ri = right_idx;
  a.lkey = static_cast<const uint8_t*>(lkey);
  a.lkb = lkey_bytes;
  a.lval = static_cast<const uint8_t*>(lval);
  a.lvb = lval_bytes;
  a.lv_bits = lval ? lval_bits : 0;
  a.rval = static_cast<const uint8_t*>(rval);
  a.rvb = rval_bytes;
  a.rv_bits = rval ? rval_bits : 0;
  const uint64_t blocks = (nout + kJoinThreads - 1) / kJoinThreads;
  const int grid = persistent_grid((const void*)join_gather_kernel, kJoinThreads, 0, blocks);
  join_gather_kernel<<<grid, kJoinThreads, 0, as_stream(stream)>>>(a);
  RFX_CUDA_TRY(cudaGetLastError());
  return RFX_OK;
}

extern "C" size_t rfx_join_tuples_workspace(uint64_t nl) { return fb_layout(nullptr, nl, true).total; }

extern "C" rfx_status rfx_join_tuples(void* out, uint32_t out_bytes, uint64_t capacity, uint64_t* d_count,
                                      const void* left, uint64_t nl, uint32_t left_bytes, uint32_t left_value_bits,
                                      const void* right, uint64_t nr, uint32_t right_bytes, uint32_t right_value_bits,
                                      void* workspace, size_t workspace_bytes, void* stream) {
  const bool w_ok = (left_bytes == 4 || left_bytes == 8 || left_bytes == 16) &&
                    (right_bytes == 4 || right_bytes == 8 || right_bytes == 16) &&
                    (out_bytes == 4 || out_bytes == 8 || out_bytes == 16);
  if (!w_ok || left_value_bits >= left_bytes * 8u || right_value_bits >= right_bytes * 8u) return RFX_ERR_UNSUPPORTED;
  if (!d_count || (nl && !left) || (nr && !right) || (capacity && !out)) return RFX_ERR_INVALID;
  if ((nl && !aligned_to(left, left_bytes)) || (nr && !aligned_to(right, right_bytes)) ||
      (capacity && !aligned_to(out, out_bytes)))
    return RFX_ERR_INVALID;
  cudaStream_t s = as_stream(stream);
  FbLayout L = fb_layout(workspace, nl, true);
  if (!workspace || workspace_bytes < L.total) return RFX_ERR_WORKSPACE;
  uint32_t* err = device_error_word();
  if (!err) return RFX_ERR_CUDA;
  RFX_CUDA_TRY(cudaMemsetAsync(workspace, 0, L.clear, s));
  FindBoundsArgs a;
  std::memset(&a, 0, sizeof(a));
  a.left = static_cast<const uint8_t*>(left);
  a.nl = nl;
  a.right = static_cast<const uint8_t*>(right);
  a.nr = nr;
  a.lshift = left_value_bits;
  a.rshift = right_value_bits;
  a.lb64 = L.lb64;
  a.off64 = L.off64;
  a.tile_owner = L.tile_owner;
  a.n_owner = L.n_owner;
  a.d_total = d_count;
  a.status = L.status;
  a.tile_counter = L.counter;
  a.err = err;
  rfx_status st = dispatch_fb(left_bytes, right_bytes, a, s);
  if (st != RFX_OK || capacity == 0 || nl == 0) return st;
  TupleJoinArgs j;
  j.left = static_cast<const uint8_t*>(left);
  j.nl = nl;
  j.right = static_cast<const uint8_t*>(right);
  j.nr = nr;
  j.rv_bits = right_value_bits;
  j.lb64 = L.lb64;
  j.off64 = L.off64;
  j.out = static_cast<uint8_t*>(out);
  j.cap = capacity;
  j.tile_owner = L.tile_owner;
  j.n_owner = L.n_owner;
  j.err = err;
  return dispatch_tj(left_bytes, right_bytes, out_bytes, j, s);
}

extern "C" size_t rfx_join_aggregate_workspace(uint64_t nr, uint32_t out_key_bytes) {
  return ja_layout(nullptr, nr, out_key_bytes).total;
}

// The join of left and right on their keys followed by SUM(right value) and COUNT per key,
// without the join rows: the right side is reduced to its groups, then each group whose
// key occurs on the left is kept with its sum and count multiplied by the number of left
// rows that carry the key -- per key the join has n_left(k) x n_right(k) rows whose values
// sum to n_left(k) x (sum of the right values), and the products wrap modulo 2^64 / 2^32
// exactly as the sums over the join rows do.
extern "C" rfx_status rfx_join_aggregate(const void* left, uint64_t nl, uint32_t left_bytes, uint32_t left_value_bits,
                                         const void* right, uint64_t nr, uint32_t right_bytes,
                                         uint32_t right_value_bits, uint32_t value_shift, uint32_t value_bits,
                                         void* out_keys, uint32_t out_key_bytes, int64_t* out_sums,
                                         uint32_t* out_counts, uint64_t* d_groups, void* workspace,
                                         size_t workspace_bytes, void* stream) {
  const bool w_ok = (left_bytes == 4 || left_bytes == 8 || left_bytes == 16) &&
                    (right_bytes == 4 || right_bytes == 8 || right_bytes == 16) &&
                    (out_key_bytes == 4 || out_key_bytes == 8);
  if (!w_ok || left_value_bits >= left_bytes * 8u || right_value_bits >= right_bytes * 8u || value_bits > 64 ||
      value_shift + value_bits > right_bytes * 8u)
    return RFX_ERR_UNSUPPORTED;
  // the right key is stored in out_key_bytes (bits above are dropped, as
  // rfx_reduce_tuples drops them): the caller's key fields must fit that width
  if (!d_groups || (nl && !left) || (nr && !right) || (nr && (!out_keys || !out_sums || !out_counts)))
    return RFX_ERR_INVALID;
  if ((nl && !aligned_to(left, left_bytes)) || (nr && !aligned_to(right, right_bytes)) ||
      (nr && !aligned_to(out_keys, out_key_bytes)))
    return RFX_ERR_INVALID;
  cudaStream_t s = as_stream(stream);
  JaLayout L = ja_layout(workspace, nr, out_key_bytes);
  if (!workspace || workspace_bytes < L.total) return RFX_ERR_WORKSPACE;
  if (nr == 0) return cuda_fail(cudaMemsetAsync(d_groups, 0, sizeof(uint64_t), s));
  uint32_t* err = device_error_word();
  if (!err) return RFX_ERR_CUDA;
  rfx_status st = rfx_reduce_tuples(right, nr, nullptr, right_bytes, right_value_bits, value_shift, value_bits,
                                    L.gkeys, out_key_bytes, L.gsum, L.gcnt, L.ngroups, L.rws, L.rws_bytes, stream);
  if (st != RFX_OK) return st;
  RFX_CUDA_TRY(cudaMemsetAsync(static_cast<uint8_t*>(workspace) + L.clear_off, 0, L.clear, s));
  FindBoundsArgs a;
  std::memset(&a, 0, sizeof(a));
  a.left = L.gkeys;
  a.nl = nr;
  a.d_nl = L.ngroups;
  a.right = static_cast<const uint8_t*>(left);
  a.nr = nl;
  a.lshift = 0;
  a.rshift = left_value_bits;
  a.d_total = d_groups;
  a.status = L.status;
  a.tile_counter = L.counter;
  a.err = err;
  a.gsum = L.gsum;
  a.gcnt = L.gcnt;
  a.okey = static_cast<uint8_t*>(out_keys);
  a.osum = out_sums;
  a.ocnt = out_counts;
  return dispatch_group(out_key_bytes, left_bytes, a, s);
}

// ---- reference-compatible entries (synchronous, own their scratch) ----

// redfox::find_bounds_{8,16,32,64,128} (ModernGPUJoin.cu:109-663): sizes in elements,
// *result_size (device) = number of matches.
extern "C" rfx_status rfx_find_bounds_compat(int32_t* lower_bound, int32_t* left_count, uint64_t* result_size,
                                             const void* left_key, uint64_t left_size, const void* right_key,
                                             uint64_t right_size, uint32_t key_bytes) {
  cudaStream_t s = 0;
  const size_t need = find_bounds_workspace_impl(left_size);
  void* ws = nullptr;
  RFX_CUDA_TRY(cudaMallocAsync(&ws, need, s));
  rfx_status st = find_bounds_impl(lower_bound, left_count, result_size, left_key, left_size, right_key, right_size,
                                   key_bytes, ws, need, s);
  cudaFreeAsync(ws, s);
  if (st != RFX_OK) return st;
  RFX_CUDA_TRY(cudaStreamSynchronize(s));
  return RFX_OK;
}

// redfox::join (ModernGPUJoin.cu:665-733): result_size and input_size in elements.
extern "C" rfx_status rfx_join_compat(int32_t* left_indices, int32_t* right_indices, uint64_t result_size,
                                      const int32_t* lower_bound, const int32_t* left_count, uint64_t input_size) {
  rfx_status st = join_expand_impl(left_indices, right_indices, result_size, nullptr, lower_bound, left_count,
                                   input_size, 0);
  if (st != RFX_OK) return st;
  RFX_CUDA_TRY(cudaStreamSynchronize(0));
  return RFX_OK;
}

// Second half of rfx_join_tuples: expands and assembles from the bounds and offsets that a
// preceding rfx_join_tuples call (any capacity, 0 to count only) left in the same
// workspace, so the caller can size the output from *d_count in between -- the shape of
// the reference's find_bounds -> join_get_result_size -> Resize -> join_main + gather.
extern "C" rfx_status rfx_join_tuples_emit(void* out, uint32_t out_bytes, uint64_t capacity, const void* left,
                                           uint64_t nl, uint32_t left_bytes, const void* right, uint64_t nr,
                                           uint32_t right_bytes, uint32_t right_value_bits, void* workspace,
                                           size_t workspace_bytes, void* stream) {
  const bool w_ok = (left_bytes == 4 || left_bytes == 8 || left_bytes == 16) &&
                    (right_bytes == 4 || right_bytes == 8 || right_bytes == 16) &&
                    (out_bytes == 4 || out_bytes == 8 || out_bytes == 16);
  if (!w_ok || right_value_bits >= right_bytes * 8u) return RFX_ERR_UNSUPPORTED;
  if (capacity == 0 || nl == 0) return RFX_OK;
  if (!out || !left || (nr && !right) || !aligned_to(out, out_bytes)) return RFX_ERR_INVALID;
  FbLayout L = fb_layout(workspace, nl, true);
  if (!workspace || workspace_bytes < L.total) return RFX_ERR_WORKSPACE;
  TupleJoinArgs j;
  j.left = static_cast<const uint8_t*>(left);
  j.nl = nl;
  j.right = static_cast<const uint8_t*>(right);
  j.nr = nr;
  j.rv_bits = right_value_bits;
  j.lb64 = L.lb64;
  j.off64 = L.off64;
  j.out = static_cast<uint8_t*>(out);
  j.cap = capacity;
  j.tile_owner = L.tile_owner;
  j.n_owner = L.n_owner;
  j.err = device_error_word();
  return dispatch_tj(left_bytes, right_bytes, out_bytes, j, as_stream(stream));
}
