// setops_abi.cu -- C ABI of union / difference / intersection / unique, and the
// reference-compatible set_union / difference / unique entries.
#include <cstring>

#include "host_common.h"
#include "setops_kernels.cuh"
#include "tune.h"

namespace rfx {
namespace {

bool elem_width(uint32_t e) { return e == 1 || e == 2 || e == 4 || e == 8 || e == 16; }

struct FilterLayout {
  uint64_t* status;
  uint32_t* counter;
  uint64_t* split;   // 3 words per tile, and per tile boundary plus one (set_split_kernel, set_bounds_kernel)
  uint8_t* mask;     // two-pass and warp-segment forms: one bit per element
  uint32_t* counts;  // two-pass and warp-segment forms: kept elements per tile
  uint32_t* wcounts; // warp-segment form: kept elements per warp segment
  uint64_t* offsets; // two-pass and warp-segment forms: each tile's output offset
  size_t clear;
  size_t total;
};

FilterLayout filter_layout(void* ws, uint64_t n) {
  FilterLayout L;
  Carver c(ws);
  const uint64_t tiles = (n + kSetTileMin - 1) / kSetTileMin + 1;
  const uint64_t mark_tiles = (n + kSetTileMin - 1) / kSetTileMin + 1;   // tiles of 4 items per thread at the most
  L.status = c.take<uint64_t>(tiles);
  L.counter = c.take<uint32_t>(1);
  L.clear = align_up(c.used, 256);
  c.used = L.clear;
  L.split = c.take<uint64_t>(3 * (tiles + 1));
  L.mask = c.take<uint8_t>(mark_tiles * kSetThreads);
  L.counts = c.take<uint32_t>(mark_tiles);
  L.wcounts = c.take<uint32_t>(mark_tiles * kSegWarps);
  L.offsets = c.take<uint64_t>(mark_tiles);
  L.total = align_up(c.used, 256);
  return L;
}

template <int E, int IPT>
rfx_status launch_filter_ipt(int mode, SetFilterArgs& a, cudaStream_t s) {
  constexpr int TILE = kSetThreads * IPT;
  const uint64_t tiles = (a.na + TILE - 1) / TILE;
  if (mode != KEEP_HEADS && tiles) {
    const uint64_t work = 3 * tiles * 32;   // one warp per search
    const int g = (int)((work + 255) / 256);
    set_split_kernel<E, TILE><<<g, 256, 0, s>>>(a.a, a.na, a.b, a.nb, const_cast<uint64_t*>(a.split));
    RFX_CUDA_TRY(cudaGetLastError());
  }
  const void* k = mode == KEEP_MATCHED ? (const void*)set_filter_kernel<E, KEEP_MATCHED, IPT>
                : mode == KEEP_UNMATCHED ? (const void*)set_filter_kernel<E, KEEP_UNMATCHED, IPT>
                                         : (const void*)set_filter_kernel<E, KEEP_HEADS, IPT>;
  const int grid = persistent_grid(k, kSetThreads, 0, tiles ? tiles : 1);
  if (mode == KEEP_MATCHED) set_filter_kernel<E, KEEP_MATCHED, IPT><<<grid, kSetThreads, 0, s>>>(a);
  else if (mode == KEEP_UNMATCHED) set_filter_kernel<E, KEEP_UNMATCHED, IPT><<<grid, kSetThreads, 0, s>>>(a);
  else set_filter_kernel<E, KEEP_HEADS, IPT><<<grid, kSetThreads, 0, s>>>(a);
  RFX_CUDA_TRY(cudaGetLastError());
  return RFX_OK;
}

// The two-pass form: split entries, mark (keep bits and per-tile counts), offsets and the
// total, compaction.  Needs no cleared workspace.
template <int E, int IPT>
rfx_status launch_two_pass(int mode, SetFilterArgs& a, const FilterLayout& L, cudaStream_t s) {
  constexpr int TILE = kSetThreads * IPT;
  const uint64_t tiles = (a.na + TILE - 1) / TILE;
  if (tiles) {
    const uint64_t work = 3 * tiles * 32;   // one warp per search
    set_split_kernel<E, TILE><<<(int)((work + 255) / 256), 256, 0, s>>>(a.a, a.na, a.b, a.nb, L.split);
    RFX_CUDA_TRY(cudaGetLastError());
    a.split = L.split;
    auto k = mode == KEEP_MATCHED ? set_mark_kernel<E, KEEP_MATCHED, IPT> : set_mark_kernel<E, KEEP_UNMATCHED, IPT>;
    // the B window a tile is expected to need (nb / na per item, 1.25x, 512 more), at least
    // 2048 elements and at most 48 KiB
    typedef SetWord<E> WT;
    double want = 1.25 * TILE * ((double)a.nb / (double)a.na) + 512.0;
    if (want < 2048.0) want = 2048.0;
    if (want * sizeof(WT) > 48.0 * 1024) want = 48.0 * 1024 / sizeof(WT);
    a.wcap = (uint32_t)want;
    const size_t smem = align_up((size_t)a.wcap * sizeof(WT), 16);
    RFX_CUDA_TRY(allow_smem((const void*)k, smem));
    const int grid = persistent_grid((const void*)k, kSetThreads, smem, tiles);
    k<<<grid, kSetThreads, smem, s>>>(a, L.mask, L.counts);
    RFX_CUDA_TRY(cudaGetLastError());
  }
  set_offsets_kernel<<<1, kOffsetThreads, 0, s>>>(L.counts, tiles, L.offsets, a.d_count);
  RFX_CUDA_TRY(cudaGetLastError());
  if (tiles) {
    const int grid = persistent_grid((const void*)set_compact_kernel<E, IPT>, kSetThreads, 0, tiles);
    set_compact_kernel<E, IPT><<<grid, kSetThreads, 0, s>>>(a.a, a.na, L.mask, L.offsets, a.out, a.na);
    RFX_CUDA_TRY(cudaGetLastError());
  }
  return RFX_OK;
}

// The warp-segment form's B window capacity (elements per buffer) for n_a elements filtered
// against n_b: 1.25x the expected window of a tile plus 512, at least 2048, a multiple of 4;
// 0 when a buffer would exceed 32 KiB (the two-pass form's single window serves those).
template <int E, int IPT>
uint32_t seg_wcap(uint64_t na, uint64_t nb) {
  double want = 1.25 * (double)(kSetThreads * IPT) * ((double)nb / (double)(na ? na : 1)) + 512.0;
  if (want < 2048.0) want = 2048.0;
  const uint32_t w = ((uint32_t)(want < 1e9 ? want : 1e9) + 3u) & ~3u;
  return (uint64_t)seg_buffer_elems<E>(w) * E > 32u * 1024u ? 0u : w;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// The warp-segment form (4- and 8-byte elements, 16-byte aligned A and B): bounds per tile
// boundary, mark (keep bits, counts per tile and per warp segment), offsets and the total,
// compaction.  Needs no cleared workspace.  Returns RFX_ERR_UNSUPPORTED for inputs it does
// not take.
template <int E, int IPT>
rfx_status launch_seg(int mode, SetFilterArgs& a, const FilterLayout& L, cudaStream_t s) {
  if constexpr (E != 4 && E != 8) {
    return RFX_ERR_UNSUPPORTED;
  } else {
    constexpr int TILE = kSetThreads * IPT;
    const uint64_t tiles = (a.na + TILE - 1) / TILE;
    const uint32_t wcap = seg_wcap<E, IPT>(a.na, a.nb);
    if (!wcap || (a.na && !aligned16(a.a)) || (a.nb && !aligned16(a.b))) return RFX_ERR_UNSUPPORTED;
    if (tiles) {
      const uint64_t work = (tiles + 1) * 32;   // one warp per tile boundary
      set_bounds_kernel<E, TILE><<<(int)((work + 255) / 256), 256, 0, s>>>(a.a, a.na, a.b, a.nb, L.split);
      RFX_CUDA_TRY(cudaGetLastError());
      a.split = L.split;
      a.wcap = wcap;
      auto k = mode == KEEP_MATCHED ? set_mark_seg_kernel<E, KEEP_MATCHED, IPT> : set_mark_seg_kernel<E, KEEP_UNMATCHED, IPT>;
      const size_t smem = 2 * (size_t)seg_buffer_elems<E>(wcap) * E;
      RFX_CUDA_TRY(allow_smem((const void*)k, smem));
      const int grid = persistent_grid((const void*)k, kSetThreads, smem, tiles);
      k<<<grid, kSetThreads, smem, s>>>(a, L.mask, L.counts, L.wcounts);
      RFX_CUDA_TRY(cudaGetLastError());
    }
    set_offsets_kernel<<<1, kOffsetThreads, 0, s>>>(L.counts, tiles, L.offsets, a.d_count);
    RFX_CUDA_TRY(cudaGetLastError());
    if (tiles) {
      const int grid = persistent_grid((const void*)set_compact_seg_kernel<E, IPT>, kSetThreads, 0, tiles);
      set_compact_seg_kernel<E, IPT><<<grid, kSetThreads, 0, s>>>(a.a, a.na, L.mask, L.offsets, L.wcounts, a.out, a.na);
      RFX_CUDA_TRY(cudaGetLastError());
    }
    return RFX_OK;
  }
}

// Variants of intersection / difference / union's B - A: 0 (the default) the warp-segment
// form with 16 items per thread; 1, 2, 3 the one-pass form (decoupled look-back) with 8, 4
// and 16 items per thread; 4 the two-pass form with 16 items per thread; 5 the warp-segment
// form with 8; 6 the two-pass form with 8.  The warp-segment form takes fewer items per
// thread where a tile's B window would not fit (16 -> 8 -> 4), and the two-pass form with 8
// items where it does not apply at all.  Unique and filters whose output overlaps A (in
// place) always take the one-pass form with 8 items per thread.  The one-pass form's
// look-back status and tile counter are zeroed before each launch.
template <int E>
rfx_status launch_filter(int mode, SetFilterArgs& a, cudaStream_t s, const FilterLayout* L, bool in_place) {
  auto run = [&](int v) -> rfx_status {
    if ((v == 0 || v == 5) && L) {
      rfx_status st = v == 0 ? launch_seg<E, 16>(mode, a, *L, s) : RFX_ERR_UNSUPPORTED;
      if (st == RFX_ERR_UNSUPPORTED) st = launch_seg<E, 8>(mode, a, *L, s);
      if (st == RFX_ERR_UNSUPPORTED) st = launch_seg<E, 4>(mode, a, *L, s);
      if (st != RFX_ERR_UNSUPPORTED) return st;
      v = 6;
    }
    if (v == 6 && L) return launch_two_pass<E, 8>(mode, a, *L, s);
    if (v == 4 && L) return launch_two_pass<E, 16>(mode, a, *L, s);
    if (L) RFX_CUDA_TRY(cudaMemsetAsync(L->status, 0, L->clear, s));
    if (v <= 1 || v >= 5 || mode == KEEP_HEADS) return launch_filter_ipt<E, 8>(mode, a, s);
    return v == 2 ? launch_filter_ipt<E, 4>(mode, a, s) : launch_filter_ipt<E, 16>(mode, a, s);
  };
  if (mode == KEEP_HEADS || !L) return run(1);
  if (in_place) return run(1);
  return run(tune_pick(TUNE_SET_FILTER, ((uint64_t)E << 8) | (uint64_t)mode, a.na + a.nb, 7, run, s));
}

rfx_status dispatch_filter(uint32_t e, int mode, SetFilterArgs& a, cudaStream_t s, const FilterLayout* L = nullptr,
                           bool in_place = false) {
  switch (e) {
    case 1: return launch_filter<1>(mode, a, s, L, in_place);
    case 2: return launch_filter<2>(mode, a, s, L, in_place);
    case 4: return launch_filter<4>(mode, a, s, L, in_place);
    case 8: return launch_filter<8>(mode, a, s, L, in_place);
    case 16: return launch_filter<16>(mode, a, s, L, in_place);
    default: return RFX_ERR_UNSUPPORTED;
  }
}

template <int E>
rfx_status launch_merge(const void* a, uint64_t na, const void* d, uint64_t nd_max, const uint64_t* d_nd, void* out,
                        uint64_t* d_count, uint64_t* mp, cudaStream_t s) {
  const uint64_t tiles = (na + nd_max + kMergeTile - 1) / kMergeTile;
  if constexpr (E == 4 || E == 8) {
    // the staged merge: partitions of every tile first, then the tiles
    if (mp && aligned16(a) && aligned16(d) && aligned16(out)) {
      const uint64_t work = (tiles + 1) * 32;   // one warp per tile boundary
      merge_partition_kernel<E><<<(int)((work + 255) / 256), 256, 0, s>>>(
          static_cast<const uint8_t*>(a), na, static_cast<const uint8_t*>(d), nd_max, d_nd, mp);
      RFX_CUDA_TRY(cudaGetLastError());
      const size_t smem = merge_staged_smem<E>();
      RFX_CUDA_TRY(allow_smem((const void*)merge_staged_kernel<E>, smem));
      const int grid = persistent_grid((const void*)merge_staged_kernel<E>, kSetThreads, smem, tiles ? tiles : 1);
      merge_staged_kernel<E><<<grid, kSetThreads, smem, s>>>(static_cast<const uint8_t*>(a), na,
                                                              static_cast<const uint8_t*>(d), nd_max, d_nd, mp,
                                                              static_cast<uint8_t*>(out), d_count);
      RFX_CUDA_TRY(cudaGetLastError());
      return RFX_OK;
    }
  }
  const int grid = persistent_grid((const void*)merge_kernel<E>, kSetThreads, 0, tiles ? tiles : 1);
  merge_kernel<E><<<grid, kSetThreads, 0, s>>>(static_cast<const uint8_t*>(a), na, static_cast<const uint8_t*>(d),
                                               nd_max, d_nd, static_cast<uint8_t*>(out), d_count);
  RFX_CUDA_TRY(cudaGetLastError());
  return RFX_OK;
}

rfx_status dispatch_merge(uint32_t e, const void* a, uint64_t na, const void* d, uint64_t nd_max, const uint64_t* d_nd,
                          void* out, uint64_t* d_count, uint64_t* mp, cudaStream_t s) {
  switch (e) {
    case 1: return launch_merge<1>(a, na, d, nd_max, d_nd, out, d_count, mp, s);
    case 2: return launch_merge<2>(a, na, d, nd_max, d_nd, out, d_count, mp, s);
    case 4: return launch_merge<4>(a, na, d, nd_max, d_nd, out, d_count, mp, s);
    case 8: return launch_merge<8>(a, na, d, nd_max, d_nd, out, d_count, mp, s);
    case 16: return launch_merge<16>(a, na, d, nd_max, d_nd, out, d_count, mp, s);
    default: return RFX_ERR_UNSUPPORTED;
  }
}

template <int E>
rfx_status launch_prev(const void* a, uint64_t n, void* prev, cudaStream_t s) {
  const uint64_t tiles = (n + kSetTile - 1) / kSetTile;
  const int grid = (int)((tiles + 255) / 256);
  tile_prev_kernel<E><<<grid ? grid : 1, 256, 0, s>>>(static_cast<const uint8_t*>(a), n, static_cast<uint8_t*>(prev),
                                                      kSetTile);
  RFX_CUDA_TRY(cudaGetLastError());
  return RFX_OK;
}

bool aligned_to(const void* p, uint32_t b) { return (reinterpret_cast<uintptr_t>(p) % (b < 16 ? b : 16)) == 0; }

struct SetLayout {
  FilterLayout f;
  uint8_t* diff;
  uint64_t* d_nd;
  uint64_t* mp;   // union: where each merge tile's first diagonal crosses A
  size_t total;
};

SetLayout set_layout(void* ws, uint32_t op, uint64_t na, uint64_t nb, uint32_t e) {
  SetLayout L;
  // union filters B against A, the others filter A against B
  const uint64_t nf = op == RFX_SET_UNION ? nb : na;
  L.f = filter_layout(ws, nf);
  Carver c(ws);
  c.used = L.f.total;
  L.diff = op == RFX_SET_UNION ? c.take<uint8_t>(nb * e) : nullptr;
  L.d_nd = op == RFX_SET_UNION ? c.take<uint64_t>(1) : nullptr;
  L.mp = op == RFX_SET_UNION ? c.take<uint64_t>((na + nb + kMergeTile - 1) / kMergeTile + 2) : nullptr;
  L.total = align_up(c.used, 256);
  return L;
}

}  // namespace

size_t set_op_workspace_impl(uint32_t op, uint64_t na, uint64_t nb, uint32_t e) {
  return set_layout(nullptr, op, na, nb, e).total;
}

rfx_status set_op_impl(uint32_t op, void* out, uint64_t* d_count, const void* a, uint64_t na, const void* b, uint64_t nb,
                       uint32_t e, void* ws, size_t wsb, cudaStream_t s) {
  if (!elem_width(e) || op > RFX_SET_INTERSECTION) return RFX_ERR_UNSUPPORTED;
  if (!d_count || (na && !a) || (nb && !b) || ((na || nb) && !out)) return RFX_ERR_INVALID;
  if ((na && !aligned_to(a, e)) || (nb && !aligned_to(b, e)) || (out && !aligned_to(out, e))) return RFX_ERR_INVALID;
  SetLayout L = set_layout(ws, op, na, nb, e);
  if (!ws || wsb < L.total) return RFX_ERR_WORKSPACE;
  uint32_t* err = device_error_word();
  if (!err) return RFX_ERR_CUDA;
  SetFilterArgs f;
  std::memset(&f, 0, sizeof(f));
  f.status = L.f.status;
  f.tile_counter = L.f.counter;
  f.split = L.f.split;
  f.err = err;
  if (op == RFX_SET_UNION) {
    f.a = static_cast<const uint8_t*>(b);  // B - A: the copies of B beyond A's
    f.na = nb;
    f.b = static_cast<const uint8_t*>(a);
    f.nb = na;
    f.out = L.diff;
    f.d_count = L.d_nd;
    rfx_status st = dispatch_filter(e, KEEP_UNMATCHED, f, s, &L.f);
    if (st != RFX_OK) return st;
    return dispatch_merge(e, a, na, L.diff, nb, L.d_nd, out, d_count, L.mp, s);
  }
  f.a = static_cast<const uint8_t*>(a);
  f.na = na;
  f.b = static_cast<const uint8_t*>(b);
  f.nb = nb;
  f.out = static_cast<uint8_t*>(out);
  f.d_count = d_count;
  // an output overlapping A (in place) needs the one-pass form, whose writes never pass
  // the inputs not yet read
  const uintptr_t oa = reinterpret_cast<uintptr_t>(out), aa = reinterpret_cast<uintptr_t>(a);
  const bool overlap = na && oa < aa + na * e && aa < oa + na * e;
  return dispatch_filter(e, op == RFX_SET_INTERSECTION ? KEEP_MATCHED : KEEP_UNMATCHED, f, s, &L.f, overlap);
}

size_t unique_workspace_impl(uint64_t n, uint32_t e) {
  FilterLayout f = filter_layout(nullptr, n);
  Carver c(nullptr);
  c.used = f.total;
  c.take<uint8_t>(((n + kSetTileMin - 1) / kSetTileMin + 1) * (e < 16 ? 16 : e));
  return align_up(c.used, 256);
}

rfx_status unique_impl(void* data, uint64_t n, uint64_t* d_count, uint32_t e, void* ws, size_t wsb, cudaStream_t s) {
  if (!elem_width(e)) return RFX_ERR_UNSUPPORTED;
  if (!d_count || (n && !data)) return RFX_ERR_INVALID;
  if (n && !aligned_to(data, e)) return RFX_ERR_INVALID;
  FilterLayout f = filter_layout(ws, n);
  Carver c(ws);
  c.used = f.total;
  uint8_t* prev = c.take<uint8_t>(((n + kSetTileMin - 1) / kSetTileMin + 1) * (e < 16 ? 16 : e));
  if (!ws || wsb < align_up(c.used, 256)) return RFX_ERR_WORKSPACE;
  uint32_t* err = device_error_word();
  if (!err) return RFX_ERR_CUDA;
  RFX_CUDA_TRY(cudaMemsetAsync(ws, 0, f.clear, s));
  if (n) {
    rfx_status st;
    switch (e) {
      case 1: st = launch_prev<1>(data, n, prev, s); break;
      case 2: st = launch_prev<2>(data, n, prev, s); break;
      case 4: st = launch_prev<4>(data, n, prev, s); break;
      case 8: st = launch_prev<8>(data, n, prev, s); break;
      default: st = launch_prev<16>(data, n, prev, s); break;
    }
    if (st != RFX_OK) return st;
  }
  SetFilterArgs a;
  std::memset(&a, 0, sizeof(a));
  a.a = static_cast<const uint8_t*>(data);
  a.na = n;
  a.prev = prev;
  a.out = static_cast<uint8_t*>(data);
  a.d_count = d_count;
  a.status = f.status;
  a.tile_counter = f.counter;
  a.err = err;
  return dispatch_filter(e, KEEP_HEADS, a, s);
}

namespace {
uint32_t type_bytes(uint64_t type) {
  switch (type) {
    case RFX_I8: return 1;
    case RFX_I16: return 2;
    case RFX_I32: return 4;
    case RFX_I64: return 8;
    case RFX_I128: return 16;
    default: return 0;
  }
}

__global__ void scale_kernel(uint64_t* p, uint64_t factor) { *p *= factor; }

// Reference byte-size convention: *size (device) = output bytes.
rfx_status set_compat(uint32_t op, void* result, uint64_t* size, void* lb, void* le, void* rb, void* re, uint64_t type) {
  const uint32_t e = type_bytes(type);
  if (!e) return RFX_ERR_UNSUPPORTED;
  if (!size) return RFX_ERR_INVALID;
  const uint64_t na = (uint64_t)((uint8_t*)le - (uint8_t*)lb) / e, nb = (uint64_t)((uint8_t*)re - (uint8_t*)rb) / e;
  cudaStream_t s = 0;
  const size_t need = set_op_workspace_impl(op, na, nb, e);
  void* ws = nullptr;
  RFX_CUDA_TRY(cudaMallocAsync(&ws, need, s));
  rfx_status st = set_op_impl(op, result, size, lb, na, rb, nb, e, ws, need, s);
  if (st == RFX_OK) scale_kernel<<<1, 1, 0, s>>>(size, e);
  cudaFreeAsync(ws, s);
  if (st != RFX_OK) return st;
  RFX_CUDA_TRY(cudaStreamSynchronize(s));
  return RFX_OK;
}
}  // namespace

}  // namespace rfx

using namespace rfx;

extern "C" size_t rfx_set_op_workspace(uint32_t op, uint64_t na, uint64_t nb, uint32_t elem_bytes) {
  return set_op_workspace_impl(op, na, nb, elem_bytes);
}

extern "C" rfx_status rfx_set_op(uint32_t op, void* out, uint64_t* d_count, const void* a, uint64_t na, const void* b,
                                 uint64_t nb, uint32_t elem_bytes, void* workspace, size_t workspace_bytes, void* stream) {
  return set_op_impl(op, out, d_count, a, na, b, nb, elem_bytes, workspace, workspace_bytes, as_stream(stream));
}

extern "C" size_t rfx_unique_workspace(uint64_t n, uint32_t elem_bytes) { return unique_workspace_impl(n, elem_bytes); }

extern "C" rfx_status rfx_unique(void* data, uint64_t n, uint64_t* d_count, uint32_t elem_bytes, void* workspace,
                                 size_t workspace_bytes, void* stream) {
  return unique_impl(data, n, d_count, elem_bytes, workspace, workspace_bytes, as_stream(stream));
}

extern "C" rfx_status rfx_set_union_compat(void* result, uint64_t* size, void* lbegin, void* lend, void* rbegin,
                                           void* rend, uint32_t type) {
  return set_compat(RFX_SET_UNION, result, size, lbegin, lend, rbegin, rend, type);
}

extern "C" rfx_status rfx_difference_compat(void* result, uint64_t* size, void* lbegin, void* lend, void* rbegin,
                                            void* rend, uint32_t type) {
  return set_compat(RFX_SET_DIFFERENCE, result, size, lbegin, lend, rbegin, rend, type);
}

extern "C" rfx_status rfx_intersection_compat(void* result, uint64_t* size, void* lbegin, void* lend, void* rbegin,
                                              void* rend, uint32_t type) {
  return set_compat(RFX_SET_INTERSECTION, result, size, lbegin, lend, rbegin, rend, type);
}

// redfox::unique (Unique.cu:36-114): *size (device) holds the input bytes and receives
// the output bytes; types I8..I64.  A single element is left as it is, as in the
// reference.
extern "C" rfx_status rfx_unique_compat(void* begin, uint64_t* size, uint64_t type) {
  const uint32_t e = type_bytes(type);
  if (!e || e > 8) return RFX_ERR_UNSUPPORTED;
  if (!size) return RFX_ERR_INVALID;
  uint64_t bytes = 0;
  RFX_CUDA_TRY(cudaMemcpy(&bytes, size, sizeof(bytes), cudaMemcpyDeviceToHost));
  const uint64_t n = bytes / e;
  if (n <= 1) return RFX_OK;
  cudaStream_t s = 0;
  const size_t need = unique_workspace_impl(n, e);
  void* ws = nullptr;
  RFX_CUDA_TRY(cudaMallocAsync(&ws, need, s));
  rfx_status st = unique_impl(begin, n, size, e, ws, need, s);
  if (st == RFX_OK) scale_kernel<<<1, 1, 0, s>>>(size, e);
  cudaFreeAsync(ws, s);
  if (st != RFX_OK) return st;
  RFX_CUDA_TRY(cudaStreamSynchronize(s));
  return RFX_OK;
}
