// reduce_abi.cu -- C ABI of reduce-by-key / count, and the reference-compatible
// count_* / total_64_32 entries with device-resident byte sizes (Reduce.cu).
#include <cstdlib>
#include <cstring>

#include "host_common.h"
#include "reduce_kernels.cuh"
#include "tune.h"

namespace rfx {
namespace {

struct RedLayout {
  uint32_t* flags;
  uint32_t* counter;
  SegPair* agg;
  SegPair* inc;
  size_t clear_bytes;
  size_t total;
};

RedLayout red_layout(void* ws, uint64_t n) {
  RedLayout L;
  const uint64_t tiles = (n + kRedTile - 1) / kRedTile + 1;
  Carver c(ws);
  L.flags = c.take<uint32_t>(tiles);
  L.counter = c.take<uint32_t>(1);
  L.clear_bytes = align_up(c.used, 256);
  c.used = L.clear_bytes;
  L.agg = c.take<SegPair>(tiles);
  L.inc = c.take<SegPair>(tiles);
  L.total = align_up(c.used, 256);
  return L;
}

template <int K, int VK>
rfx_status launch(ReduceArgs& a, cudaStream_t s) {
  auto k = reduce_by_key_kernel<K, VK>;
  const uint64_t tiles = (a.n_max + kRedTile - 1) / kRedTile;
  const int grid = persistent_grid((const void*)k, kRedThreads, 0, tiles ? tiles : 1);
  k<<<grid, kRedThreads, 0, s>>>(a);
  RFX_CUDA_TRY(cudaGetLastError());
  return RFX_OK;
}

template <int K>
rfx_status launch_k(ReduceArgs& a, int vk, cudaStream_t s) {
  switch (vk) {
    case VAL_NONE: return launch<K, VAL_NONE>(a, s);
    case VAL_U32: return launch<K, VAL_U32>(a, s);
    case VAL_I64: return launch<K, VAL_I64>(a, s);
    default: return RFX_ERR_UNSUPPORTED;
  }
}

rfx_status run_reduce(ReduceArgs& a, uint32_t kb, int vk, void* ws, size_t ws_bytes, cudaStream_t s) {
  RedLayout L = red_layout(ws, a.n_max);
  if (!ws || ws_bytes < L.total) return RFX_ERR_WORKSPACE;
  a.flags = L.flags;
  a.tile_counter = L.counter;
  a.agg = L.agg;
  a.inc = L.inc;
  a.err = device_error_word();
  if (!a.err) return RFX_ERR_CUDA;
  RFX_CUDA_TRY(cudaMemsetAsync(ws, 0, L.clear_bytes, s));
  switch (kb) {
    case 1: return launch_k<1>(a, vk, s);
    case 2: return launch_k<2>(a, vk, s);
    case 4: return launch_k<4>(a, vk, s);
    case 8: return launch_k<8>(a, vk, s);
    case 16: return launch_k<16>(a, vk, s);
    case 32: return launch_k<32>(a, vk, s);
    default: return RFX_ERR_UNSUPPORTED;
  }
}

bool aligned_to(const void* p, uint32_t b) {
  return (reinterpret_cast<uintptr_t>(p) % (b < 16 ? b : 16)) == 0;
}

// Tiles of the TMA-staged tuple reduce: 256 (default) or 128 128-byte lines; records are
// sized for the smaller tile.
constexpr int kRowRedThreadsMin = 128;

struct RowLayout {
  SegRecord* records;
  uint32_t* counter;
  size_t total;
};

RowLayout row_layout(void* ws, uint64_t n, uint32_t row_bytes) {
  const uint64_t tile_rows = (uint64_t)kRowRedThreadsMin * kRingLineBytes / row_bytes;
  const uint64_t tiles = (n + tile_rows - 1) / tile_rows + 1;
  Carver c(ws);
  RowLayout L;
  L.records = c.take<SegRecord>(tiles);
  L.counter = c.take<uint32_t>(1);
  L.total = align_up(c.used, 256);
  return L;
}

// The chunked staged reduce: one look-back record per chunk (at most one chunk per
// resident block), and scratch for n / 4 groups (plus a floor for small inputs): a chunk
// whose groups do not fit its share -- more than one group per 4 rows -- runs its rows a
// second time, writing directly.
constexpr uint64_t kMaxChunks = 4096;
constexpr int kChunkStages = 3;
constexpr uint64_t kChunkRowsPerSlot = 4;

struct ChunkLayout {
  SegRecord* records;
  uint32_t* counter;
  size_t clear;
  uint8_t* keys;
  int64_t* sums;
  uint32_t* counts;
  uint64_t slots;
  size_t total;
};

ChunkLayout chunk_layout(void* ws, uint64_t n) {
  Carver c(ws);
  ChunkLayout L;
  L.records = c.take<SegRecord>(kMaxChunks);
  L.counter = c.take<uint32_t>(1);
  L.clear = align_up(c.used, 256);
  L.slots = n / kChunkRowsPerSlot + 65536;
  L.keys = c.take<uint8_t>(L.slots * 16);
  L.sums = c.take<int64_t>(L.slots);
  L.counts = c.take<uint32_t>(L.slots);
  L.total = align_up(c.used, 256);
  return L;
}

}  // namespace

size_t reduce_workspace_impl(uint64_t n) {
  const size_t a = red_layout(nullptr, n).total, b = row_layout(nullptr, n, 16).total;
  const size_t c = chunk_layout(nullptr, n).total;
  const size_t ab = a > b ? a : b;
  return ab > c ? ab : c;
}

rfx_status reduce_impl(const void* keys, uint64_t n, const uint64_t* d_n, uint32_t kb, const void* vals, uint32_t vk,
                       void* out_keys, void* out_vals, uint32_t* out_counts, uint64_t* d_groups, void* ws,
                       size_t ws_bytes, cudaStream_t s) {
  if (!d_groups || (!keys && n) || (!out_keys && n)) return RFX_ERR_INVALID;
  if (vk > VAL_I64 || (vk != VAL_NONE && !vals && n)) return RFX_ERR_INVALID;
  if (n && (!aligned_to(keys, kb) || !aligned_to(out_keys, kb))) return RFX_ERR_INVALID;
  ReduceArgs a;
  std::memset(&a, 0, sizeof(a));
  a.keys = static_cast<const uint8_t*>(keys);
  a.vals = vals;
  a.n_max = n;
  a.d_n = d_n;
  a.n_div = 1;
  a.out_keys = static_cast<uint8_t*>(out_keys);
  a.out_vals = out_vals;
  a.out_counts = out_counts;
  a.d_groups = d_groups;
  return run_reduce(a, kb, (int)vk, ws, ws_bytes, s);
}

}  // namespace rfx

using namespace rfx;

extern "C" size_t rfx_reduce_by_key_workspace(uint64_t n) { return reduce_workspace_impl(n); }

extern "C" rfx_status rfx_reduce_by_key(const void* keys, uint64_t n, const uint64_t* d_n, uint32_t key_bytes,
                                        const void* values, uint32_t value_kind, void* out_keys, void* out_values,
                                        uint32_t* out_counts, uint64_t* d_groups, void* workspace,
                                        size_t workspace_bytes, void* stream) {
  return reduce_impl(keys, n, d_n, key_bytes, values, value_kind, out_keys, out_values, out_counts, d_groups,
                     workspace, workspace_bytes, as_stream(stream));
}

namespace {
// Reference byte-size convention (Reduce.cu): *key_size / *value_size hold bytes on the
// device on entry and are overwritten with the output byte sizes.  The reference reads
// them back to the host first (a synchronous copy); so does this entry, to size the
// launch, then it runs on the default stream and synchronises.
rfx_status count_like(const void* k, const void* v, void* ok, void* ov, uint64_t* key_size, uint64_t* value_size,
                      uint32_t kb, int vk) {
  if (!key_size || !value_size) return RFX_ERR_INVALID;
  uint64_t kbytes = 0;
  RFX_CUDA_TRY(cudaMemcpy(&kbytes, key_size, sizeof(kbytes), cudaMemcpyDeviceToHost));
  const uint64_t n = kbytes / kb;
  const size_t need = reduce_workspace_impl(n);
  void* ws = nullptr;
  cudaStream_t s = 0;
  RFX_CUDA_TRY(cudaMallocAsync(&ws, need, s));
  uint64_t* groups = nullptr;
  RFX_CUDA_TRY(cudaMallocAsync(&groups, sizeof(uint64_t), s));
  ReduceArgs a;
  std::memset(&a, 0, sizeof(a));
  a.keys = static_cast<const uint8_t*>(k);
  a.vals = v;
  a.n_max = n;  // read above; *key_size is overwritten with the output size
  a.d_n = nullptr;
  a.n_div = 1;
  a.out_keys = static_cast<uint8_t*>(ok);
  a.out_vals = ov;
  a.d_groups = groups;
  a.d_groups_bytes_k = key_size;
  a.d_groups_bytes_v = value_size;
  rfx_status st = run_reduce(a, kb, vk, ws, need, s);
  cudaFreeAsync(ws, s);
  cudaFreeAsync(groups, s);
  if (st != RFX_OK) return st;
  RFX_CUDA_TRY(cudaStreamSynchronize(s));
  return RFX_OK;
}
}  // namespace

// count_{8,16,32,128,256} (Reduce.cu:175-660): u32 column summed per run of keys.
extern "C" rfx_status rfx_count_compat(const void* key_begin, const void* value_begin, void* result_key_begin,
                                       void* result_value_begin, uint64_t* key_size, uint64_t* value_size,
                                       uint32_t key_bytes) {
  return count_like(key_begin, value_begin, result_key_begin, result_value_begin, key_size, value_size, key_bytes,
                    VAL_U32);
}

// total_64_32 (Reduce.cu:1138-1215): u64 keys, u32 values summed.
extern "C" rfx_status rfx_total_64_32_compat(const void* key_begin, const void* value_begin, void* result_key_begin,
                                             void* result_value_begin, uint64_t* key_size, uint64_t* value_size) {
  return count_like(key_begin, value_begin, result_key_begin, result_value_begin, key_size, value_size, 8, VAL_U32);
}

// The exact int64 SUM the reference lacks, with the same byte-size convention.
extern "C" rfx_status rfx_total_i64_compat(const void* key_begin, const void* value_begin, void* result_key_begin,
                                           void* result_value_begin, uint64_t* key_size, uint64_t* value_size,
                                           uint32_t key_bytes) {
  return count_like(key_begin, value_begin, result_key_begin, result_value_begin, key_size, value_size, key_bytes,
                    VAL_I64);
}

namespace rfx {
namespace {
template <int RB, int OKB>
rfx_status launch_tuples(TupleReduceArgs& a, cudaStream_t s) {
  auto k = reduce_tuples_kernel<RB, OKB>;
  const uint64_t tiles = (a.r.n_max + kRedTile - 1) / kRedTile;
  const int grid = persistent_grid((const void*)k, kRedThreads, 0, tiles ? tiles : 1);
  k<<<grid, kRedThreads, 0, s>>>(a);
  RFX_CUDA_TRY(cudaGetLastError());
  return RFX_OK;
}
template <int RB>
rfx_status launch_tuples_o(uint32_t okb, TupleReduceArgs& a, cudaStream_t s) {
  switch (okb) {
    case 4: return launch_tuples<RB, 4>(a, s);
    case 8: return launch_tuples<RB, 8>(a, s);
    case 16: return launch_tuples<RB, 16>(a, s);
    default: return RFX_ERR_UNSUPPORTED;
  }
}
}  // namespace
}  // namespace rfx

namespace rfx {
namespace {
// The TMA-staged form: rows 16-byte aligned; the workspace of the register-tiled form
// (kRedTile rows per tile, 52 bytes per tile) always covers its records (32 bytes per
// tile of at least kRedTile rows).
template <int RB, int SHAPE, int NT>
rfx_status launch_rows(const void* rows, uint64_t n, RowReduceArgs& a, cudaStream_t s) {
  auto k = reduce_rows_kernel<RB, SHAPE, kRowRedStages, NT>;
  const size_t smem = (size_t)kRowRedStages * NT * kRingLineBytes + 1024;
  RFX_CUDA_TRY(allow_smem((const void*)k, smem));
  CUtensorMap map;
  const uint64_t lines = n * RB / kRingLineBytes;
  a.full_lines = encode_line_map(&map, rows, lines, NT) ? lines : 0;
  const uint64_t tiles = (n * RB + NT * kRingLineBytes - 1) / (NT * kRingLineBytes);
  const int grid = persistent_grid((const void*)k, NT, smem, tiles ? tiles : 1);
  k<<<grid, NT, smem, s>>>(map, a);
  RFX_CUDA_TRY(cudaGetLastError());
  return RFX_OK;
}

// The chunked form (256-line tiles): chunks of whole tiles, one per block.
template <int RB, int SHAPE>
rfx_status launch_chunks(const void* rows, uint64_t n, const RowReduceArgs& a, const ChunkLayout& L,
                         cudaStream_t s) {
  constexpr int NT = 256;
  auto k = reduce_chunks_kernel<RB, SHAPE, kChunkStages, NT>;
  const size_t smem = (size_t)kChunkStages * NT * kRingLineBytes + 1024;
  RFX_CUDA_TRY(allow_smem((const void*)k, smem));
  ChunkReduceArgs ca;
  std::memset(&ca, 0, sizeof(ca));
  ca.r = a;
  ca.r.records = L.records;
  ca.r.tile_counter = L.counter;
  CUtensorMap map;
  const uint64_t lines = n * RB / kRingLineBytes;
  ca.r.full_lines = encode_line_map(&map, rows, lines, NT) ? lines : 0;
  const uint64_t tiles = (n * RB + NT * kRingLineBytes - 1) / (NT * kRingLineBytes);
  const uint64_t grid = (uint64_t)persistent_grid((const void*)k, NT, smem, tiles ? tiles : 1);
  ca.tiles_per_chunk = tiles ? (tiles + grid - 1) / grid : 1;
  const uint64_t chunks = tiles ? (tiles + ca.tiles_per_chunk - 1) / ca.tiles_per_chunk : 1;
  if (chunks > kMaxChunks) return RFX_ERR_UNSUPPORTED;
  const uint64_t cap = L.slots / chunks;
  ca.cap = (uint32_t)(cap < 0xffffffffull ? cap : 0xffffffffull);
  ca.s_keys = L.keys;
  ca.s_sums = L.sums;
  ca.s_counts = L.counts;
  k<<<(int)chunks, NT, smem, s>>>(map, ca);
  RFX_CUDA_TRY(cudaGetLastError());
  return RFX_OK;
}

// The warp-chunked form: 4 KB tiles (32 lines), each warp of a block streams its own
// sub-chunk of whole tiles.
constexpr int kWarpChunkWarps = 8;
constexpr int kWarpChunkStages = 3;
// On inputs above kWarpChunkSpreadBytes, tiles of a warp's sub-chunk at the most (256 KB),
// unless that would take more than kMaxChunks chunks: one sub-chunk per resident warp spreads
// the warps streaming at once over the whole input, a page apart each, and on inputs of many
// GB the address translations miss (a 10 GB reduce ran at half speed); smaller sub-chunks,
// claimed in order, keep them within a few hundred MB.  Below that size the per-chunk costs
// of smaller sub-chunks outweigh it (a 0.96 GB reduce: 0.35 ms with one sub-chunk per warp,
// 0.44 ms with 256 KB ones).
constexpr uint64_t kWarpChunkMaxTiles = 64;
constexpr uint64_t kWarpChunkSpreadBytes = 2ull << 30;

template <int RB, int SHAPE>
rfx_status launch_warps(const void* rows, uint64_t n, const RowReduceArgs& a, const ChunkLayout& L,
                        cudaStream_t s) {
  constexpr int W = kWarpChunkWarps, LINES = 32;
  auto k = reduce_warps_kernel<RB, SHAPE, kWarpChunkStages, W>;
  const size_t smem = (size_t)W * kWarpChunkStages * LINES * kRingLineBytes + 1024;
  RFX_CUDA_TRY(allow_smem((const void*)k, smem));
  ChunkReduceArgs ca;
  std::memset(&ca, 0, sizeof(ca));
  ca.r = a;
  ca.r.records = L.records;
  ca.r.tile_counter = L.counter;
  CUtensorMap map;
  const uint64_t lines = n * RB / kRingLineBytes;
  ca.r.full_lines = encode_line_map(&map, rows, lines, LINES) ? lines : 0;
  const uint64_t tiles = (n * RB + LINES * kRingLineBytes - 1) / (LINES * kRingLineBytes);
  const uint64_t want = tiles ? (tiles + W - 1) / W : 1;
  const uint64_t grid = (uint64_t)persistent_grid((const void*)k, W * 32, smem, want);
  ca.tiles_per_chunk = tiles ? (tiles + grid * W - 1) / (grid * W) : 1;   // tiles per warp
  if (n * RB > kWarpChunkSpreadBytes && ca.tiles_per_chunk > kWarpChunkMaxTiles) {
    const uint64_t floor_tpc = (tiles + kMaxChunks * W - 1) / (kMaxChunks * W);
    ca.tiles_per_chunk = floor_tpc > kWarpChunkMaxTiles ? floor_tpc : kWarpChunkMaxTiles;
  }
  const uint64_t blocks = tiles ? (tiles + ca.tiles_per_chunk * W - 1) / (ca.tiles_per_chunk * W) : 1;
  if (blocks > kMaxChunks) return RFX_ERR_UNSUPPORTED;
  const uint64_t cap = L.slots / (blocks * W);
  ca.cap = (uint32_t)(cap < 0xffffffffull ? cap : 0xffffffffull);
  ca.s_keys = L.keys;
  ca.s_sums = L.sums;
  ca.s_counts = L.counts;
  k<<<(int)blocks, W * 32, smem, s>>>(map, ca);
  RFX_CUDA_TRY(cudaGetLastError());
  return RFX_OK;
}

// Variant 0: warp-chunked; 1: block-chunked, 256-line tiles; 2: look-back per tile,
// 256-line tiles; 3: look-back per tile, 128-line tiles.
template <int RB, int SHAPE>
rfx_status launch_rows_v(int v, const void* rows, uint64_t n, RowReduceArgs& a, void* ws, cudaStream_t s) {
  if (v <= 1) {
    const ChunkLayout L = chunk_layout(ws, n);
    RFX_CUDA_TRY(cudaMemsetAsync(ws, 0, L.clear, s));
    return v == 0 ? launch_warps<RB, SHAPE>(rows, n, a, L, s) : launch_chunks<RB, SHAPE>(rows, n, a, L, s);
  }
  RFX_CUDA_TRY(cudaMemsetAsync(ws, 0, row_layout(ws, n, RB).total, s));
  return v == 2 ? launch_rows<RB, SHAPE, 256>(rows, n, a, s) : launch_rows<RB, SHAPE, 128>(rows, n, a, s);
}

rfx_status reduce_rows_staged(const void* rows, uint64_t n, const uint64_t* d_n, uint32_t row_bytes,
                              uint32_t key_shift, uint32_t value_shift, uint64_t val_mask, void* out_keys,
                              uint32_t out_key_bytes, int64_t* out_sums, uint32_t* out_counts, uint64_t* d_groups,
                              void* workspace, uint32_t* err, cudaStream_t s) {
  const RowLayout L = row_layout(workspace, n, row_bytes);
  RowReduceArgs a;
  std::memset(&a, 0, sizeof(a));
  a.rows = static_cast<const uint8_t*>(rows);
  a.n_max = n;
  a.d_n = d_n;
  a.key_shift = key_shift;
  a.val_shift = value_shift;
  a.val_mask = val_mask;
  a.out_key_bytes = out_key_bytes;
  a.out_keys = static_cast<uint8_t*>(out_keys);
  a.out_sums = out_sums;
  a.out_counts = out_counts;
  a.d_groups = d_groups;
  a.records = L.records;
  a.tile_counter = L.counter;
  a.err = err;
  const int shape = (row_bytes == 16 && value_shift == 0 && val_mask == ~0ull && key_shift == 96)   ? 1
                    : (row_bytes == 16 && value_shift == 0 && val_mask == ~0ull && key_shift == 64) ? 2
                                                                                                   : 0;
  auto run = [&](int v) -> rfx_status {
    if (shape == 1) return launch_rows_v<16, ROW16_K32_V64>(v, rows, n, a, workspace, s);
    if (shape == 2) return launch_rows_v<16, ROW16_K64_V64>(v, rows, n, a, workspace, s);
    switch (row_bytes) {
      case 4: return launch_rows_v<4, ROW_GENERIC>(v, rows, n, a, workspace, s);
      case 8: return launch_rows_v<8, ROW_GENERIC>(v, rows, n, a, workspace, s);
      default: return launch_rows_v<16, ROW_GENERIC>(v, rows, n, a, workspace, s);
    }
  };
  const uint64_t shape_key = ((uint64_t)row_bytes << 32) | ((uint64_t)shape << 24) | (key_shift << 8) | value_shift;
  return run(tune_pick(TUNE_REDUCE_ROWS, shape_key, n, 4, run, s));
}
}  // namespace
}  // namespace rfx

extern "C" rfx_status rfx_reduce_tuples(const void* rows, uint64_t n, const uint64_t* d_n, uint32_t row_bytes,
                                        uint32_t key_shift, uint32_t value_shift, uint32_t value_bits,
                                        void* out_keys, uint32_t out_key_bytes, int64_t* out_sums,
                                        uint32_t* out_counts, uint64_t* d_groups, void* workspace,
                                        size_t workspace_bytes, void* stream) {
  if (!(row_bytes == 4 || row_bytes == 8 || row_bytes == 16) || key_shift >= row_bytes * 8u || value_bits == 0 ||
      value_bits > 64 || value_shift + value_bits > row_bytes * 8u)
    return RFX_ERR_UNSUPPORTED;
  if (!(out_key_bytes == 4 || out_key_bytes == 8 || out_key_bytes == 16)) return RFX_ERR_UNSUPPORTED;
  if (!d_groups || (n && (!rows || !out_keys))) return RFX_ERR_INVALID;
  if (n && (reinterpret_cast<uintptr_t>(rows) % row_bytes) != 0) return RFX_ERR_INVALID;
  cudaStream_t s = as_stream(stream);
  RedLayout L = red_layout(workspace, n);
  if (!workspace || workspace_bytes < L.total) return RFX_ERR_WORKSPACE;
  uint32_t* err = device_error_word();
  if (!err) return RFX_ERR_CUDA;
  const uint64_t vmask = value_bits >= 64 ? ~0ull : ((1ull << value_bits) - 1);
  if ((reinterpret_cast<uintptr_t>(rows) & 15u) == 0 && std::getenv("RFX_REDUCE_REGS") == nullptr) {
    if (workspace_bytes < row_layout(nullptr, n, row_bytes).total || workspace_bytes < chunk_layout(nullptr, n).total)
      return RFX_ERR_WORKSPACE;
    return reduce_rows_staged(rows, n, d_n, row_bytes, key_shift, value_shift, vmask, out_keys, out_key_bytes,
                              out_sums, out_counts, d_groups, workspace, err, s);
  }
  RFX_CUDA_TRY(cudaMemsetAsync(workspace, 0, L.clear_bytes, s));
  TupleReduceArgs a;
  std::memset(&a, 0, sizeof(a));
  a.r.keys = static_cast<const uint8_t*>(rows);
  a.r.n_max = n;
  a.r.d_n = d_n;
  a.r.n_div = 1;
  a.r.out_keys = static_cast<uint8_t*>(out_keys);
  a.r.out_vals = out_sums;
  a.r.out_counts = out_counts;
  a.r.d_groups = d_groups;
  a.r.flags = L.flags;
  a.r.tile_counter = L.counter;
  a.r.agg = L.agg;
  a.r.inc = L.inc;
  a.r.err = err;
  a.key_shift = key_shift;
  a.val_shift = value_shift;
  a.val_mask = value_bits >= 64 ? ~0ull : ((1ull << value_bits) - 1);
  switch (row_bytes) {
    case 4: return launch_tuples_o<4>(out_key_bytes, a, s);
    case 8: return launch_tuples_o<8>(out_key_bytes, a, s);
    default: return launch_tuples_o<16>(out_key_bytes, a, s);
  }
}
