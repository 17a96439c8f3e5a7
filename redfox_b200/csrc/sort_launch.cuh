// sort_launch.cuh -- host launchers of the radix sort, instantiated per key width in
// sort_k{1,2,4,8,16,32,64}.cu.
#pragma once

#include "host_common.h"
#include "sort_kernels.cuh"
#include "sort_onesweep.cuh"
#include "tune.h"

namespace rfx {

struct SortPlan {
  uint8_t* keys;
  uint8_t* vals;
  const uint8_t* src_keys;   // when set, the first pass and the histogram read these instead
  const uint8_t* src_vals;   // of keys / vals, which then only receive (out-of-place sort)
  uint8_t* alt_keys;
  uint8_t* alt_vals;
  uint8_t* alt2_keys;   // a second pair of alternate buffers (may be null): an odd number
  uint8_t* alt2_vals;   // of passes >= 3 then ends in keys / vals without a copy
  uint64_t n;
  uint32_t begin_bit;
  uint32_t end_bit;     // end_bit - begin_bit <= 128
  uint32_t passes;
  uint32_t* ghist;      // [passes][256]
  uint32_t* trivial;    // [passes]
  uint32_t* done;       // 1
  uint32_t* counters;   // [passes]
  uint32_t* status;     // [passes][tiles][256]
  uint64_t tiles;
  bool skip_trivial;
  uint32_t* host_trivial;  // pinned or pageable host copy for skip_trivial
  uint32_t* err;
  cudaStream_t stream;
  int executed;         // out: passes run
  bool in_alt;          // out: the sorted data ended in the alternate buffers
};

// Look-back status words are laid out per tile of the smallest tile any pass variant
// uses, so every variant's tiles fit the same status area.
template <int K, int V>
constexpr int min_sort_tile() {
  if constexpr (V == 0 && (K == 4 || K == 8 || K == 16)) {
    constexpr int a = SortTuning<K, V>::TILE, b = OsTuning<K, OsIpt<K>::SMALL>::TILE;
    constexpr int c = OsTuning<K, OsIpt<K>::DEF>::TILE, d = OsTuning<K, OsIpt<K>::ALT>::TILE;
    constexpr int ab = a < b ? a : b, cd = c < d ? c : d;
    return ab < cd ? ab : cd;
  } else {
    return SortTuning<K, V>::TILE;
  }
}

template <int K, int V>
uint64_t sort_tiles(uint64_t n) {
  return (n + min_sort_tile<K, V>() - 1) / min_sort_tile<K, V>();
}

template <int K, int V>
rfx_status run_sort_kv(SortPlan& s) {
  // histogram of every digit
  {
    auto hk = sort_histogram_kernel<K>;
    const uint64_t blocks = (s.n + kSortThreads * 8 - 1) / (kSortThreads * 8);
    const int grid = persistent_grid((const void*)hk, kSortThreads, 0, blocks ? blocks : 1);
    hk<<<grid, kSortThreads, 0, s.stream>>>(s.src_keys ? s.src_keys : s.keys, s.n, s.begin_bit, s.end_bit, s.passes,
                                            s.ghist, s.trivial, s.done);
    RFX_CUDA_TRY(cudaGetLastError());
  }
  uint32_t triv[kMaxSortPasses] = {0};
  if (s.skip_trivial) {
    RFX_CUDA_TRY(cudaMemcpyAsync(s.host_trivial, s.trivial, s.passes * sizeof(uint32_t), cudaMemcpyDeviceToHost, s.stream));
    RFX_CUDA_TRY(cudaStreamSynchronize(s.stream));
    for (uint32_t p = 0; p < s.passes; ++p) triv[p] = s.host_trivial[p];
  }
  // Pass variants: 0 = the per-tile pass (every width, values too; the next tile's keys
  // prefetched into shared memory); 1 / 2 / 3 = the pipelined onesweep pass (TMA stages +
  // a look-back warp, one block per SM) with its default / fewer / other items per thread,
  // where it applies: keys without values in 4/8/16-byte containers on 16-byte aligned
  // buffers; 4 = the per-tile pass ranking with __match_any_sync instead of bit ballots
  // (same keys).  The autotuner may pick per size class.
  const size_t tile_smem = SortBuffers<K, V>::SMEM;
  RFX_CUDA_TRY(allow_smem((const void*)sort_pass_kernel<K, V>, tile_smem));
  if constexpr (V == 0 && (K == 4 || K == 8 || K == 16))
    RFX_CUDA_TRY(allow_smem((const void*)sort_pass_kernel<K, V, true>, tile_smem));
  const int tile_grid = persistent_grid((const void*)sort_pass_kernel<K, V>, SortTuning<K, V>::THREADS, tile_smem,
                                        s.tiles ? s.tiles : 1);
  constexpr bool kOnesweep = V == 0 && (K == 4 || K == 8 || K == 16);
  bool os_ok = false;
  int os_grid[3] = {0, 0, 0};   // default, small, alternative tiles
  if constexpr (kOnesweep) {
    os_ok = ((reinterpret_cast<uintptr_t>(s.keys) | reinterpret_cast<uintptr_t>(s.alt_keys) |
              reinterpret_cast<uintptr_t>(s.alt2_keys)) & 15u) == 0;
    if (os_ok) {
      auto prep = [&](const void* k, size_t smem, int tile, int* grid) -> rfx_status {
        const uint64_t ot = (s.n + tile - 1) / tile;
        if (ot > s.tiles) return RFX_ERR_INVALID;   // the status area holds s.tiles tiles
        RFX_CUDA_TRY(allow_smem(k, smem));
        *grid = persistent_grid(k, kOsThreads, smem, ot ? ot : 1);
        return RFX_OK;
      };
      using TD = OsTuning<K, OsIpt<K>::DEF>;
      using TS = OsTuning<K, OsIpt<K>::SMALL>;
      using TL = OsTuning<K, OsIpt<K>::ALT>;
      rfx_status st = prep((const void*)sort_onesweep_kernel<K, TD::IPT>, TD::SMEM, TD::TILE, &os_grid[0]);
      if (st == RFX_OK) st = prep((const void*)sort_onesweep_kernel<K, TS::IPT>, TS::SMEM, TS::TILE, &os_grid[1]);
      if (st == RFX_OK) st = prep((const void*)sort_onesweep_kernel<K, TL::IPT>, TL::SMEM, TL::TILE, &os_grid[2]);
      if (st == RFX_ERR_INVALID) os_ok = false;   // not expected: the per-tile pass runs instead
      else if (st != RFX_OK) return st;
    }
  }
  // Buffers the passes go through: b[0] = keys, pass j reads b[j] and writes b[j + 1].
  // An even number of passes alternates keys / alt and ends in keys; an odd number >= 3
  // goes keys -> alt -> alt2 -> keys and then alternates, so it ends in keys too; a single
  // pass (or no second buffer) ends in alt, which the caller copies back.
  uint32_t npass = 0;
  for (uint32_t p = 0; p < s.passes; ++p) npass += triv[p] ? 0u : 1u;
  uint8_t* kb[kMaxSortPasses + 1];
  uint8_t* vb[kMaxSortPasses + 1];
  const bool three = (npass % 2 == 1) && npass >= 3 && s.alt2_keys && (V == 0 || s.alt2_vals);
  for (uint32_t j = 0; j <= npass; ++j) {
    const bool at_keys = three ? (j == 0 || (j >= 3 && j % 2 == 1)) : (j % 2 == 0);
    const bool at_alt2 = three && j == 2;
    kb[j] = at_keys ? s.keys : at_alt2 ? s.alt2_keys : s.alt_keys;
    vb[j] = at_keys ? s.vals : at_alt2 ? s.alt2_vals : s.alt_vals;
  }
  if (s.src_keys) {
    // out of place: the first pass reads the source (never written); a single pass writes
    // straight into keys / vals
    kb[0] = const_cast<uint8_t*>(s.src_keys);
    vb[0] = const_cast<uint8_t*>(s.src_vals);
    if (npass == 1) {
      kb[1] = s.keys;
      vb[1] = s.vals;
    }
  }
  s.executed = 0;
  s.in_alt = npass ? kb[npass] != s.keys : false;   // no pass at all: the data is where it was
  for (uint32_t p = 0; p < s.passes; ++p) {
    if (triv[p]) continue;
    SortPassArgs a;
    a.keys_in = kb[s.executed];
    a.keys_out = kb[s.executed + 1];
    a.vals_in = vb[s.executed];
    a.vals_out = vb[s.executed + 1];
    a.n = s.n;
    a.shift = s.begin_bit + 8 * p;
    const uint32_t w = s.end_bit - a.shift < 8 ? s.end_bit - a.shift : 8;
    a.mask = (1u << w) - 1;
    a.gexcl = s.ghist + p * kRadix;
    a.status = s.status + (uint64_t)p * s.tiles * kRadix;
    a.tile_counter = s.counters + p;
    a.err = s.err;
    // a pass reads kin and writes kout only, so a candidate can run again (the tuner
    // times each one); the look-back words and the tile counter are cleared between runs
    bool fresh = true;
    auto launch = [&](int v) -> rfx_status {
      if (!fresh) {
        RFX_CUDA_TRY(cudaMemsetAsync(a.status, 0, (size_t)s.tiles * kRadix * sizeof(uint32_t), s.stream));
        RFX_CUDA_TRY(cudaMemsetAsync(a.tile_counter, 0, sizeof(uint32_t), s.stream));
      }
      fresh = false;
      if constexpr (kOnesweep) {
        using TD = OsTuning<K, OsIpt<K>::DEF>;
        using TS = OsTuning<K, OsIpt<K>::SMALL>;
        using TL = OsTuning<K, OsIpt<K>::ALT>;
        if (v == 4)
          sort_pass_kernel<K, V, true><<<tile_grid, SortTuning<K, V>::THREADS, tile_smem, s.stream>>>(a);
        else if (os_ok && v == 1)
          sort_onesweep_kernel<K, TD::IPT><<<os_grid[0], kOsThreads, TD::SMEM, s.stream>>>(a);
        else if (os_ok && v == 2)
          sort_onesweep_kernel<K, TS::IPT><<<os_grid[1], kOsThreads, TS::SMEM, s.stream>>>(a);
        else if (os_ok && v == 3)
          sort_onesweep_kernel<K, TL::IPT><<<os_grid[2], kOsThreads, TL::SMEM, s.stream>>>(a);
        else
          sort_pass_kernel<K, V><<<tile_grid, SortTuning<K, V>::THREADS, tile_smem, s.stream>>>(a);
      } else {
        sort_pass_kernel<K, V><<<tile_grid, SortTuning<K, V>::THREADS, tile_smem, s.stream>>>(a);
      }
      RFX_CUDA_TRY(cudaGetLastError());
      return RFX_OK;
    };
    const int v = os_ok ? tune_pick(TUNE_SORT_PASS, (uint64_t)K << 8 | V, s.n, 5, launch, s.stream) : 0;
    rfx_status st = launch(v);
    if (st != RFX_OK) return st;
    ++s.executed;
  }
  return RFX_OK;
}

template <int K>
rfx_status run_sort(SortPlan& s, uint32_t vbytes) {
  switch (vbytes) {
    case 0: return run_sort_kv<K, 0>(s);
    case 1: return run_sort_kv<K, 1>(s);
    case 2: return run_sort_kv<K, 2>(s);
    case 4: return run_sort_kv<K, 4>(s);
    case 8: return run_sort_kv<K, 8>(s);
    case 16: return run_sort_kv<K, 16>(s);
    default: return RFX_ERR_UNSUPPORTED;
  }
}

template <int K>
uint64_t sort_tiles_for(uint64_t n, uint32_t vbytes) {
  switch (vbytes) {
    case 0: return sort_tiles<K, 0>(n);
    case 1: return sort_tiles<K, 1>(n);
    case 2: return sort_tiles<K, 2>(n);
    case 4: return sort_tiles<K, 4>(n);
    case 8: return sort_tiles<K, 8>(n);
    default: return sort_tiles<K, 16>(n);
  }
}

#define RFX_INSTANTIATE_SORT(K)                                  \
  template rfx_status run_sort<K>(SortPlan&, uint32_t);          \
  template uint64_t sort_tiles_for<K>(uint64_t, uint32_t);

}  // namespace rfx
