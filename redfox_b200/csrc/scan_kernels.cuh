// scan_kernels.cuh -- select / arith / project / filter-aggregate kernels over packed
// rows, templated on the input and output container widths (bytes).
//
// Layout in HBM: a relation is an array of packed tuples (the reference's BasicType
// images), row-major, 1..64 bytes per row.  Each thread owns whole rows; rows are loaded
// with the widest vector access the container allows.  Fields are cut out of a per-thread
// limb slot in shared memory laid out structure-of-arrays (limb l of thread t at
// [l * THREADS + t]), so the descriptor-chosen limb index is a uniform address offset and
// every access is bank-conflict free.
#pragma once

#include "rfx_device.cuh"
#include "scan_program.h"

namespace rfx {

constexpr int kScanThreads = 256;
constexpr int kScanRowsPerThread = 2;
constexpr int kScanTile = kScanThreads * kScanRowsPerThread;

template <int W>
struct Limbs {
  static constexpr int N = W <= 8 ? 1 : W / 8;
};

// ------------------------------------------------------------------ row load / store
template <int W>
__device__ __forceinline__ void load_row(const uint8_t* base, uint64_t i, uint64_t (&L)[Limbs<W>::N]) {
  if constexpr (W == 1) {
    L[0] = __ldg(base + i);
  } else if constexpr (W == 2) {
    L[0] = __ldg(reinterpret_cast<const uint16_t*>(base) + i);
  } else if constexpr (W == 4) {
    L[0] = __ldg(reinterpret_cast<const uint32_t*>(base) + i);
  } else if constexpr (W == 8) {
    L[0] = __ldg(reinterpret_cast<const unsigned long long*>(base) + i);
  } else {
    const ulonglong2* p = reinterpret_cast<const ulonglong2*>(base + i * W);
#pragma unroll
    for (int k = 0; k < W / 16; ++k) {
      ulonglong2 v = __ldg(p + k);
      L[2 * k] = v.x;
      L[2 * k + 1] = v.y;
    }
  }
}

template <int W>
__device__ __forceinline__ void store_row(uint8_t* base, uint64_t i, const uint64_t (&L)[Limbs<W>::N]) {
  if constexpr (W == 1) {
    base[i] = (uint8_t)L[0];
  } else if constexpr (W == 2) {
    reinterpret_cast<uint16_t*>(base)[i] = (uint16_t)L[0];
  } else if constexpr (W == 4) {
    reinterpret_cast<uint32_t*>(base)[i] = (uint32_t)L[0];
  } else if constexpr (W == 8) {
    reinterpret_cast<unsigned long long*>(base)[i] = L[0];
  } else {
    ulonglong2* p = reinterpret_cast<ulonglong2*>(base + i * W);
#pragma unroll
    for (int k = 0; k < W / 16; ++k) p[k] = make_ulonglong2(L[2 * k], L[2 * k + 1]);
  }
}

// ------------------------------------------------------------------ per-thread slots
// Shared memory per thread (SoA): the input row limbs, kMaxExt appended fields,
// kMaxRegs expression registers and the output row limbs.
template <int WIN, int WOUT>
struct Slots {
  static constexpr int NIN = Limbs<WIN>::N;
  static constexpr int NOUT = Limbs<WOUT>::N;
  static constexpr int PER_THREAD = NIN + kMaxExt + kMaxRegs + NOUT;
  static constexpr int IN = 0, EXT = NIN, REG = NIN + kMaxExt, OUT = NIN + kMaxExt + kMaxRegs;
};

__device__ __forceinline__ uint64_t wmask(uint32_t w) { return w >= 64 ? ~0ull : ((1ull << w) - 1); }

// Field of the input row held in the slot (lo limb + the next one for straddling fields).
template <int NIN>
__device__ __forceinline__ uint64_t slot_field(const uint64_t* s, const FieldLoc& f) {
  const uint64_t lo = s[f.limb * kScanThreads];
  const uint64_t hi = (f.limb + 1 < NIN) ? s[(f.limb + 1) * kScanThreads] : 0ull;
  const uint64_t v = f.off ? ((lo >> f.off) | (hi << (64 - f.off))) : lo;
  return v & wmask(f.width);
}

template <int NIN>
__device__ __forceinline__ uint64_t vfield(const ScanProgram& p, const uint64_t* in_slot,
                                           const uint64_t* ext_slot, uint32_t v) {
  if (v < p.nfields) return slot_field<NIN>(in_slot, p.in_loc[v]);
  return ext_slot[(v - p.nfields) * kScanThreads];
}

// All comparisons ANDed (select_field_constant / select_field_field, Select.h).
template <int NIN>
__device__ __forceinline__ bool eval_predicate(const ScanProgram& p, const uint64_t* in_slot) {
  bool pass = true;
  for (uint32_t c = 0; c < p.ncmp; ++c) {
    const CmpDesc& d = p.cmps[c];
    const uint64_t a = (d.a_var ? slot_field<NIN>(in_slot, p.in_loc[d.a_field]) : d.a_const) & d.tmask;
    const uint64_t b = (d.b_var ? slot_field<NIN>(in_slot, p.in_loc[d.b_field]) : d.b_const) & d.tmask;
    bool r;
    switch (d.op) {
      case RFX_EQ: r = a == b; break;
      case RFX_NE: r = a != b; break;
      case RFX_SLT: case RFX_LT: r = a < b; break;
      case RFX_SLE: case RFX_LE: r = a <= b; break;
      case RFX_SGT: case RFX_GT: r = a > b; break;
      default: r = a >= b; break;
    }
    pass = pass && r;
  }
  return pass;
}

// Expression program: appends the arith fields into the ext slot.
template <int NIN>
__device__ __forceinline__ void eval_arith(const ScanProgram& p, const uint64_t* in_slot,
                                           uint64_t* ext_slot, uint64_t* reg_slot) {
  for (uint32_t k = 0; k < p.ninstr; ++k) {
    const Instr ins = p.code[k];
    uint64_t* rd = reg_slot + ins.dst * kScanThreads;
    const uint64_t a = reg_slot[ins.a * kScanThreads];
    const uint64_t b = reg_slot[ins.b * kScanThreads];
    switch (ins.op) {
      case OP_FIELD: *rd = vfield<NIN>(p, in_slot, ext_slot, ins.field) & ins.imm; break;
      case OP_CONST: *rd = ins.imm; break;
      case OP_ADD64: *rd = a + b; break;
      case OP_SUB64: *rd = a - b; break;
      case OP_MUL64: *rd = a * b; break;
      case OP_ADD_S32: *rd = (uint64_t)(int64_t)(int32_t)(uint32_t)(a + b); break;
      case OP_SUB_S32: *rd = (uint64_t)(int64_t)(int32_t)(uint32_t)(a - b); break;
      case OP_MUL_S32: *rd = (uint64_t)(int64_t)(int32_t)(uint32_t)(a * b); break;
      case OP_ADD_U32: *rd = (uint32_t)(a + b); break;
      case OP_SUB_U32: *rd = (uint32_t)(a - b); break;
      case OP_MUL_U32: *rd = (uint32_t)(a * b); break;
      case OP_DIV_S32:
      case OP_MOD_S32: {
        const int32_t x = (int32_t)(uint32_t)a, y = (int32_t)(uint32_t)b;
        int32_t r;
        if (y == 0) r = 0;
        else if (x == INT32_MIN && y == -1) r = ins.op == OP_DIV_S32 ? x : 0;
        else r = ins.op == OP_DIV_S32 ? x / y : x % y;
        *rd = (uint64_t)(int64_t)r;
        break;
      }
      case OP_DIV_U32:
      case OP_MOD_U32: {
        const uint32_t x = (uint32_t)a, y = (uint32_t)b;
        *rd = y == 0 ? 0u : (ins.op == OP_DIV_U32 ? x / y : x % y);
        break;
      }
      case OP_DIV_S64:
      case OP_MOD_S64: {
        const int64_t x = (int64_t)a, y = (int64_t)b;
        int64_t r;
        if (y == 0) r = 0;
        else if (x == INT64_MIN && y == -1) r = ins.op == OP_DIV_S64 ? x : 0;
        else r = ins.op == OP_DIV_S64 ? x / y : x % y;
        *rd = (uint64_t)r;
        break;
      }
      case OP_DIV_U64:
      case OP_MOD_U64:
        *rd = b == 0 ? 0ull : (ins.op == OP_DIV_U64 ? a / b : a % b);
        break;
      case OP_STORE_EXT: ext_slot[ins.field * kScanThreads] = a & ins.imm; break;
      default: break;
    }
  }
}

// Projection into the output limbs (insert<> into a zeroed tuple, Project.h:58-100).
template <int NIN, int NOUT>
__device__ __forceinline__ void build_output(const ScanProgram& p, const uint64_t* in_slot,
                                             const uint64_t* ext_slot, uint64_t* out_slot,
                                             uint64_t (&O)[NOUT]) {
#pragma unroll
  for (int l = 0; l < NOUT; ++l) out_slot[l * kScanThreads] = 0;
  for (uint32_t k = 0; k < p.nout; ++k) {
    const FieldLoc f = p.out_loc[k];
    const uint32_t src = p.out_src[k];
    const uint64_t v = src == 0xff ? 0ull : (vfield<NIN>(p, in_slot, ext_slot, src) & wmask(f.width));
    out_slot[f.limb * kScanThreads] |= v << f.off;
    if (f.off && f.off + f.width > 64 && f.limb + 1 < NOUT) out_slot[(f.limb + 1) * kScanThreads] |= v >> (64 - f.off);
  }
#pragma unroll
  for (int l = 0; l < NOUT; ++l) O[l] = out_slot[l * kScanThreads];
}

// ------------------------------------------------------------------ compaction kernel
// MODE 0: select (the row itself is the output); MODE 1: select + arith + project;
// MODE 2: map without a predicate (arith / project alone), no compaction.
template <int WIN, int WOUT, int MODE>
__global__ void __launch_bounds__(kScanThreads)
scan_compact_kernel(const __grid_constant__ ScanProgram p, const uint8_t* __restrict__ in,
                    uint64_t n, uint8_t* __restrict__ out, uint64_t* __restrict__ d_count,
                    uint64_t* __restrict__ tile_status, uint32_t* __restrict__ tile_counter,
                    uint32_t* err) {
  using S = Slots<WIN, WOUT>;
  extern __shared__ __align__(16) uint64_t smem[];
  __shared__ uint32_t s_cnt[kScanRowsPerThread][kScanThreads / 32];
  __shared__ uint64_t s_prefix;
  __shared__ uint32_t s_tile;
  const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
  uint64_t* my = smem + t;
  uint64_t* in_slot = my + S::IN * kScanThreads;
  uint64_t* ext_slot = my + S::EXT * kScanThreads;
  uint64_t* reg_slot = my + S::REG * kScanThreads;
  uint64_t* out_slot = my + S::OUT * kScanThreads;
  const uint64_t num_tiles = (n + kScanTile - 1) / kScanTile;

  for (uint64_t iter = 0;; ++iter) {
    uint64_t tile;
    if constexpr (MODE == 2) {
      // no look-back: tiles are assigned statically
      tile = iter * gridDim.x + blockIdx.x;
    } else {
      // dynamic tile order keeps every look-back predecessor resident
      if (t == 0) s_tile = atomicAdd(tile_counter, 1u);
      __syncthreads();
      tile = s_tile;
    }
    if (tile >= num_tiles) break;
    uint64_t O[kScanRowsPerThread][S::NOUT];
    bool sel[kScanRowsPerThread];
#pragma unroll
    for (int j = 0; j < kScanRowsPerThread; ++j) {
      const uint64_t i = tile * kScanTile + (uint64_t)j * kScanThreads + t;
      sel[j] = false;
      if (i < n) {
        uint64_t L[S::NIN];
        load_row<WIN>(in, i, L);
#pragma unroll
        for (int l = 0; l < S::NIN; ++l) in_slot[l * kScanThreads] = L[l];
        if constexpr (MODE == 2) {
          sel[j] = true;
        } else {
          sel[j] = eval_predicate<S::NIN>(p, in_slot);
        }
        if constexpr (MODE == 0) {
#pragma unroll
          for (int l = 0; l < S::NOUT; ++l) O[j][l] = L[l];
        } else {
          if (sel[j]) {
            eval_arith<S::NIN>(p, in_slot, ext_slot, reg_slot);
            build_output<S::NIN, S::NOUT>(p, in_slot, ext_slot, out_slot, O[j]);
          }
        }
      }
    }
    if constexpr (MODE == 2) {
#pragma unroll
      for (int j = 0; j < kScanRowsPerThread; ++j) {
        const uint64_t i = tile * kScanTile + (uint64_t)j * kScanThreads + t;
        if (sel[j]) store_row<WOUT>(out, i, O[j]);
      }
      continue;
    }
    // ranks in input order (j-major, then warp, then lane)
    uint32_t rank[kScanRowsPerThread];
#pragma unroll
    for (int j = 0; j < kScanRowsPerThread; ++j) {
      const unsigned b = __ballot_sync(0xffffffffu, sel[j]);
      rank[j] = __popc(b & ((1u << lane) - 1u));
      if (lane == 0) s_cnt[j][warp] = __popc(b);
    }
    __syncthreads();
    if (warp == 0) {
      // exclusive scan of the (j, warp) counts, then look-back for the tile prefix
      constexpr int NC = kScanRowsPerThread * (kScanThreads / 32);
      static_assert(NC <= 32, "count slots must fit one warp");
      uint32_t c = lane < NC ? s_cnt[lane / (kScanThreads / 32)][lane % (kScanThreads / 32)] : 0u;
      uint32_t incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += v;
      }
      const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
      if (lane < NC) s_cnt[lane / (kScanThreads / 32)][lane % (kScanThreads / 32)] = incl - c;
      const uint64_t prefix = lookback_exclusive(tile_status, (uint32_t)tile, total, err);
      if (lane == 0) {
        s_prefix = prefix;
        if (tile == num_tiles - 1) *d_count = prefix + total;
      }
    }
    __syncthreads();
    const uint64_t base = s_prefix;
#pragma unroll
    for (int j = 0; j < kScanRowsPerThread; ++j)
      if (sel[j]) {
        const uint64_t pos = base + s_cnt[j][warp] + rank[j];
        if (pos < n) store_row<WOUT>(out, pos, O[j]);  // guards a timed-out look-back
      }
    __syncthreads();
  }
  if (n == 0 && blockIdx.x == 0 && t == 0) *d_count = 0;
}

// ------------------------------------------------------------------ aggregate kernel
// Per-thread private accumulators (SoA in shared memory) when the group table is small,
// otherwise one per-block table updated with shared-memory atomics.  Blocks fold their
// table into a global one with atomics; the last block to finish writes the non-empty
// groups in ascending key order.
template <int WIN, bool PRIVATE>
__global__ void __launch_bounds__(kScanThreads)
scan_aggregate_kernel(const __grid_constant__ ScanProgram p, const uint8_t* __restrict__ in,
                      uint64_t n, unsigned long long* __restrict__ gacc,
                      uint32_t* __restrict__ done_counter, uint64_t* __restrict__ out_keys,
                      int64_t* __restrict__ out_sums, uint64_t* __restrict__ out_counts,
                      uint64_t* __restrict__ d_groups, uint32_t* err) {
  constexpr int NIN = Limbs<WIN>::N;
  constexpr int PER = NIN + kMaxExt + kMaxRegs;
  extern __shared__ __align__(16) uint64_t smem[];
  __shared__ bool s_last;
  const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
  uint64_t* my = smem + t;
  uint64_t* in_slot = my;
  uint64_t* ext_slot = my + NIN * kScanThreads;
  uint64_t* reg_slot = my + (NIN + kMaxExt) * kScanThreads;
  const uint32_t nv = p.nsum + 1;  // sums then the count
  const uint32_t nacc = p.ngroups_total * nv;
  // accumulator area after the per-thread slots
  unsigned long long* acc = reinterpret_cast<unsigned long long*>(smem + PER * kScanThreads);
  if (PRIVATE) {
    for (uint32_t k = 0; k < nacc; ++k) acc[k * kScanThreads + t] = 0;
  } else {
    for (uint32_t k = t; k < nacc; k += kScanThreads) acc[k] = 0;
    __syncthreads();
  }
  const uint64_t stride = (uint64_t)gridDim.x * kScanThreads;
  for (uint64_t i = (uint64_t)blockIdx.x * kScanThreads + t; i < n; i += 2 * stride) {
    uint64_t L0[NIN], L1[NIN];
    const uint64_t i1 = i + stride;
    load_row<WIN>(in, i, L0);
    if (i1 < n) load_row<WIN>(in, i1, L1);
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      if (r == 1 && i1 >= n) break;
#pragma unroll
      for (int l = 0; l < NIN; ++l) in_slot[l * kScanThreads] = r ? L1[l] : L0[l];
      if (!eval_predicate<NIN>(p, in_slot)) continue;
      eval_arith<NIN>(p, in_slot, ext_slot, reg_slot);
      uint32_t g = 0;
      bool ok = true;
      for (uint32_t k = 0; k < p.ngroup; ++k) {
        const uint64_t v = vfield<NIN>(p, in_slot, ext_slot, p.group_src[k]);
        ok = ok && v < p.group_domain[k];
        g += (uint32_t)v * p.group_stride[k];
      }
      if (!ok) {
        raise_error(err, kErrCapacity);
        continue;
      }
      const uint32_t b = g * nv;
      if (PRIVATE) {
        for (uint32_t j = 0; j < p.nsum; ++j) acc[(b + j) * kScanThreads + t] += vfield<NIN>(p, in_slot, ext_slot, p.sum_src[j]);
        acc[(b + p.nsum) * kScanThreads + t] += 1ull;
      } else {
        for (uint32_t j = 0; j < p.nsum; ++j) atomicAdd(&acc[b + j], (unsigned long long)vfield<NIN>(p, in_slot, ext_slot, p.sum_src[j]));
        atomicAdd(&acc[b + p.nsum], 1ull);
      }
    }
  }
  __syncthreads();
  // fold this block into the global table
  if (PRIVATE) {
    for (uint32_t k = warp; k < nacc; k += kScanThreads / 32) {
      unsigned long long s = 0;
      for (uint32_t tt = lane; tt < kScanThreads; tt += 32) s += acc[k * kScanThreads + tt];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0 && s) atomicAdd(&gacc[k], s);
    }
  } else {
    for (uint32_t k = t; k < nacc; k += kScanThreads)
      if (acc[k]) atomicAdd(&gacc[k], acc[k]);
  }
  __threadfence();
  __syncthreads();
  if (t == 0) s_last = atomicAdd(done_counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // last block: compact the non-empty groups in group-index (= packed key) order
  if (warp == 0) {
    uint64_t written = 0;
    for (uint32_t g0 = 0; g0 < p.ngroups_total; g0 += 32) {
      const uint32_t g = g0 + lane;
      unsigned long long cnt = 0;
      if (g < p.ngroups_total) cnt = atomicAdd(&gacc[g * nv + p.nsum], 0ull);
      const unsigned m = __ballot_sync(0xffffffffu, cnt != 0);
      if (cnt) {
        const uint64_t pos = written + __popc(m & ((1u << lane) - 1u));
        uint64_t key = 0;
        uint32_t rem = g;
        for (uint32_t k = 0; k < p.ngroup; ++k) {
          const uint32_t v = rem / p.group_stride[k];
          rem -= v * p.group_stride[k];
          key = (p.group_bits[k] >= 64 ? 0ull : key << p.group_bits[k]) | v;
        }
        out_keys[pos] = key;
        out_counts[pos] = cnt;
        for (uint32_t j = 0; j < p.nsum; ++j) out_sums[pos * p.nsum + j] = (int64_t)atomicAdd(&gacc[g * nv + j], 0ull);
      }
      written += __popc(m);
    }
    if (lane == 0) *d_groups = written;
  }
}

}  // namespace rfx
