// scan_jit.cpp -- generates plan-specialised CUDA source for the scan kernels
// (select / arith / project with compaction, and the fused filter-aggregate) from a
// compiled ScanProgram.  The generated code computes exactly what the interpreting
// kernels of scan_kernels.cuh compute -- same integer semantics, same row order, same
// accumulation -- with every descriptor choice turned into a constant: fields are cut
// from fixed limb positions of the row held in registers and each expression
// instruction becomes one C statement.
#include <cstdio>
#include <sstream>
#include <string>

#include "host_common.h"
#include "jit.h"
#include "scan_program.h"

namespace rfx {

namespace {

// Device helpers shared by all generated kernels (no headers are available to NVRTC).
const char* kPreamble = R"RFX(
typedef unsigned long long u64;
typedef long long i64;
typedef unsigned int u32;
typedef int i32;
typedef unsigned short u16;
typedef unsigned char u8;
struct __align__(16) U2 { u64 x, y; };
// comparison constants, a kernel parameter: plans that differ only in their constants
// share one compiled kernel
struct RfxConsts { u64 c[16]; };

static __device__ __forceinline__ u64 s32(u64 v) { return (u64)(i64)(i32)(u32)v; }
static __device__ __forceinline__ u64 u32v(u64 v) { return (u64)(u32)v; }
static __device__ __forceinline__ u64 divmod_s32(u64 a, u64 b, bool mod) {
  const i32 x = (i32)(u32)a, y = (i32)(u32)b;
  i32 r;
  if (y == 0) r = 0;
  else if (x == (i32)0x80000000u && y == -1) r = mod ? 0 : x;
  else r = mod ? x % y : x / y;
  return (u64)(i64)r;
}
static __device__ __forceinline__ u64 divmod_u32(u64 a, u64 b, bool mod) {
  const u32 x = (u32)a, y = (u32)b;
  return y == 0 ? 0ull : (u64)(mod ? x % y : x / y);
}
static __device__ __forceinline__ u64 divmod_s64(u64 a, u64 b, bool mod) {
  const i64 x = (i64)a, y = (i64)b;
  i64 r;
  if (y == 0) r = 0;
  else if (x == (i64)0x8000000000000000ull && y == -1) r = mod ? 0 : x;
  else r = mod ? x % y : x / y;
  return (u64)r;
}
static __device__ __forceinline__ u64 divmod_u64(u64 a, u64 b, bool mod) {
  return b == 0 ? 0ull : (mod ? a % b : a / b);
}
static __device__ __forceinline__ void raise_error(u32* err, u32 code) {
  if (err) atomicCAS(err, 0u, code);
}
static __device__ __forceinline__ u64 ld_relaxed_u64(const u64* p) {
  u64 v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
static __device__ __forceinline__ void st_relaxed_u64(u64* p, u64 v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
#define FLAG_AGG (1ull << 62)
#define FLAG_INC (2ull << 62)
#define VAL_MASK ((1ull << 62) - 1)
#define SPIN_LIMIT (1u << 22)
// warp 0 of a tile: publish the aggregate, return the exclusive prefix (bounded waits)
static __device__ __forceinline__ void lb_publish(u64* status, u32 tile, u64 agg) {
  st_relaxed_u64(&status[tile], (tile == 0 ? FLAG_INC : FLAG_AGG) | (agg & VAL_MASK));
}
// Look-back of a tile whose aggregate was published earlier (lb_publish); whole warp.
static __device__ __forceinline__ u64 lookback_resolve(u64* status, u32 tile, u64 agg, u32* err) {
  const u32 lane = threadIdx.x & 31;
  if (tile == 0) return 0;
  u64 prefix = 0;
  long long base = (long long)tile - 1;
  u32 spins = 0;
  while (true) {
    const long long idx = base - (long long)lane;
    const u64 s = idx >= 0 ? ld_relaxed_u64(&status[idx]) : FLAG_INC;
    const u64 flag = s & ~VAL_MASK;
    const unsigned not_ready = __ballot_sync(0xffffffffu, flag == 0);
    const unsigned inc = __ballot_sync(0xffffffffu, flag == FLAG_INC);
    const unsigned upto = inc ? ((inc & (0u - inc)) << 1) - 1 : 0xffffffffu;
    if (not_ready & upto) {
      if (++spins > SPIN_LIMIT) { raise_error(err, 4u); break; }
      __nanosleep(spins < 64 ? 20 : 200);
      continue;
    }
    u64 v = ((upto >> lane) & 1u) ? (s & VAL_MASK) : 0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    prefix += v;
    if (inc) break;
    base -= 32;
  }
  if (lane == 0) st_relaxed_u64(&status[tile], FLAG_INC | ((prefix + agg) & VAL_MASK));
  return prefix;
}
static __device__ __forceinline__ u64 lookback(u64* status, u32 tile, u64 agg, u32* err) {
  const u32 lane = threadIdx.x & 31;
  if (tile == 0) {
    if (lane == 0) st_relaxed_u64(&status[0], FLAG_INC | (agg & VAL_MASK));
    return 0;
  }
  if (lane == 0) st_relaxed_u64(&status[tile], FLAG_AGG | (agg & VAL_MASK));
  u64 prefix = 0;
  long long base = (long long)tile - 1;
  u32 spins = 0;
  while (true) {
    const long long idx = base - (long long)lane;
    const u64 s = idx >= 0 ? ld_relaxed_u64(&status[idx]) : FLAG_INC;
    const u64 flag = s & ~VAL_MASK;
    const unsigned not_ready = __ballot_sync(0xffffffffu, flag == 0);
    const unsigned inc = __ballot_sync(0xffffffffu, flag == FLAG_INC);
    const unsigned upto = inc ? ((inc & (0u - inc)) << 1) - 1 : 0xffffffffu;
    if (not_ready & upto) {
      if (++spins > SPIN_LIMIT) { raise_error(err, 4u); break; }
      __nanosleep(spins < 64 ? 20 : 200);
      continue;
    }
    u64 v = ((upto >> lane) & 1u) ? (s & VAL_MASK) : 0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    prefix += v;
    if (inc) break;
    base -= 32;
  }
  if (lane == 0) st_relaxed_u64(&status[tile], FLAG_INC | ((prefix + agg) & VAL_MASK));
  return prefix;
}
)RFX";

std::string hex(uint64_t v) {
  char b[32];
  std::snprintf(b, sizeof(b), "0x%llxull", (unsigned long long)v);
  return b;
}

uint64_t wmask(uint32_t w) { return w >= 64 ? ~0ull : ((1ull << w) - 1); }

int limbs(uint32_t bytes) { return bytes <= 8 ? 1 : (int)(bytes / 8); }

// Row load into u64 L[NL] / store from u64 O[NL].
std::string load_code(uint32_t W, const std::string& dst, const std::string& idx) {
  std::ostringstream s;
  switch (W) {
    case 1: s << dst << "[0] = __ldg(in + " << idx << ");"; break;
    case 2: s << dst << "[0] = __ldg((const u16*)in + " << idx << ");"; break;
    case 4: s << dst << "[0] = __ldg((const u32*)in + " << idx << ");"; break;
    case 8: s << dst << "[0] = __ldg((const u64*)in + " << idx << ");"; break;
    default: {
      s << "{ const U2* p_ = (const U2*)(in + (" << idx << ") * " << W << "ull);";
      for (uint32_t k = 0; k < W / 16; ++k)
        s << " { U2 v_ = p_[" << k << "]; " << dst << "[" << 2 * k << "] = v_.x; " << dst << "[" << 2 * k + 1
          << "] = v_.y; }";
      s << " }";
    }
  }
  return s.str();
}

std::string store_code(uint32_t W, const std::string& src, const std::string& idx) {
  std::ostringstream s;
  switch (W) {
    case 1: s << "out[" << idx << "] = (u8)" << src << "[0];"; break;
    case 2: s << "((u16*)out)[" << idx << "] = (u16)" << src << "[0];"; break;
    case 4: s << "((u32*)out)[" << idx << "] = (u32)" << src << "[0];"; break;
    case 8: s << "((u64*)out)[" << idx << "] = " << src << "[0];"; break;
    default: {
      s << "{ U2* p_ = (U2*)(out + (" << idx << ") * " << W << "ull);";
      for (uint32_t k = 0; k < W / 16; ++k)
        s << " { U2 v_; v_.x = " << src << "[" << 2 * k << "]; v_.y = " << src << "[" << 2 * k + 1 << "]; p_[" << k
          << "] = v_; }";
      s << " }";
    }
  }
  return s.str();
}

std::string field_expr(const FieldLoc& f, int nl, const std::string& L) {
  std::ostringstream s;
  if (f.width == 0) return "0ull";
  if (f.off == 0) {
    s << "(" << L << "[" << (int)f.limb << "] & " << hex(wmask(f.width)) << ")";
  } else if ((uint32_t)f.off + f.width <= 64 || f.limb + 1 >= nl) {
    s << "((" << L << "[" << (int)f.limb << "] >> " << (int)f.off << ") & " << hex(wmask(f.width)) << ")";
  } else {
    s << "(((" << L << "[" << (int)f.limb << "] >> " << (int)f.off << ") | (" << L << "[" << (int)f.limb + 1 << "] << "
      << 64 - f.off << ")) & " << hex(wmask(f.width)) << ")";
  }
  return s.str();
}

// Virtual field v as an expression (input field or appended field E<j>).
std::string vfield(const ScanProgram& p, uint32_t v) {
  if (v < p.nfields) return "F" + std::to_string(v);
  return "E" + std::to_string(v - p.nfields);
}

// Per-row body: defines F<i>, `keep`, and (inside `if (keep)`) the E<j> values.
std::string row_body(const ScanProgram& p, const std::string& L) {
  std::ostringstream s;
  const int nl = limbs(p.in_bytes);
  for (uint32_t i = 0; i < p.nfields; ++i) s << "const u64 F" << i << " = " << field_expr(p.in_loc[i], nl, L) << ";\n";
  s << "bool keep = true;\n";
  static const char* ops[] = {"", "==", "!=", "<", "<", "<=", "<=", ">", ">", ">=", ">="};
  for (uint32_t c = 0; c < p.ncmp; ++c) {
    const CmpDesc& d = p.cmps[c];
    std::string a = d.a_var ? "F" + std::to_string(d.a_field) : "K.c[" + std::to_string(2 * c) + "]";
    std::string b = d.b_var ? "F" + std::to_string(d.b_field) : "K.c[" + std::to_string(2 * c + 1) + "]";
    s << "keep = keep && (((" << a << ") & " << hex(d.tmask) << ") " << ops[d.op] << " ((" << b << ") & "
      << hex(d.tmask) << "));\n";
  }
  for (uint32_t j = 0; j < p.narith; ++j) s << "u64 E" << j << " = 0;\n";
  if (p.ninstr) {
    s << "if (keep) {\n";
    for (int r = 0; r < kMaxRegs; ++r) s << "u64 R" << r << " = 0;\n";
    for (uint32_t k = 0; k < p.ninstr; ++k) {
      const Instr& in = p.code[k];
      const std::string d = "R" + std::to_string(in.dst), a = "R" + std::to_string(in.a), b = "R" + std::to_string(in.b);
      switch (in.op) {
        case OP_FIELD: s << d << " = " << vfield(p, in.field) << " & " << hex(in.imm) << ";\n"; break;
        case OP_CONST: s << d << " = " << hex(in.imm) << ";\n"; break;
        case OP_ADD64: s << d << " = " << a << " + " << b << ";\n"; break;
        case OP_SUB64: s << d << " = " << a << " - " << b << ";\n"; break;
        case OP_MUL64: s << d << " = " << a << " * " << b << ";\n"; break;
        case OP_ADD_S32: s << d << " = s32(" << a << " + " << b << ");\n"; break;
        case OP_SUB_S32: s << d << " = s32(" << a << " - " << b << ");\n"; break;
        case OP_MUL_S32: s << d << " = s32(" << a << " * " << b << ");\n"; break;
        case OP_ADD_U32: s << d << " = u32v(" << a << " + " << b << ");\n"; break;
        case OP_SUB_U32: s << d << " = u32v(" << a << " - " << b << ");\n"; break;
        case OP_MUL_U32: s << d << " = u32v(" << a << " * " << b << ");\n"; break;
        case OP_DIV_S32: s << d << " = divmod_s32(" << a << ", " << b << ", false);\n"; break;
        case OP_MOD_S32: s << d << " = divmod_s32(" << a << ", " << b << ", true);\n"; break;
        case OP_DIV_U32: s << d << " = divmod_u32(" << a << ", " << b << ", false);\n"; break;
        case OP_MOD_U32: s << d << " = divmod_u32(" << a << ", " << b << ", true);\n"; break;
        case OP_DIV_S64: s << d << " = divmod_s64(" << a << ", " << b << ", false);\n"; break;
        case OP_MOD_S64: s << d << " = divmod_s64(" << a << ", " << b << ", true);\n"; break;
        case OP_DIV_U64: s << d << " = divmod_u64(" << a << ", " << b << ", false);\n"; break;
        case OP_MOD_U64: s << d << " = divmod_u64(" << a << ", " << b << ", true);\n"; break;
        case OP_STORE_EXT: s << "E" << in.field << " = " << a << " & " << hex(in.imm) << ";\n"; break;
        default: break;
      }
    }
    s << "}\n";
  }
  return s.str();
}

constexpr int kJitThreads = 256;

std::string gen_aggregate(const ScanProgram& p, bool priv, int rows) {
  const int nl = limbs(p.in_bytes);
  const uint32_t nv = p.nsum + 1;
  std::ostringstream s;
  s << kPreamble;
  s << "#define NT " << kJitThreads << "\n#define NL " << nl << "\n#define G " << p.ngroups_total << "\n#define NV " << nv
    << "\n#define NS " << p.nsum << "\n#define NACC (G * NV)\n";
  s << "static __device__ __forceinline__ void process(const u64 (&L)[NL], u64* acc, u32 t, u32* err, "
       "const RfxConsts& K) {\n";
  s << row_body(p, "L");
  s << "if (!keep) return;\n";
  s << "u32 g = 0;\nbool ok = true;\n";
  for (uint32_t k = 0; k < p.ngroup; ++k) {
    s << "{ const u64 gv = " << vfield(p, p.group_src[k]) << "; ok = ok && gv < " << p.group_domain[k] << "ull; g += (u32)gv * "
      << p.group_stride[k] << "u; }\n";
  }
  s << "if (!ok) { raise_error(err, 3u); return; }\n";
  s << "const u32 b = g * NV;\n";
  for (uint32_t j = 0; j < p.nsum; ++j) {
    if (priv)
      s << "acc[(b + " << j << ") * NT + t] += " << vfield(p, p.sum_src[j]) << ";\n";
    else
      s << "atomicAdd((unsigned long long*)&acc[b + " << j << "], (unsigned long long)" << vfield(p, p.sum_src[j]) << ");\n";
  }
  if (priv) s << "acc[(b + NS) * NT + t] += 1ull;\n";
  else s << "atomicAdd((unsigned long long*)&acc[b + NS], 1ull);\n";
  s << "}\n";
  s << R"RFX(
extern "C" __global__ void __launch_bounds__(NT) rfx_plan_aggregate(
    const u8* __restrict__ in, u64 n, unsigned long long* __restrict__ gacc, u32* __restrict__ done,
    u64* __restrict__ out_keys, i64* __restrict__ out_sums, u64* __restrict__ out_counts,
    u64* __restrict__ d_groups, u32* err, const RfxConsts K) {
  extern __shared__ __align__(16) u64 acc[];
  __shared__ bool s_last;
  const u32 t = threadIdx.x, lane = t & 31, warp = t >> 5;
)RFX";
  if (priv)
    s << "  for (u32 k = 0; k < NACC; ++k) acc[k * NT + t] = 0;\n";
  else
    s << "  for (u32 k = t; k < NACC; k += NT) acc[k] = 0;\n  __syncthreads();\n";
  // `rows` rows per thread per iteration, all loads issued before any is used
  s << "  const u64 stride = (u64)gridDim.x * NT;\n";
  s << "  for (u64 i = (u64)blockIdx.x * NT + t; i < n; i += " << rows << " * stride) {\n";
  s << "    u64 L[" << rows << "][NL];\n";
  for (int r = 0; r < rows; ++r)
    s << "    { const u64 ii = i + " << r << " * stride; if (ii < n) { "
      << load_code(p.in_bytes, "L[" + std::to_string(r) + "]", "ii") << " } }\n";
  for (int r = 0; r < rows; ++r) s << "    if (i + " << r << " * stride < n) process(L[" << r << "], acc, t, err, K);\n";
  s << "  }\n  __syncthreads();\n";
  if (priv)
    s << R"RFX(
  for (u32 k = warp; k < NACC; k += NT / 32) {
    unsigned long long v = 0;
    for (u32 tt = lane; tt < NT; tt += 32) v += acc[k * NT + tt];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0 && v) atomicAdd(&gacc[k], v);
  }
)RFX";
  else
    s << "  for (u32 k = t; k < NACC; k += NT) if (acc[k]) atomicAdd(&gacc[k], (unsigned long long)acc[k]);\n";
  s << R"RFX(
  __threadfence();
  __syncthreads();
  if (t == 0) s_last = atomicAdd(done, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (warp == 0) {
    u64 written = 0;
    for (u32 g0 = 0; g0 < G; g0 += 32) {
      const u32 g = g0 + lane;
      unsigned long long cnt = 0;
      if (g < G) cnt = atomicAdd(&gacc[g * NV + NS], 0ull);
      const unsigned m = __ballot_sync(0xffffffffu, cnt != 0);
      if (cnt) {
        const u64 pos = written + __popc(m & ((1u << lane) - 1u));
        u64 key = 0;
        u32 rem = g;
)RFX";
  for (uint32_t k = 0; k < p.ngroup; ++k) {
    s << "        { const u32 v = rem / " << p.group_stride[k] << "u; rem -= v * " << p.group_stride[k] << "u; key = "
      << (p.group_bits[k] >= 64 ? "(u64)v" : "(key << " + std::to_string(p.group_bits[k]) + ") | v") << "; }\n";
  }
  s << R"RFX(
        out_keys[pos] = key;
        out_counts[pos] = cnt;
        for (u32 j = 0; j < NS; ++j) out_sums[pos * NS + j] = (i64)atomicAdd(&gacc[g * NV + j], 0ull);
      }
      written += __popc(m);
    }
    if (lane == 0) *d_groups = written;
  }
}
)RFX";
  return s.str();
}

// Compaction / map kernel.  mode 0: select (row unchanged), 1: select + project,
// 2: map (no predicate, no compaction).
std::string gen_compact(const ScanProgram& p, int mode, uint32_t wout, int rows_per_thread) {
  const int nl = limbs(p.in_bytes);
  const int no = limbs(wout);
  std::ostringstream s;
  s << kPreamble;
  s << "#define NT " << kJitThreads << "\n#define NL " << nl << "\n#define NO " << no << "\n#define IPT "
    << rows_per_thread << "\n#define TILE (NT * IPT)\n";
  s << "static __device__ __forceinline__ bool process(const u64 (&L)[NL], u64 (&O)[NO], const RfxConsts& K) {\n";
  s << row_body(p, "L");
  if (mode == 0) {
    s << "for (int l = 0; l < NO; ++l) O[l] = L[l];\n";
  } else {
    s << "if (keep) {\n";
    s << "for (int l = 0; l < NO; ++l) O[l] = 0;\n";
    for (uint32_t k = 0; k < p.nout; ++k) {
      const FieldLoc f = p.out_loc[k];
      if (p.out_src[k] == 0xff || f.width == 0) continue;
      const std::string v = "(" + vfield(p, p.out_src[k]) + " & " + hex(wmask(f.width)) + ")";
      s << "O[" << (int)f.limb << "] |= " << v << " << " << (int)f.off << ";\n";
      if (f.off && (uint32_t)f.off + f.width > 64 && f.limb + 1 < no)
        s << "O[" << (int)f.limb + 1 << "] |= " << v << " >> " << 64 - f.off << ";\n";
    }
    s << "}\n";
  }
  s << "return keep;\n}\n";
  if (mode == 2) {
    s << R"RFX(
extern "C" __global__ void __launch_bounds__(NT) rfx_plan_compact(
    const u8* __restrict__ in, u64 n, u8* __restrict__ out, u64* __restrict__ d_count,
    u64* __restrict__ status, u32* __restrict__ tile_counter, u32* err, const RfxConsts K) {
  const u32 t = threadIdx.x;
  const u64 num_tiles = (n + TILE - 1) / TILE;
  for (u64 tile = blockIdx.x; tile < num_tiles; tile += gridDim.x) {
    u64 L[IPT][NL];
    u64 O[IPT][NO];
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
      const u64 i = tile * TILE + (u64)j * NT + t;
      if (i < n) { )RFX" << load_code(p.in_bytes, "L[j]", "i") << R"RFX( }
    }
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
      const u64 i = tile * TILE + (u64)j * NT + t;
      if (i < n) { process(L[j], O[j], K); )RFX" << store_code(wout, "O[j]", "i") << R"RFX( }
    }
  }
}
)RFX";
    return s.str();
  }
  // Compaction, one tile ahead, with a look-back warp: the eight compute warps claim,
  // load and evaluate tile k+1, stage its kept rows (compacted, limb-major) in shared
  // memory and publish its count, while the ninth warp resolves tile k's offset by
  // look-back; then all warps write tile k's staged rows out as one contiguous run.  No
  // look-back stands between a claim and that tile's count, a tile is resolved a whole
  // step after its count was published, and the look-back's L2 round trips overlap the
  // next tile's loads.
  s << R"RFX(
#define NTB (NT + 32)
extern "C" __global__ void __launch_bounds__(NTB) rfx_plan_compact(
    const u8* __restrict__ in, u64 n, u8* __restrict__ out, u64* __restrict__ d_count,
    u64* __restrict__ status, u32* __restrict__ tile_counter, u32* err, const RfxConsts K) {
  extern __shared__ __align__(16) u64 sstage[];      // [2][NO][TILE]
  __shared__ u32 s_cnt[2][IPT][NT / 32];
  __shared__ u32 s_total[2];
  __shared__ u32 s_tile[2];
  __shared__ u64 s_prefix;
  const u32 t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const u64 num_tiles = (n + TILE - 1) / TILE;
  // compute warps only (barrier 1 over NT threads): claim, load, evaluate, rank and
  // stage one tile into buffer b; publish its count
  auto fill = [&](int b) {
    if (t == 0) s_tile[b] = atomicAdd(tile_counter, 1u);
    asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory");
    const u64 tile = s_tile[b];
    if (tile >= num_tiles) return;
    u64 L[IPT][NL];
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
      const u64 i = tile * TILE + (u64)j * NT + t;
      if (i < n) { )RFX" << load_code(p.in_bytes, "L[j]", "i") << R"RFX( }
    }
    u64 O[IPT][NO];
    bool sel[IPT];
    u32 rank[IPT];
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
      const u64 i = tile * TILE + (u64)j * NT + t;
      sel[j] = i < n ? process(L[j], O[j], K) : false;
      const unsigned bal = __ballot_sync(0xffffffffu, sel[j]);
      rank[j] = __popc(bal & ((1u << lane) - 1u));
      if (lane == 0) s_cnt[b][j][warp] = __popc(bal);
    }
    asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory");
    if (warp == 0) {
      // exclusive scan of the IPT x warps counts, 32 at a time
      const u32 NC = IPT * (NT / 32);
      u32 total = 0;
      for (u32 c0 = 0; c0 < NC; c0 += 32) {
        const u32 idx = c0 + lane;
        const u32 c = idx < NC ? s_cnt[b][idx / (NT / 32)][idx % (NT / 32)] : 0u;
        u32 incl = c;
        for (int o = 1; o < 32; o <<= 1) {
          const u32 v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= (u32)o) incl += v;
        }
        if (idx < NC) s_cnt[b][idx / (NT / 32)][idx % (NT / 32)] = total + incl - c;
        total += __shfl_sync(0xffffffffu, incl, 31);
      }
      if (lane == 0) {
        s_total[b] = total;
        lb_publish(status, (u32)tile, total);
      }
    }
    asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory");
    u64* st = sstage + (size_t)b * NO * TILE;
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
      if (sel[j]) {
        const u32 r = s_cnt[b][j][warp] + rank[j];
#pragma unroll
        for (int l = 0; l < NO; ++l) st[(size_t)l * TILE + r] = O[j][l];
      }
    }
  };
  if (t < NT) fill(0);
  __syncthreads();
  u64 tc = s_tile[0];
  for (int b = 0; tc < num_tiles; b ^= 1) {
    if (t < NT) {
      fill(b ^ 1);
    } else {
      const u64 prefix = lookback_resolve(status, (u32)tc, s_total[b], err);
      if (lane == 0) {
        s_prefix = prefix;
        if (tc == num_tiles - 1) *d_count = prefix + s_total[b];
      }
    }
    __syncthreads();
    const u64 base = s_prefix;
    const u32 total = s_total[b];
    const u64* st = sstage + (size_t)b * NO * TILE;
    for (u32 r = t; r < total; r += NTB) {
      const u64 pos = base + r;
      if (pos < n) {
        u64 O1[NO];
#pragma unroll
        for (int l = 0; l < NO; ++l) O1[l] = st[(size_t)l * TILE + r];
        )RFX" << store_code(wout, "O1", "pos") << R"RFX(
      }
    }
    tc = s_tile[b ^ 1];
    __syncthreads();
  }
}
)RFX";
  return s.str();
}

struct HostConsts {
  uint64_t c[16];
};
static_assert(kMaxCmp * 2 <= 16, "constant slots");

HostConsts consts_of(const ScanProgram& p) {
  HostConsts k;
  for (auto& v : k.c) v = 0;
  for (uint32_t c = 0; c < p.ncmp; ++c) {
    k.c[2 * c] = p.cmps[c].a_const;
    k.c[2 * c + 1] = p.cmps[c].b_const;
  }
  return k;
}

// The source of a plan with its comparison constants cleared: the compile cache key.
ScanProgram without_consts(const ScanProgram& p) {
  ScanProgram q = p;
  for (uint32_t c = 0; c < q.ncmp; ++c) q.cmps[c].a_const = q.cmps[c].b_const = 0;
  return q;
}

}  // namespace

// Launches the specialised aggregate kernel; RFX_ERR_UNSUPPORTED when it cannot be
// compiled (the caller falls back to the interpreting kernel).
rfx_status jit_aggregate(const ScanProgram& p, const void* in, uint64_t n, unsigned long long* gacc, uint32_t* done,
                         uint64_t* out_keys, int64_t* out_sums, uint64_t* out_counts, uint64_t* d_groups, uint32_t* err,
                         cudaStream_t stream, int variant) {
  const uint32_t nacc = p.ngroups_total * (p.nsum + 1);
  const bool priv = nacc <= 24;
  // rows per thread per iteration by row width (64-byte rows: 3 keeps 0.57 ms per 60M
  // rows against 0.69 with 2), one more for variant 1, one fewer for variant 2
  int rows = p.in_bytes >= 64 ? 3 : p.in_bytes >= 32 ? 4 : p.in_bytes >= 16 ? 6 : 8;
  if (variant == 1) rows += 1;
  if (variant == 2 && rows > 1) rows -= 1;
  cudaKernel_t k;
  rfx_status st = jit_kernel(gen_aggregate(without_consts(p), priv, rows), "rfx_plan_aggregate", &k);
  if (st != RFX_OK) return st;
  const size_t smem = (priv ? (size_t)nacc * kJitThreads : (size_t)nacc) * sizeof(uint64_t);
  RFX_CUDA_TRY(allow_smem((const void*)k, smem));
  const uint64_t blocks = (n + (uint64_t)rows * kJitThreads - 1) / ((uint64_t)rows * kJitThreads);
  const int grid = persistent_grid((const void*)k, kJitThreads, smem, blocks ? blocks : 1);
  HostConsts kc = consts_of(p);
  void* args[] = {(void*)&in, (void*)&n, (void*)&gacc, (void*)&done, (void*)&out_keys, (void*)&out_sums,
                  (void*)&out_counts, (void*)&d_groups, (void*)&err, (void*)&kc};
  RFX_CUDA_TRY(cudaLaunchKernel((const void*)k, dim3(grid), dim3(kJitThreads), args, smem, stream));
  return RFX_OK;
}

rfx_status jit_compact(const ScanProgram& p, int mode, const void* in, uint64_t n, void* out, uint64_t* d_count,
                       uint64_t* status, uint32_t* counter, uint32_t* err, cudaStream_t stream, uint64_t tile_rows,
                       int variant) {
  const uint32_t wout = mode == 0 ? p.in_bytes : p.out_bytes;
  // rows per thread by row width (registers hold one tile's rows), doubled by variant 1
  // and halved by variant 2; tiles are never smaller than the workspace's tile_rows, so
  // its status array suffices
  const uint32_t wmax = p.in_bytes > wout ? p.in_bytes : wout;
  int ipt = wmax >= 32 ? 2 : wmax >= 16 ? 4 : 8;
  if (variant == 1 && ipt < 16) ipt *= 2;
  if (variant == 2) ipt /= 2;
  if ((uint64_t)ipt * kJitThreads < tile_rows) ipt = (int)(tile_rows / kJitThreads);
  tile_rows = (uint64_t)ipt * kJitThreads;
  cudaKernel_t k;
  rfx_status st = jit_kernel(gen_compact(without_consts(p), mode, wout, ipt), "rfx_plan_compact", &k);
  if (st != RFX_OK) return st;
  const uint64_t tiles = (n + tile_rows - 1) / tile_rows;
  const uint32_t no = (wout + 7) / 8;
  const size_t smem = mode == 2 ? 0 : 2ull * no * tile_rows * sizeof(uint64_t);
  if (smem) RFX_CUDA_TRY(allow_smem((const void*)k, smem));
  const int threads = mode == 2 ? kJitThreads : kJitThreads + 32;   // + the look-back warp
  const int grid = persistent_grid((const void*)k, threads, smem, tiles ? tiles : 1);
  HostConsts kc = consts_of(p);
  void* args[] = {(void*)&in, (void*)&n, (void*)&out, (void*)&d_count, (void*)&status, (void*)&counter, (void*)&err,
                  (void*)&kc};
  RFX_CUDA_TRY(cudaLaunchKernel((const void*)k, dim3(grid), dim3(threads), args, smem, stream));
  return RFX_OK;
}

}  // namespace rfx
