// reduce_f64_abi.cu -- reduce-by-key over double values: the reference's total_*_double
// (thrust::reduce_by_key with plus<double>), min_32_double (minimum<double>) and the
// scalar total_double / max_double / count of Reduce.cu:742-1536.
//
// Sums are exact, then rounded once (round to nearest, ties to even): every double is a
// 53-bit integer times a power of two, so a run's sum is accumulated as a two's-complement
// integer in units of 2^L over W 64-bit limbs (add with carry).  Integer addition is
// associative, so the result does not depend on how the work is split -- unlike a
// floating-point tree, whose rounding follows its shape.  The fast window is W = 3 limbs
// with L set from the largest exponent in the input (a pre-pass): exact for every value
// within 2^107 of the largest, with room for 2^30 terms.  A value below that window with
// bits that would be lost raises a flag, and a second pass with W = 34 limbs and
// L = -1074, which covers every finite double, runs -- its kernels are always enqueued and
// return at once unless the flag is set, so no host round trip is needed.  Specials
// follow IEEE addition: NaN if any NaN or both infinities, else the infinity, and an
// exact zero is -0 only when every term is -0.
//
// The minimum follows the reference's fold acc = (acc < v ? acc : v) exactly: a later
// element replaces an equal one (so -0 / +0 ties go to the later), a NaN sets the
// accumulator and the next element replaces it.  That fold is associative as a
// combination of run summaries, so the parallel result equals the sequential one bit for
// bit.
//
// Structure: units of 4096 elements, one warp per unit.  A pre-pass counts each unit's run
// heads (taking the exponent maximum for sums) and one block scans the counts into each
// unit's first run index; the main pass folds a unit in registers and warp shuffles,
// writes every run that starts and ends inside it at its final index, and leaves the
// partial before its first head and the partial from its last head for the fix-up, a
// segmented scan over units that closes the runs crossing units.
#include <cstring>

#include "host_common.h"
#include "rfx_device.cuh"

namespace rfx {
namespace {

constexpr int kFixThreads = 256;
constexpr int kNarrowLimbs = 3;   // 192 bits: every value within 2^107 of the largest
constexpr int kWideLimbs = 34;    // 2176 bits: every finite double
constexpr int kWideL = -1074;

enum : uint32_t { kSumNaN = 1, kSumPosInf = 2, kSumNegInf = 4, kSumNotNegZero = 8 };

// ------------------------------------------------------------------ exact sum
// W 64-bit limbs holding a two's-complement integer (limb 0 lowest) in units of 2^L.
// Additions are exact modulo 2^(64W); the true sum stays inside the signed range by the
// choice of L, so the result is exact and independent of the order of the additions.
template <int W>
struct SumOp {
  struct P {
    unsigned long long l[W];
    uint32_t flags;
    uint32_t pad;
  };
  __device__ __forceinline__ static P identity() {
    P p;
#pragma unroll
    for (int k = 0; k < W; ++k) p.l[k] = 0;
    p.flags = 0;
    p.pad = 0;
    return p;
  }
  // acc += a (neg: acc -= a) where a has limbs lo at q, hi at q + 1.
  __device__ __forceinline__ static void accumulate(unsigned long long* acc, int q, unsigned long long lo,
                                                    unsigned long long hi, bool neg) {
    if constexpr (W == 3) {
      const unsigned long long a0 = q == 0 ? lo : 0ull, a1 = q == 0 ? hi : lo, a2 = q == 0 ? 0ull : hi;
      if (!neg)
        asm("add.cc.u64 %0, %0, %3;\n\taddc.cc.u64 %1, %1, %4;\n\taddc.u64 %2, %2, %5;"
            : "+l"(acc[0]), "+l"(acc[1]), "+l"(acc[2])
            : "l"(a0), "l"(a1), "l"(a2));
      else
        asm("sub.cc.u64 %0, %0, %3;\n\tsubc.cc.u64 %1, %1, %4;\n\tsubc.u64 %2, %2, %5;"
            : "+l"(acc[0]), "+l"(acc[1]), "+l"(acc[2])
            : "l"(a0), "l"(a1), "l"(a2));
    } else {
      unsigned long long c = 0;
      for (int k = q; k < W; ++k) {
        const unsigned long long a = k == q ? lo : k == q + 1 ? hi : 0ull;
        if (!neg) {
          const unsigned __int128 t = (unsigned __int128)acc[k] + a + c;
          acc[k] = (unsigned long long)t;
          c = (unsigned long long)(t >> 64);
        } else {
          const unsigned __int128 t = (unsigned __int128)acc[k] - a - c;
          acc[k] = (unsigned long long)t;
          c = (unsigned long long)(t >> 64) ? 1ull : 0ull;
        }
        if (k > q && c == 0) break;
      }
    }
  }
  __device__ __forceinline__ static void add(P& p, double x, int L, uint32_t* inexact) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    const uint32_t eb = (uint32_t)(b >> 52) & 0x7ffu;
    const unsigned long long frac = b & ((1ull << 52) - 1);
    const bool neg = (b >> 63) != 0;
    if (b != 0x8000000000000000ull) p.flags |= kSumNotNegZero;
    if (eb == 0x7ffu) {
      p.flags |= frac ? kSumNaN : (neg ? kSumNegInf : kSumPosInf);
      return;
    }
    if (eb == 0 && frac == 0) return;
    unsigned long long m = eb ? (frac | (1ull << 52)) : frac;
    int s = (int)(eb ? eb : 1u) - 1075 - L;  // the mantissa's LSB in units of 2^L
    if (s < 0) {
      const int r = -s;
      if (r >= 64 ? m != 0 : (m & ((1ull << r) - 1)) != 0) atomicOr(inexact, 1u);
      m = r >= 64 ? 0 : m >> r;
      s = 0;
    }
    const int q = s >> 6, o = s & 63;
    if (q + 1 >= W) {  // above the window: only when L was not set from this input's maximum
      atomicOr(inexact, 1u);
      return;
    }
    const unsigned long long lo = m << o;
    const unsigned long long hi = o ? m >> (64 - o) : 0ull;
    accumulate(p.l, q, lo, hi, neg);
  }
  __device__ __forceinline__ static P combine(const P& a, const P& b) {
    P r;
    if constexpr (W == 3) {
      r.l[0] = a.l[0];
      r.l[1] = a.l[1];
      r.l[2] = a.l[2];
      asm("add.cc.u64 %0, %0, %3;\n\taddc.cc.u64 %1, %1, %4;\n\taddc.u64 %2, %2, %5;"
          : "+l"(r.l[0]), "+l"(r.l[1]), "+l"(r.l[2])
          : "l"(b.l[0]), "l"(b.l[1]), "l"(b.l[2]));
    } else {
      unsigned long long c = 0;
      for (int k = 0; k < W; ++k) {
        const unsigned __int128 t = (unsigned __int128)a.l[k] + b.l[k] + c;
        r.l[k] = (unsigned long long)t;
        c = (unsigned long long)(t >> 64);
      }
    }
    r.flags = a.flags | b.flags;
    r.pad = 0;
    return r;
  }
  // Bits [pos, pos + len) of the limbs (len <= 64, pos >= 0).
  __device__ static unsigned long long bits_at(const unsigned long long* l, int pos, int len) {
    if (len <= 0) return 0;
    const int k = pos >> 6, o = pos & 63;
    const unsigned long long d0 = k < W ? l[k] : 0ull, d1 = k + 1 < W ? l[k + 1] : 0ull;
    unsigned long long v = (d0 >> o) | (o ? d1 << (64 - o) : 0ull);
    if (len < 64) v &= (1ull << len) - 1;
    return v;
  }
  __device__ static bool any_below(const unsigned long long* l, int pos) {
    const int k = pos >> 6;
    for (int i = 0; i < k && i < W; ++i)
      if (l[i]) return true;
    if (k < W && (pos & 63) && (l[k] & ((1ull << (pos & 63)) - 1))) return true;
    return false;
  }
  // The correctly rounded double of the accumulated value, as bits.
  __device__ static unsigned long long finalize(const P& p, int L) {
    if ((p.flags & kSumNaN) || ((p.flags & kSumPosInf) && (p.flags & kSumNegInf))) return 0x7ff8000000000000ull;
    if (p.flags & kSumPosInf) return 0x7ff0000000000000ull;
    if (p.flags & kSumNegInf) return 0xfff0000000000000ull;
    unsigned long long r[W];
#pragma unroll
    for (int k = 0; k < W; ++k) r[k] = p.l[k];
    const bool neg = (r[W - 1] >> 63) != 0;
    if (neg) {  // magnitude = two's complement negation
      unsigned long long c = 1;
#pragma unroll
      for (int k = 0; k < W; ++k) {
        const unsigned long long t = ~r[k] + c;
        c = (c && t == 0) ? 1ull : 0ull;
        r[k] = t;
      }
    }
    int top = -1;
    for (int k = W - 1; k >= 0; --k)
      if (r[k]) {
        top = 64 * k + 63 - __clzll(r[k]);
        break;
      }
    if (top < 0) return (p.flags & kSumNotNegZero) ? 0ull : 0x8000000000000000ull;
    const unsigned long long sgn = neg ? 0x8000000000000000ull : 0ull;
    int e = top + L;  // the value lies in [2^e, 2^(e+1))
    if (e > 1023) return sgn | 0x7ff0000000000000ull;
    const bool normal = e >= -1022;
    const int lsb = normal ? top - 52 : -1074 - L;  // bit that becomes the result's LSB
    unsigned long long mant;
    if (lsb <= 0) {
      mant = bits_at(r, 0, top + 1) << (-lsb);
    } else {
      mant = bits_at(r, lsb, top - lsb + 1);
      const bool round = (bits_at(r, lsb - 1, 1) & 1ull) != 0;
      const bool sticky = any_below(r, lsb - 1);
      if (round && (sticky || (mant & 1ull))) ++mant;
    }
    if (normal) {
      if (mant == (1ull << 53)) {
        mant >>= 1;
        if (++e > 1023) return sgn | 0x7ff0000000000000ull;
      }
      return sgn | ((unsigned long long)(e + 1023) << 52) | (mant & ((1ull << 52) - 1));
    }
    return sgn | mant;  // subnormal; 2^52 after rounding is the smallest normal
  }
};

// ------------------------------------------------------------------ minimum (the fold)
struct MinOp {
  struct P {
    unsigned long long v;  // bits of the fold value (a NaN while pending)
    uint32_t any;          // an element after the last NaN was folded
    uint32_t nan;          // a NaN occurs in the summarised range
  };
  __device__ __forceinline__ static P identity() { return P{0ull, 0u, 0u}; }
  __device__ __forceinline__ static void add(P& p, double x, int, uint32_t*) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    if (x != x) {
      p = P{b, 0u, 1u};
    } else if (!p.any) {
      p.v = b;
      p.any = 1u;
    } else {
      const double a = __longlong_as_double((long long)p.v);
      p.v = a < x ? p.v : b;
    }
  }
  // a is the earlier range, b the later one.
  __device__ __forceinline__ static P combine(const P& a, const P& b) {
    if (b.nan) return b;
    if (!b.any) return a;
    if (!a.any) return P{b.v, 1u, a.nan};
    const double x = __longlong_as_double((long long)a.v), y = __longlong_as_double((long long)b.v);
    return P{x < y ? a.v : b.v, 1u, a.nan};
  }
  __device__ static unsigned long long finalize(const P& p, int) { return p.v; }
};

// ------------------------------------------------------------------ keys
struct Key {
  unsigned long long lo, hi;
};

template <int KB>
__device__ __forceinline__ Key load_key(const uint8_t* keys, uint64_t i) {
  if constexpr (KB == 0) return Key{0ull, 0ull};
  if constexpr (KB == 1) return Key{keys[i], 0ull};
  if constexpr (KB == 2) return Key{reinterpret_cast<const uint16_t*>(keys)[i], 0ull};
  if constexpr (KB == 4) return Key{reinterpret_cast<const uint32_t*>(keys)[i], 0ull};
  if constexpr (KB == 8) return Key{reinterpret_cast<const unsigned long long*>(keys)[i], 0ull};
  if constexpr (KB == 16) {
    const ulonglong2 v = reinterpret_cast<const ulonglong2*>(keys)[i];
    return Key{v.x, v.y};
  }
  return Key{0ull, 0ull};
}

template <int KB>
__device__ __forceinline__ void store_key(uint8_t* out, uint64_t r, const Key& k) {
  if constexpr (KB == 1) out[r] = (uint8_t)k.lo;
  if constexpr (KB == 2) reinterpret_cast<uint16_t*>(out)[r] = (uint16_t)k.lo;
  if constexpr (KB == 4) reinterpret_cast<uint32_t*>(out)[r] = (uint32_t)k.lo;
  if constexpr (KB == 8) reinterpret_cast<unsigned long long*>(out)[r] = k.lo;
  if constexpr (KB == 16) reinterpret_cast<ulonglong2*>(out)[r] = make_ulonglong2(k.lo, k.hi);
}

// ------------------------------------------------------------------ segmented scan
template <typename P>
struct Seg {
  P v;
  uint32_t f;  // a head (run start) lies in the summarised range
  uint32_t pad;
};

template <class Op>
__device__ __forceinline__ Seg<typename Op::P> seg_combine(const Seg<typename Op::P>& a,
                                                           const Seg<typename Op::P>& b) {
  if (b.f) return b;
  Seg<typename Op::P> r;
  r.v = Op::combine(a.v, b.v);
  r.f = a.f;
  r.pad = 0;
  return r;
}

template <typename T>
__device__ __forceinline__ T shfl_up_any(const T& x, int delta) {
  constexpr int W = (int)((sizeof(T) + 3) / 4);
  uint32_t w[W];
  memcpy(w, &x, sizeof(T));
#pragma unroll
  for (int i = 0; i < W; ++i) w[i] = __shfl_up_sync(0xffffffffu, w[i], delta);
  T r;
  memcpy(&r, w, sizeof(T));
  return r;
}

template <typename T>
__device__ __forceinline__ T shfl_any(const T& x, int src) {
  constexpr int W = (int)((sizeof(T) + 3) / 4);
  uint32_t w[W];
  memcpy(w, &x, sizeof(T));
#pragma unroll
  for (int i = 0; i < W; ++i) w[i] = __shfl_sync(0xffffffffu, w[i], src);
  T r;
  memcpy(&r, w, sizeof(T));
  return r;
}

// Exclusive segmented scan over the NT threads of a block (thread order); also returns the
// block's inclusive total.  `warp_tot` holds NT / 32 entries.
template <class Op, int NT>
__device__ Seg<typename Op::P> block_seg_scan(const Seg<typename Op::P>& x, Seg<typename Op::P>* warp_tot,
                                              Seg<typename Op::P>& total) {
  using S = Seg<typename Op::P>;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  S inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const S y = shfl_up_any(inc, o);
    if (lane >= o) inc = seg_combine<Op>(y, inc);
  }
  S exc = shfl_up_any(inc, 1);
  if (lane == 31) warp_tot[warp] = inc;
  __syncthreads();
  S pre;
  pre.v = Op::identity();
  pre.f = 0;
  pre.pad = 0;
  for (int w = 0; w < warp; ++w) pre = seg_combine<Op>(pre, warp_tot[w]);
  if (lane == 0) {
    exc = pre;
  } else {
    exc = seg_combine<Op>(pre, exc);
  }
  total = pre;
  for (int w = warp; w < NT / 32; ++w) total = seg_combine<Op>(total, warp_tot[w]);
  __syncthreads();
  return exc;
}

// ------------------------------------------------------------------ kernels
struct F64Args {
  const uint8_t* keys;
  const double* vals;
  uint64_t n;
  const unsigned long long* emit;  // if set, out key of a run = emit[head] (8 bytes)
  uint8_t* out_keys;
  double* out_vals;
  uint64_t* d_groups;
  uint64_t* status;     // look-back words, one per tile
  uint32_t* counter;    // tile counter
  uint32_t* tile_heads;
  uint32_t* tile_base;
  void* tile_first;     // Op::P per tile
  void* tile_last;
  void* exc;            // Seg<P> per tile (fix-up)
  void* chunk_agg;      // Seg<P> per fix-up chunk
  const int* d_emax;    // max biased exponent (sums with the narrow window)
  int fixed_L;          // used when d_emax is null
  uint32_t* inexact;
  const uint32_t* gate;   // if set, the kernels do nothing unless *gate != 0
  uint32_t* err;
};

__device__ __forceinline__ bool gated_off(const F64Args& a) { return a.gate && *a.gate == 0u; }

__device__ __forceinline__ int window_L(const F64Args& a) {
  if (!a.d_emax) return a.fixed_L;
  const int e = *a.d_emax;
  return (e > 1 ? e : 1) - 1182;
}

// Fix-up, step 1: per chunk of kFixThreads tiles, the exclusive segmented scan of the
// tile summaries (a tile with a head contributes its last partial, else its whole sum).
template <class Op>
__global__ void __launch_bounds__(kFixThreads) f64_fix_scan(F64Args a, uint64_t tiles) {
  if (gated_off(a)) return;
  using P = typename Op::P;
  using S = Seg<P>;
  __shared__ S s_warp[kFixThreads / 32];
  const uint64_t u = (uint64_t)blockIdx.x * kFixThreads + threadIdx.x;
  S x;
  x.pad = 0;
  if (u < tiles) {
    x.f = a.tile_heads[u] > 0;
    x.v = x.f ? reinterpret_cast<const P*>(a.tile_last)[u] : reinterpret_cast<const P*>(a.tile_first)[u];
  } else {
    x.f = 0;
    x.v = Op::identity();
  }
  S total;
  const S e = block_seg_scan<Op, kFixThreads>(x, s_warp, total);
  if (u < tiles) reinterpret_cast<S*>(a.exc)[u] = e;
  if (threadIdx.x == 0) reinterpret_cast<S*>(a.chunk_agg)[blockIdx.x] = total;
}

// Step 2: exclusive segmented scan over the chunk aggregates (one block, in order).
template <class Op>
__global__ void __launch_bounds__(kFixThreads) f64_fix_chunks(F64Args a, uint64_t chunks) {
  if (gated_off(a)) return;
  using S = Seg<typename Op::P>;
  __shared__ S s_warp[kFixThreads / 32];
  __shared__ S s_carry;
  if (threadIdx.x == 0) {
    s_carry.v = Op::identity();
    s_carry.f = 0;
    s_carry.pad = 0;
  }
  __syncthreads();
  S* agg = reinterpret_cast<S*>(a.chunk_agg);
  for (uint64_t base = 0; base < chunks; base += kFixThreads) {
    const uint64_t c = base + threadIdx.x;
    S x;
    if (c < chunks) {
      x = agg[c];
    } else {
      x.v = Op::identity();
      x.f = 0;
      x.pad = 0;
    }
    S total;
    const S e = block_seg_scan<Op, kFixThreads>(x, s_warp, total);
    const S carry = s_carry;
    __syncthreads();
    if (c < chunks) agg[c] = seg_combine<Op>(carry, e);  // now the chunk's exclusive prefix
    if (threadIdx.x == 0) s_carry = seg_combine<Op>(carry, total);
    __syncthreads();
  }
}

// Step 3: the runs that cross tile boundaries.  Tile u with a head closes the run of the
// previous head (the last head of an earlier tile); the last tile also closes the last run.
template <class Op>
__global__ void __launch_bounds__(kFixThreads) f64_fix_apply(F64Args a, uint64_t tiles) {
  if (gated_off(a)) return;
  using P = typename Op::P;
  using S = Seg<P>;
  const uint64_t u = (uint64_t)blockIdx.x * kFixThreads + threadIdx.x;
  if (u >= tiles) return;
  const int L = window_L(a);
  const S pre = reinterpret_cast<const S*>(a.chunk_agg)[blockIdx.x];
  const S x = seg_combine<Op>(pre, reinterpret_cast<const S*>(a.exc)[u]);
  const bool has_head = a.tile_heads[u] > 0;
  if (has_head && x.f) {
    const P y = Op::combine(x.v, reinterpret_cast<const P*>(a.tile_first)[u]);
    a.out_vals[a.tile_base[u] - 1] = __longlong_as_double((long long)Op::finalize(y, L));
  }
  if (u == tiles - 1) {
    S self;
    self.f = has_head;
    self.v = has_head ? reinterpret_cast<const P*>(a.tile_last)[u] : reinterpret_cast<const P*>(a.tile_first)[u];
    self.pad = 0;
    const S y = seg_combine<Op>(x, self);
    a.out_vals[a.tile_base[u] + a.tile_heads[u] - 1] = __longlong_as_double((long long)Op::finalize(y.v, L));
  }
}

// ------------------------------------------------------------------ warp units
// The default path: units of kF64UnitItems elements, one warp per unit.  A pre-pass counts
// every unit's run heads (and takes the exponent maximum for sums); one block scans the
// counts into each unit's first run index.  The main pass then needs nothing from other
// units: a warp folds its unit in 256-element steps (8 per lane) with shuffles only,
// writes every run that starts and ends inside the unit at its final index, and leaves the
// partial before the unit's first head and the partial from its last head for the fix-up
// above, which treats units as tiles.
constexpr int kF64UnitItems = 4096;
constexpr int kF64WarpIPT = 8;

template <int KB>
__global__ void __launch_bounds__(256) f64_unit_count(F64Args a, uint64_t units, int* emax) {
  if (gated_off(a)) return;
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t gw = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  int m = 1;
  for (uint64_t u = gw; u < units; u += nw) {
    const uint64_t e0 = u * kF64UnitItems, e1 = min(e0 + (uint64_t)kF64UnitItems, a.n);
    uint32_t c = 0;
    for (uint64_t e = e0 + lane; e < e1; e += 32) {
      bool h = e == 0;
      if constexpr (KB > 0) {
        if (!h) {
          const Key k = load_key<KB>(a.keys, e), pk = load_key<KB>(a.keys, e - 1);
          h = k.lo != pk.lo || k.hi != pk.hi;
        }
      }
      c += h;
      if (emax) {
        const int eb = (int)(((unsigned long long)__double_as_longlong(a.vals[e]) >> 52) & 0x7ffu);
        if (eb != 0x7ff && eb > m) m = eb;
      }
    }
    c = __reduce_add_sync(0xffffffffu, c);
    if (lane == 0) a.tile_heads[u] = c;
  }
  if (emax) {
    m = __reduce_max_sync(0xffffffffu, m);
    if (lane == 0) atomicMax(emax, m);
  }
}

// Exclusive scan of the unit head counts (one block, in order) and the number of runs.
__global__ void __launch_bounds__(1024) f64_unit_scan(F64Args a, uint64_t units) {
  if (gated_off(a)) return;
  __shared__ uint32_t s_warp[32];
  __shared__ uint64_t s_carry;
  const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if (t == 0) s_carry = 0;
  __syncthreads();
  for (uint64_t b = 0; b < units; b += 1024) {
    const uint64_t u = b + t;
    const uint32_t x = u < units ? a.tile_heads[u] : 0u;
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= (uint32_t)o) inc += y;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    uint32_t wpre = 0, tot = 0;
    for (uint32_t w = 0; w < 32; ++w) {
      if (w < warp) wpre += s_warp[w];
      tot += s_warp[w];
    }
    const uint64_t carry = s_carry;
    if (u < units) a.tile_base[u] = (uint32_t)(carry + wpre + inc - x);
    __syncthreads();
    if (t == 0) s_carry = carry + tot;
    __syncthreads();
  }
  if (t == 0) *a.d_groups = s_carry;
}

template <int KB, class Op>
__global__ void __launch_bounds__(256) f64_unit_kernel(F64Args a, uint64_t units) {
  if (gated_off(a)) return;
  using P = typename Op::P;
  using S = Seg<P>;
  constexpr int V = kF64WarpIPT;
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t gw = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const int L = window_L(a);
  for (uint64_t u = gw; u < units; u += nw) {
    const uint64_t e0 = u * kF64UnitItems, e1 = min(e0 + (uint64_t)kF64UnitItems, a.n);
    const uint64_t ubase = a.tile_base[u];
    S carry;
    carry.v = Op::identity();
    carry.f = 0;
    carry.pad = 0;
    uint64_t heads_so_far = 0;
    for (uint64_t tb = e0; tb < e1; tb += 32 * V) {
      const uint64_t first = tb + (uint64_t)lane * V;
      Key keys[V];
      double vals[V];
      uint32_t hm = 0;
#pragma unroll
      for (int j = 0; j < V; ++j) {
        keys[j] = Key{0ull, 0ull};
        vals[j] = 0.0;
        if (first + j < e1) {
          keys[j] = load_key<KB>(a.keys, first + j);
          vals[j] = a.vals[first + j];
        }
      }
      Key pk;
      pk.lo = __shfl_sync(0xffffffffu, keys[V - 1].lo, lane ? lane - 1 : 0);
      pk.hi = __shfl_sync(0xffffffffu, keys[V - 1].hi, lane ? lane - 1 : 0);
      if (lane == 0 && first > 0 && first < e1) pk = load_key<KB>(a.keys, first - 1);
#pragma unroll
      for (int j = 0; j < V; ++j) {
        if (first + j < e1) {
          const Key q = j ? keys[j - 1] : pk;
          const bool h = first + j == 0 || (KB > 0 && (keys[j].lo != q.lo || keys[j].hi != q.hi));
          hm |= (uint32_t)h << j;
        }
      }
      // run index of this lane's first head
      const uint32_t cnt = (uint32_t)__popc(hm);
      uint32_t inc = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= (uint32_t)o) inc += y;
      }
      const uint32_t ttot = __shfl_sync(0xffffffffu, inc, 31);
      const uint64_t run_base = ubase + heads_so_far + (inc - cnt);
      // keys at heads; runs that end inside this lane
      P cur = Op::identity(), pfirst = Op::identity();
      bool seen = false;
      uint32_t r = 0;
#pragma unroll
      for (int j = 0; j < V; ++j) {
        if (first + j < e1) {
          if ((hm >> j) & 1u) {
            if (a.emit)
              reinterpret_cast<unsigned long long*>(a.out_keys)[run_base + r] = a.emit[first + j];
            else
              store_key<KB>(a.out_keys, run_base + r, keys[j]);
            if (seen)
              a.out_vals[run_base + r - 1] = __longlong_as_double((long long)Op::finalize(cur, L));
            else
              pfirst = cur;
            cur = Op::identity();
            seen = true;
            ++r;
          }
          Op::add(cur, vals[j], L, a.inexact);
        }
      }
      if (!seen) pfirst = cur;
      // everything before this lane in the unit, then the run that ends before its first head
      S x;
      x.v = seen ? cur : pfirst;
      x.f = seen;
      x.pad = 0;
      S incl = x;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const S y = shfl_up_any(incl, o);
        if (lane >= (uint32_t)o) incl = seg_combine<Op>(y, incl);
      }
      S ex = shfl_up_any(incl, 1);
      if (lane == 0) {
        ex.v = Op::identity();
        ex.f = 0;
        ex.pad = 0;
      }
      const S X = seg_combine<Op>(carry, ex);
      if (seen) {
        const P y = Op::combine(X.v, pfirst);
        if (X.f)
          a.out_vals[run_base - 1] = __longlong_as_double((long long)Op::finalize(y, L));
        else
          reinterpret_cast<P*>(a.tile_first)[u] = y;   // the run began before this unit
      }
      const S tt = shfl_any(incl, 31);
      carry = seg_combine<Op>(carry, tt);
      heads_so_far += ttot;
    }
    if (lane == 0) {
      if (carry.f)
        reinterpret_cast<P*>(a.tile_last)[u] = carry.v;
      else
        reinterpret_cast<P*>(a.tile_first)[u] = carry.v;
    }
  }
}

// ------------------------------------------------------------------ scalar reductions
__global__ void max_u64_kernel(const unsigned long long* v, uint64_t n, unsigned long long* out) {
  unsigned long long m = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    m = v[i] > m ? v[i] : m;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long y = __shfl_down_sync(0xffffffffu, m, o);
    m = y > m ? y : m;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__global__ void sum_u32_kernel(const uint32_t* v, uint64_t n, uint32_t* out) {
  uint32_t s = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    s += v[i];
  s = __reduce_add_sync(0xffffffffu, s);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

// ------------------------------------------------------------------ host side
struct F64Layout {
  size_t total = 0;
  uint64_t* status = nullptr;
  uint32_t* counter = nullptr;
  uint32_t* tile_heads = nullptr;
  uint32_t* tile_base = nullptr;
  void* tile_first = nullptr;
  void* tile_last = nullptr;
  void* exc = nullptr;
  void* chunk_agg = nullptr;
  int* emax = nullptr;
  uint32_t* inexact = nullptr;
  size_t clear = 0;  // bytes from the start to zero before a launch
};

template <class Op>
F64Layout f64_layout(void* ws, uint64_t n, uint64_t tile_items) {
  using P = typename Op::P;
  const uint64_t tiles = (n + tile_items - 1) / tile_items;
  const uint64_t chunks = (tiles + kFixThreads - 1) / kFixThreads;
  F64Layout l;
  Carver c(ws);
  l.status = c.take<uint64_t>(tiles + 1);
  l.counter = c.take<uint32_t>(4);
  l.emax = c.take<int>(4);
  l.inexact = c.take<uint32_t>(4);
  l.clear = c.used;
  l.tile_heads = c.take<uint32_t>(tiles + 1);
  l.tile_base = c.take<uint32_t>(tiles + 1);
  l.tile_first = c.take<P>(tiles + 1);
  l.tile_last = c.take<P>(tiles + 1);
  l.exc = c.take<Seg<P>>(tiles + 1);
  l.chunk_agg = c.take<Seg<P>>(chunks + 1);
  l.total = c.used + 256;
  return l;
}

size_t f64_core(uint64_t n) {
  const size_t a = f64_layout<SumOp<kNarrowLimbs>>(nullptr, n, kF64UnitItems).total;
  const size_t b = f64_layout<SumOp<kWideLimbs>>(nullptr, n, kF64UnitItems).total;
  const size_t c = f64_layout<MinOp>(nullptr, n, kF64UnitItems).total;
  return align_up(a > b ? (a > c ? a : c) : (b > c ? b : c), 256);
}

// The layouts, then one word past them: the narrow pass's inexact flag, which gates the
// full-range pass.
size_t f64_workspace(uint64_t n) { return f64_core(n) + 256; }

// The unit path: count + scan, one warp per unit, then the tile fix-up over units.
template <int KB, class Op>
rfx_status f64_run_units(F64Args a, void* ws, bool narrow_sum, int fixed_L, cudaStream_t s) {
  const F64Layout l = f64_layout<Op>(ws, a.n, kF64UnitItems);
  RFX_CUDA_TRY(cudaMemsetAsync(ws, 0, l.clear, s));
  a.status = l.status;
  a.counter = l.counter;
  a.tile_heads = l.tile_heads;
  a.tile_base = l.tile_base;
  a.tile_first = l.tile_first;
  a.tile_last = l.tile_last;
  a.exc = l.exc;
  a.chunk_agg = l.chunk_agg;
  a.inexact = l.inexact;
  a.d_emax = narrow_sum ? l.emax : nullptr;
  a.fixed_L = fixed_L;
  const uint64_t units = (a.n + kF64UnitItems - 1) / kF64UnitItems;
  const uint64_t chunks = (units + kFixThreads - 1) / kFixThreads;
  const uint64_t want = (units + 7) / 8;
  const int gc = persistent_grid((const void*)f64_unit_count<KB>, 256, 0, want);
  f64_unit_count<KB><<<gc, 256, 0, s>>>(a, units, narrow_sum ? l.emax : nullptr);
  RFX_CUDA_TRY(cudaGetLastError());
  f64_unit_scan<<<1, 1024, 0, s>>>(a, units);
  RFX_CUDA_TRY(cudaGetLastError());
  const int gm = persistent_grid((const void*)f64_unit_kernel<KB, Op>, 256, 0, want);
  f64_unit_kernel<KB, Op><<<gm, 256, 0, s>>>(a, units);
  RFX_CUDA_TRY(cudaGetLastError());
  f64_fix_scan<Op><<<(int)chunks, kFixThreads, 0, s>>>(a, units);
  RFX_CUDA_TRY(cudaGetLastError());
  f64_fix_chunks<Op><<<1, kFixThreads, 0, s>>>(a, chunks);
  RFX_CUDA_TRY(cudaGetLastError());
  f64_fix_apply<Op><<<(int)chunks, kFixThreads, 0, s>>>(a, units);
  RFX_CUDA_TRY(cudaGetLastError());
  return RFX_OK;
}

template <int KB>
rfx_status f64_dispatch_op(F64Args a, uint32_t op, void* ws, cudaStream_t s) {
  if (op == RFX_F64_MIN) return f64_run_units<KB, MinOp>(a, ws, false, 0, s);
  rfx_status st = f64_run_units<KB, SumOp<kNarrowLimbs>>(a, ws, true, 0, s);
  if (st != RFX_OK) return st;
  // the full-range pass runs on the device only if the narrow window lost bits
  const F64Layout l = f64_layout<SumOp<kNarrowLimbs>>(ws, a.n, kF64UnitItems);
  uint32_t* gate = reinterpret_cast<uint32_t*>(static_cast<uint8_t*>(ws) + f64_core(a.n));
  RFX_CUDA_TRY(cudaMemcpyAsync(gate, l.inexact, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  a.gate = gate;
  return f64_run_units<KB, SumOp<kWideLimbs>>(a, ws, false, kWideL, s);
}

rfx_status f64_dispatch(F64Args a, uint32_t key_bytes, uint32_t op, void* ws, cudaStream_t s) {
  switch (key_bytes) {
    case 0: return f64_dispatch_op<0>(a, op, ws, s);
    case 1: return f64_dispatch_op<1>(a, op, ws, s);
    case 2: return f64_dispatch_op<2>(a, op, ws, s);
    case 4: return f64_dispatch_op<4>(a, op, ws, s);
    case 8: return f64_dispatch_op<8>(a, op, ws, s);
    case 16: return f64_dispatch_op<16>(a, op, ws, s);
    default: return RFX_ERR_UNSUPPORTED;
  }
}

struct DevScratch {
  void* p = nullptr;
  ~DevScratch() {
    if (p) cudaFreeAsync(p, 0);
  }
};

}  // namespace

rfx_status string_codes(const unsigned long long* ptrs, uint64_t n, uint32_t* codes, uint32_t* perm,
                        uint64_t* ndistinct, cudaStream_t s);

rfx_status reduce_f64_impl(const void* keys, uint64_t n, uint32_t key_bytes, const double* values,
                           const unsigned long long* emit, uint32_t op, void* out_keys, double* out_values,
                           uint64_t* d_groups, void* ws, size_t wsb, cudaStream_t s) {
  if (op != RFX_F64_SUM && op != RFX_F64_MIN) return RFX_ERR_INVALID;
  if (key_bytes != 0 && key_bytes != 1 && key_bytes != 2 && key_bytes != 4 && key_bytes != 8 && key_bytes != 16)
    return RFX_ERR_UNSUPPORTED;
  if (!d_groups) return RFX_ERR_INVALID;
  if (n >= (1ull << 30)) return RFX_ERR_UNSUPPORTED;
  if (n == 0) {
    RFX_CUDA_TRY(cudaMemsetAsync(d_groups, 0, sizeof(uint64_t), s));
    return RFX_OK;
  }
  if (!values || !out_values || (key_bytes && !keys) || ((key_bytes || emit) && !out_keys)) return RFX_ERR_INVALID;
  if (!ws || wsb < f64_workspace(n)) return RFX_ERR_WORKSPACE;
  uint32_t* err = device_error_word();
  if (!err) return RFX_ERR_CUDA;
  F64Args a;
  std::memset(&a, 0, sizeof(a));
  a.keys = static_cast<const uint8_t*>(keys);
  a.vals = values;
  a.n = n;
  a.emit = emit;
  a.out_keys = static_cast<uint8_t*>(out_keys);
  a.out_vals = out_values;
  a.d_groups = d_groups;
  a.err = err;
  return f64_dispatch(a, key_bytes, op, ws, s);
}

}  // namespace rfx

using namespace rfx;

extern "C" size_t rfx_reduce_f64_workspace(uint64_t n) { return f64_workspace(n); }

extern "C" rfx_status rfx_reduce_f64(const void* keys, uint64_t n, uint32_t key_bytes, const double* values,
                                     uint32_t op, void* out_keys, double* out_values, uint64_t* d_groups,
                                     void* workspace, size_t workspace_bytes, void* stream) {
  return reduce_f64_impl(keys, n, key_bytes, values, nullptr, op, out_keys, out_values, d_groups, workspace,
                         workspace_bytes, as_stream(stream));
}

namespace {

// The byte-size convention of Reduce.cu: *key_size / *value_size are device byte counts,
// read on entry, replaced by the output byte counts.
rfx_status f64_compat(const void* key_begin, const void* value_begin, void* result_key_begin,
                      void* result_value_begin, uint64_t* key_size, uint64_t* value_size, uint32_t key_bytes,
                      uint32_t op, bool string_keys) {
  if (!key_size || !value_size) return RFX_ERR_INVALID;
  cudaStream_t s = 0;
  uint64_t kbytes = 0;
  RFX_CUDA_TRY(cudaMemcpy(&kbytes, key_size, sizeof(kbytes), cudaMemcpyDeviceToHost));
  const uint64_t n = kbytes / (string_keys ? 8 : key_bytes);
  uint64_t g = 0;
  if (n) {
    DevScratch ws, codes, groups;
    const size_t wsb = f64_workspace(n);
    RFX_CUDA_TRY(cudaMallocAsync(&ws.p, wsb, s));
    RFX_CUDA_TRY(cudaMallocAsync(&groups.p, 16, s));
    const void* keys = key_begin;
    const unsigned long long* emit = nullptr;
    if (string_keys) {
      RFX_CUDA_TRY(cudaMallocAsync(&codes.p, n * 4, s));
      rfx_status st = string_codes(static_cast<const unsigned long long*>(key_begin), n,
                                   static_cast<uint32_t*>(codes.p), nullptr, nullptr, s);
      if (st != RFX_OK) return st;
      keys = codes.p;
      emit = static_cast<const unsigned long long*>(key_begin);
    }
    rfx_status st = reduce_f64_impl(keys, n, key_bytes, static_cast<const double*>(value_begin), emit, op,
                                    result_key_begin, static_cast<double*>(result_value_begin),
                                    static_cast<uint64_t*>(groups.p), ws.p, wsb, s);
    if (st != RFX_OK) return st;
    RFX_CUDA_TRY(cudaMemcpyAsync(&g, groups.p, sizeof(g), cudaMemcpyDeviceToHost, s));
    RFX_CUDA_TRY(cudaStreamSynchronize(s));
  }
  const uint64_t sizes[2] = {g * (string_keys ? 8 : key_bytes), g * 8};
  RFX_CUDA_TRY(cudaMemcpy(key_size, &sizes[0], sizeof(uint64_t), cudaMemcpyHostToDevice));
  RFX_CUDA_TRY(cudaMemcpy(value_size, &sizes[1], sizeof(uint64_t), cudaMemcpyHostToDevice));
  return RFX_OK;
}

}  // namespace

extern "C" rfx_status rfx_total_double_compat(const void* key_begin, const void* value_begin, void* result_key_begin,
                                              void* result_value_begin, uint64_t* key_size, uint64_t* value_size,
                                              uint32_t key_bytes) {
  if (key_bytes != 1 && key_bytes != 2 && key_bytes != 4 && key_bytes != 8 && key_bytes != 16)
    return RFX_ERR_UNSUPPORTED;
  return f64_compat(key_begin, value_begin, result_key_begin, result_value_begin, key_size, value_size, key_bytes,
                    RFX_F64_SUM, false);
}

extern "C" rfx_status rfx_total_string_double_compat(const void* key_begin, const void* value_begin,
                                                     void* result_key_begin, void* result_value_begin,
                                                     uint64_t* key_size, uint64_t* value_size) {
  return f64_compat(key_begin, value_begin, result_key_begin, result_value_begin, key_size, value_size, 4,
                    RFX_F64_SUM, true);
}

extern "C" rfx_status rfx_min_32_double_compat(const void* key_begin, const void* value_begin,
                                               void* result_key_begin, void* result_value_begin, uint64_t* key_size,
                                               uint64_t* value_size) {
  return f64_compat(key_begin, value_begin, result_key_begin, result_value_begin, key_size, value_size, 4,
                    RFX_F64_MIN, false);
}

extern "C" rfx_status rfx_sum_double_compat(void* result, const void* begin, const void* end) {
  if (!result || (!begin && begin != end)) return RFX_ERR_INVALID;
  const uint64_t n = (static_cast<const char*>(end) - static_cast<const char*>(begin)) / 8;
  cudaStream_t s = 0;
  if (n == 0) {  // thrust::reduce of an empty range returns its initial value, 0.0
    RFX_CUDA_TRY(cudaMemset(result, 0, sizeof(double)));
    return RFX_OK;
  }
  DevScratch ws, groups;
  const size_t wsb = f64_workspace(n);
  RFX_CUDA_TRY(cudaMallocAsync(&ws.p, wsb, s));
  RFX_CUDA_TRY(cudaMallocAsync(&groups.p, 16, s));
  rfx_status st = reduce_f64_impl(nullptr, n, 0, static_cast<const double*>(begin), nullptr, RFX_F64_SUM, nullptr,
                                  static_cast<double*>(result), static_cast<uint64_t*>(groups.p), ws.p, wsb, s);
  if (st != RFX_OK) return st;
  RFX_CUDA_TRY(cudaStreamSynchronize(s));
  return RFX_OK;
}

extern "C" rfx_status rfx_max_double_compat(void* result, const void* begin, const void* end) {
  if (!result || (!begin && begin != end)) return RFX_ERR_INVALID;
  const uint64_t n = (static_cast<const char*>(end) - static_cast<const char*>(begin)) / 8;
  cudaStream_t s = 0;
  RFX_CUDA_TRY(cudaMemsetAsync(result, 0, sizeof(unsigned long long), s));
  if (n) {
    const uint64_t blocks = (n + 255) / 256, cap = (uint64_t)device_sms() * 8;
    max_u64_kernel<<<(int)(blocks < cap ? blocks : cap), 256, 0, s>>>(
        static_cast<const unsigned long long*>(begin), n, static_cast<unsigned long long*>(result));
    RFX_CUDA_TRY(cudaGetLastError());
  }
  RFX_CUDA_TRY(cudaStreamSynchronize(s));
  return RFX_OK;
}

extern "C" rfx_status rfx_count_u32_compat(void* result, const void* begin, const void* end) {
  if (!result || (!begin && begin != end)) return RFX_ERR_INVALID;
  const uint64_t n = (static_cast<const char*>(end) - static_cast<const char*>(begin)) / 4;
  cudaStream_t s = 0;
  RFX_CUDA_TRY(cudaMemsetAsync(result, 0, sizeof(uint32_t), s));
  if (n) {
    const uint64_t blocks = (n + 255) / 256, cap = (uint64_t)device_sms() * 8;
    sum_u32_kernel<<<(int)(blocks < cap ? blocks : cap), 256, 0, s>>>(static_cast<const uint32_t*>(begin), n,
                                                                     static_cast<uint32_t*>(result));
    RFX_CUDA_TRY(cudaGetLastError());
  }
  RFX_CUDA_TRY(cudaStreamSynchronize(s));
  return RFX_OK;
}
