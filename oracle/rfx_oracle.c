/*
 * rfx_oracle.c -- CPU restatement of Red Fox's RA kernel library (test infrastructure).
 *
 * The oracle is the checker for redfox_b200's CUDA kernels, never the product: only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.  Each
 * function states the reference semantics it follows with file:line citations into the
 * sidharth87/redfox tree.  Parity of this restatement is pinned by tests/golden/.
 */
#include "rfx_oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------------------------
 * Packed tuple codec -- Tuple.h
 * ----------------------------------------------------------------------------------*/

/* Clamp<v> (Tuple.h:31-37): the container width for a tuple of `bits` used bits. */
uint32_t orc_clamp_bits(uint32_t v)
{
    return v <= 8 ? 8 : v <= 16 ? 16 : v <= 32 ? 32 : v <= 64 ? 64
         : v <= 128 ? 128 : v <= 256 ? 256 : v <= 512 ? 512 : 0;
}

/* Tuple::bits (Tuple.h:735-736): the unclamped sum of the field widths. */
uint32_t orc_tuple_bits(const orc_tuple* t)
{
    uint32_t s = 0;
    for (uint32_t i = 0; i < t->nfields && i < 16; ++i) s += t->widths[i];
    return s;
}

uint32_t orc_tuple_bytes(const orc_tuple* t) { return orc_clamp_bits(orc_tuple_bits(t)) / 8; }

/* BitsAfter<index> (Tuple.h:697-705): field 0 occupies the most significant used bits. */
uint32_t orc_field_shift(const orc_tuple* t, uint32_t field)
{
    uint32_t upto = 0;
    for (uint32_t i = 0; i <= field && i < t->nfields; ++i) upto += t->widths[i];
    return orc_tuple_bits(t) - upto;
}

static inline uint64_t width_mask(uint32_t w) { return w >= 64 ? ~0ull : ((1ull << w) - 1); }

uint64_t orc_get_bits(const uint8_t* e, uint32_t ebytes, uint32_t shift, uint32_t width)
{
    if (width == 0) return 0;
    uint32_t b0 = shift >> 3, off = shift & 7;
    u128 w = 0;
    for (uint32_t k = 0; k < 9 && b0 + k < ebytes; ++k) w |= (u128)e[b0 + k] << (8 * k);
    return (uint64_t)(w >> off) & width_mask(width);
}

void orc_set_bits(uint8_t* e, uint32_t ebytes, uint32_t shift, uint32_t width, uint64_t v)
{
    if (width == 0) return;
    uint32_t b0 = shift >> 3, off = shift & 7;
    u128 w = 0;
    uint32_t nb = 0;
    for (uint32_t k = 0; k < 9 && b0 + k < ebytes; ++k, ++nb) w |= (u128)e[b0 + k] << (8 * k);
    u128 m = (u128)width_mask(width) << off;
    w = (w & ~m) | (((u128)v << off) & m);
    for (uint32_t k = 0; k < nb; ++k) e[b0 + k] = (uint8_t)(w >> (8 * k));
}

/* extract<T, Index, Tuple> (Tuple.h:777-790): (tuple >> BitsAfter) & mask(BitsAt).
 * A 64-bit field is taken whole (the intended all-ones mask). */
uint64_t orc_extract(const uint8_t* e, const orc_tuple* t, uint32_t field)
{
    if (field >= t->nfields || field >= 16) return 0;
    return orc_get_bits(e, orc_tuple_bytes(t), orc_field_shift(t, field), t->widths[field]);
}

/* insert<T, Index, Tuple> (Tuple.h:849-861): (tuple & ~mask) | ((value << shift) & mask). */
void orc_insert(uint8_t* e, const orc_tuple* t, uint32_t field, uint64_t v)
{
    if (field >= t->nfields || field >= 16) return;
    uint32_t w = t->widths[field];
    orc_set_bits(e, orc_tuple_bytes(t), orc_field_shift(t, field), w, v & width_mask(w));
}

void orc_pack_rows(uint8_t* out, size_t n, const orc_tuple* t, const uint64_t* const* cols)
{
    uint32_t W = orc_tuple_bytes(t);
    memset(out, 0, n * W);
    for (size_t i = 0; i < n; ++i)
        for (uint32_t f = 0; f < t->nfields; ++f) orc_insert(out + i * W, t, f, cols[f][i]);
}

void orc_unpack_rows(const uint8_t* in, size_t n, const orc_tuple* t, uint64_t* const* cols)
{
    uint32_t W = orc_tuple_bytes(t);
    for (size_t i = 0; i < n; ++i)
        for (uint32_t f = 0; f < t->nfields; ++f) cols[f][i] = orc_extract(in + i * W, t, f);
}

/* PackedNBytes::operator< (Tuple.h:466-534) and the gpu128 comparators
 * (ModernGPUJoin.cu:27-39, Union.cu:22-32): unsigned, most significant limb first. */
int orc_compare(const uint8_t* a, const uint8_t* b, uint32_t ebytes)
{
    for (int k = (int)ebytes - 1; k >= 0; --k) {
        if (a[k] < b[k]) return -1;
        if (a[k] > b[k]) return 1;
    }
    return 0;
}

/* Limb helpers for containers up to 64 bytes (8 little-endian 64-bit limbs). */
static void limbs_load(uint64_t L[8], const uint8_t* e, uint32_t ebytes)
{
    memset(L, 0, 8 * sizeof(uint64_t));
    memcpy(L, e, ebytes);
}
static void limbs_store(uint8_t* e, uint32_t ebytes, const uint64_t L[8]) { memcpy(e, L, ebytes); }

/* PackedNBytes::operator<< (Tuple.h:325-363), restricted to the container's limbs. */
static void limbs_shl(uint64_t L[8], uint32_t amount)
{
    uint64_t R[8] = {0};
    uint32_t q = amount / 64, r = amount % 64;
    for (int i = 7; i >= 0; --i) {
        int src = i - (int)q;
        if (src < 0) continue;
        uint64_t v = L[src] << r;
        if (r && src - 1 >= 0) v |= L[src - 1] >> (64 - r);
        R[i] = v;
    }
    memcpy(L, R, sizeof(R));
}
/* PackedNBytes::operator>> (Tuple.h:286-323). */
static void limbs_shr(uint64_t L[8], uint32_t amount)
{
    uint64_t R[8] = {0};
    uint32_t q = amount / 64, r = amount % 64;
    for (int i = 0; i < 8; ++i) {
        int src = i + (int)q;
        if (src > 7) continue;
        uint64_t v = L[src] >> r;
        if (r && src + 1 <= 7) v |= L[src + 1] << (64 - r);
        R[i] = v;
    }
    memcpy(L, R, sizeof(R));
}
static void limbs_mask_low(uint64_t L[8], uint32_t bits)
{
    for (int i = 0; i < 8; ++i) {
        uint32_t lo = (uint32_t)i * 64;
        if (bits <= lo) L[i] = 0;
        else if (bits < lo + 64) L[i] &= (1ull << (bits - lo)) - 1;
    }
}
static int limbs_cmp(const uint64_t A[8], const uint64_t B[8])
{
    for (int i = 7; i >= 0; --i) {
        if (A[i] < B[i]) return -1;
        if (A[i] > B[i]) return 1;
    }
    return 0;
}

/* ------------------------------------------------------------------------------------
 * Sort -- b40cSort.cu:58-1022 (LSD radix, stable, on bits [0, key_bits)) and
 * ModernGPUSort.cu (stable merge sort).  A stable sort is unique for a given key
 * function, so an LSD counting sort on bits [begin_bit, end_bit) restates both.
 * ----------------------------------------------------------------------------------*/
void orc_sort_pairs(void* keys, void* vals, size_t n, uint32_t kb, uint32_t vb,
                    uint32_t begin_bit, uint32_t end_bit)
{
    orc_sort_pairs_mt(keys, vals, n, kb, vb, begin_bit, end_bit, 1);
}

void orc_sort_pairs_mt(void* keys, void* vals, size_t n, uint32_t kb, uint32_t vb,
                       uint32_t begin_bit, uint32_t end_bit, int threads)
{
    if (n <= 1 || end_bit <= begin_bit) return;
    if (threads < 1) threads = 1;
    uint8_t* k0 = (uint8_t*)keys;
    uint8_t* v0 = (uint8_t*)vals;
    uint8_t* k1 = (uint8_t*)malloc(n * kb);
    uint8_t* v1 = vals ? (uint8_t*)malloc(n * vb) : NULL;
    uint8_t* digits = (uint8_t*)malloc(n);
    size_t (*hist)[256] = (size_t (*)[256])calloc((size_t)threads, sizeof(size_t[256]));
    uint8_t *ks = k0, *kd = k1, *vs = v0, *vd = v1;
    for (uint32_t bit = begin_bit; bit < end_bit; bit += 8) {
        uint32_t w = end_bit - bit < 8 ? end_bit - bit : 8;
        memset(hist, 0, (size_t)threads * sizeof(size_t[256]));
#pragma omp parallel num_threads(threads)
        {
            int t = 0, nt = 1;
#ifdef _OPENMP
            t = omp_get_thread_num();
            nt = omp_get_num_threads();
#endif
            size_t lo = n * (size_t)t / (size_t)nt, hi = n * (size_t)(t + 1) / (size_t)nt;
            for (size_t i = lo; i < hi; ++i) {
                uint8_t d = (uint8_t)orc_get_bits(ks + i * kb, kb, bit, w);
                digits[i] = d;
                hist[t][d]++;
            }
#pragma omp barrier
#pragma omp single
            {
                size_t run = 0;
                for (int d = 0; d < 256; ++d)
                    for (int tt = 0; tt < nt; ++tt) {
                        size_t c = hist[tt][d];
                        hist[tt][d] = run;
                        run += c;
                    }
            }
            for (size_t i = lo; i < hi; ++i) {
                size_t dst = hist[t][digits[i]]++;
                memcpy(kd + dst * kb, ks + i * kb, kb);
                if (vals) memcpy(vd + dst * vb, vs + i * vb, vb);
            }
        }
        uint8_t* tmp = ks; ks = kd; kd = tmp;
        tmp = vs; vs = vd; vd = tmp;
    }
    if (ks != k0) {
        memcpy(k0, ks, n * kb);
        if (vals) memcpy(v0, vs, n * vb);
    }
    free(k1);
    free(v1);
    free(digits);
    free(hist);
}

/* ------------------------------------------------------------------------------------
 * Join -- ModernGPUJoin.cu / ModernGPUJoin.h; output order of CPUJoin
 * (moderngpu/tests/benchmarkjoin.cu:40-128).
 * ----------------------------------------------------------------------------------*/
static size_t lower_bound_c(const uint8_t* a, size_t n, const uint8_t* key, uint32_t kb)
{
    size_t lo = 0, hi = n;
    while (lo < hi) {
        size_t mid = lo + (hi - lo) / 2;
        if (orc_compare(a + mid * kb, key, kb) < 0) lo = mid + 1; else hi = mid;
    }
    return lo;
}
static size_t upper_bound_c(const uint8_t* a, size_t n, const uint8_t* key, uint32_t kb)
{
    size_t lo = 0, hi = n;
    while (lo < hi) {
        size_t mid = lo + (hi - lo) / 2;
        if (orc_compare(a + mid * kb, key, kb) <= 0) lo = mid + 1; else hi = mid;
    }
    return lo;
}

/* find_bounds_{8..128} (ModernGPUJoin.cu:109-663): SortedSearch lower bound of each
 * left key in right (:161-163), SortedEqualityCount = upper - lower (:172-177,
 * sortedsearch.cuh:311-315), then an in-place exclusive Scan whose total goes to
 * *result_size (:184-188).  Counts and the scan are int32 as in the reference. */
void orc_find_bounds(int32_t* lb, int32_t* cnt, uint64_t* total,
                     const void* left, size_t nl, const void* right, size_t nr, uint32_t kb)
{
    const uint8_t* L = (const uint8_t*)left;
    const uint8_t* R = (const uint8_t*)right;
    uint64_t run = 0;
    for (size_t i = 0; i < nl; ++i) {
        size_t lo = lower_bound_c(R, nr, L + i * kb, kb);
        size_t hi = upper_bound_c(R, nr, L + i * kb, kb);
        lb[i] = (int32_t)lo;
        cnt[i] = (int32_t)(uint32_t)run;
        run += hi - lo;
    }
    *total = run;
}

/* join (ModernGPUJoin.cu:665-733) = KernelLeftJoin<Tuning, false>: output k belongs to
 * the left row i with scan[i] <= k < scan[i+1]; its right row is lower_bound[i] +
 * (k - scan[i]).  Order: left ascending, right ascending (CPUJoin :104-122). */
void orc_join_expand(int32_t* li, int32_t* ri, uint64_t nout,
                     const int32_t* lb, const int32_t* scan, size_t nl)
{
    for (size_t i = 0; i < nl; ++i) {
        uint64_t b = (uint32_t)scan[i];
        uint64_t e = (i + 1 < nl) ? (uint64_t)(uint32_t)scan[i + 1] : nout;
        for (uint64_t k = b; k < e && k < nout; ++k) {
            li[k] = (int32_t)i;
            ri[k] = (int32_t)(lb[i] + (int32_t)(k - b));
        }
    }
}

/* gather_{key_key,key_value,value_key,value_value} (ModernGPUJoin.h:43-200):
 *   out = restoreValues(lkey[li]) | (lval[li] << RightValue::bits) | rval[ri]
 * where restoreValues shifts the key left by the output's value bits (Tuple.h:929-936).
 * Absent sides are passed as NULL with zero bits. */
void orc_join_gather(void* out, uint32_t ob, uint64_t nout,
                     const int32_t* li, const int32_t* ri,
                     const void* lkey, uint32_t lkb, const void* lval, uint32_t lvb,
                     uint32_t lv_bits, const void* rval, uint32_t rvb, uint32_t rv_bits)
{
    uint8_t* O = (uint8_t*)out;
    for (uint64_t k = 0; k < nout; ++k) {
        uint64_t acc[8], tmp[8];
        limbs_load(acc, (const uint8_t*)lkey + (size_t)li[k] * lkb, lkb);
        limbs_shl(acc, lv_bits + rv_bits);
        if (lval) {
            limbs_load(tmp, (const uint8_t*)lval + (size_t)li[k] * lvb, lvb);
            limbs_shl(tmp, rv_bits);
            for (int j = 0; j < 8; ++j) acc[j] |= tmp[j];
        }
        if (rval) {
            limbs_load(tmp, (const uint8_t*)rval + (size_t)ri[k] * rvb, rvb);
            for (int j = 0; j < 8; ++j) acc[j] |= tmp[j];
        }
        limbs_store(O + k * ob, ob, acc);
    }
}

static int tuple_key_cmp(const uint8_t* a, uint32_t ab, uint32_t ashift,
                         const uint8_t* b, uint32_t bb, uint32_t bshift)
{
    uint64_t A[8], B[8];
    limbs_load(A, a, ab);
    limbs_shr(A, ashift);
    limbs_load(B, b, bb);
    limbs_shr(B, bshift);
    return limbs_cmp(A, B);
}

/* Number of rows of the fused tuple join (same matches as find_bounds + join). */
uint64_t orc_join_count_tuples(const void* left, size_t nl, uint32_t lb, uint32_t lvbits,
                               const void* right, size_t nr, uint32_t rb, uint32_t rvbits)
{
    return orc_join_tuples(NULL, 0, 0, left, nl, lb, lvbits, right, nr, rb, rvbits);
}

/* Fused sort-merge join of packed tuples sorted on their key fields (the high fields):
 * the match set and order of find_bounds + join (above), and the output tuple of
 * combine<Left, Right, Out, keys> (Tuple.h:942-955) = (L << RV bits) | (R & mask(RV)),
 * which equals gather_value_value on the split key/value arrays.  Returns the total;
 * writes the first min(total, cap) rows. */
uint64_t orc_join_tuples(void* out, uint32_t ob, uint64_t cap,
                         const void* left, size_t nl, uint32_t lbytes, uint32_t lvbits,
                         const void* right, size_t nr, uint32_t rbytes, uint32_t rvbits)
{
    const uint8_t* L = (const uint8_t*)left;
    const uint8_t* R = (const uint8_t*)right;
    uint8_t* O = (uint8_t*)out;
    uint64_t total = 0;
    size_t j0 = 0;
    for (size_t i = 0; i < nl; ++i) {
        const uint8_t* l = L + i * lbytes;
        /* lower bound of l's key in R, starting from the previous one (keys sorted) */
        if (i > 0 && tuple_key_cmp(l, lbytes, lvbits, L + (i - 1) * lbytes, lbytes, lvbits) < 0)
            j0 = 0; /* unsorted input: restart the search */
        while (j0 < nr && tuple_key_cmp(R + j0 * rbytes, rbytes, rvbits, l, lbytes, lvbits) < 0) ++j0;
        for (size_t j = j0; j < nr; ++j) {
            const uint8_t* r = R + j * rbytes;
            if (tuple_key_cmp(r, rbytes, rvbits, l, lbytes, lvbits) != 0) break;
            if (O && total < cap) {
                uint64_t acc[8], tmp[8];
                limbs_load(acc, l, lbytes);
                limbs_shl(acc, rvbits);
                limbs_load(tmp, r, rbytes);
                limbs_mask_low(tmp, rvbits);
                for (int k = 0; k < 8; ++k) acc[k] |= tmp[k];
                limbs_store(O + total * ob, ob, acc);
            }
            ++total;
        }
    }
    return total;
}

/* ------------------------------------------------------------------------------------
 * Reduce / count -- Reduce.cu: thrust::reduce_by_key over runs of equal keys
 * (equal_to on the container, compare_128/256 :85-101), plus<> on the values.
 * ----------------------------------------------------------------------------------*/
uint64_t orc_reduce_sum_i64(const void* keys, size_t n, uint32_t kb, const int64_t* vals,
                            void* out_keys, int64_t* out_vals)
{
    const uint8_t* K = (const uint8_t*)keys;
    uint8_t* OK = (uint8_t*)out_keys;
    uint64_t g = 0;
    size_t i = 0;
    while (i < n) {
        uint64_t s = 0;
        size_t j = i;
        while (j < n && memcmp(K + j * kb, K + i * kb, kb) == 0) s += (uint64_t)vals[j++];
        memcpy(OK + g * kb, K + i * kb, kb);
        out_vals[g++] = (int64_t)s;
        i = j;
    }
    return g;
}

/* count_{8,16,32,128,256} (Reduce.cu:175-660): reduce_by_key of a u32 column (the
 * generated ones of set_generate, Split_Merge.h) with plus<unsigned int>.  A NULL
 * column counts rows. */
uint64_t orc_reduce_count(const void* keys, size_t n, uint32_t kb, const uint32_t* vals,
                          void* out_keys, uint32_t* out_counts)
{
    const uint8_t* K = (const uint8_t*)keys;
    uint8_t* OK = (uint8_t*)out_keys;
    uint64_t g = 0;
    size_t i = 0;
    while (i < n) {
        uint32_t s = 0;
        size_t j = i;
        while (j < n && memcmp(K + j * kb, K + i * kb, kb) == 0) s += vals ? vals[j++] : (j++, 1u);
        memcpy(OK + g * kb, K + i * kb, kb);
        out_counts[g++] = s;
        i = j;
    }
    return g;
}

/* ------------------------------------------------------------------------------------
 * Set operations on sorted multisets -- thrust/STL semantics (Union.cu:47-148,
 * Difference.cu:35-143; intersection as benchmarksets.cu:95-125 checks it).
 * ----------------------------------------------------------------------------------*/
uint64_t orc_set_union(void* out, const void* a, size_t na, const void* b, size_t nb, uint32_t e)
{
    const uint8_t *A = (const uint8_t*)a, *B = (const uint8_t*)b;
    uint8_t* O = (uint8_t*)out;
    size_t i = 0, j = 0;
    uint64_t k = 0;
    while (i < na && j < nb) {
        int c = orc_compare(A + i * e, B + j * e, e);
        if (c < 0) memcpy(O + (k++) * e, A + (i++) * e, e);
        else if (c > 0) memcpy(O + (k++) * e, B + (j++) * e, e);
        else { memcpy(O + (k++) * e, A + (i++) * e, e); ++j; }
    }
    while (i < na) memcpy(O + (k++) * e, A + (i++) * e, e);
    while (j < nb) memcpy(O + (k++) * e, B + (j++) * e, e);
    return k;
}

uint64_t orc_set_difference(void* out, const void* a, size_t na, const void* b, size_t nb, uint32_t e)
{
    const uint8_t *A = (const uint8_t*)a, *B = (const uint8_t*)b;
    uint8_t* O = (uint8_t*)out;
    size_t i = 0, j = 0;
    uint64_t k = 0;
    while (i < na && j < nb) {
        int c = orc_compare(A + i * e, B + j * e, e);
        if (c < 0) memcpy(O + (k++) * e, A + (i++) * e, e);
        else if (c > 0) ++j;
        else { ++i; ++j; }
    }
    while (i < na) memcpy(O + (k++) * e, A + (i++) * e, e);
    return k;
}

uint64_t orc_set_intersection(void* out, const void* a, size_t na, const void* b, size_t nb, uint32_t e)
{
    const uint8_t *A = (const uint8_t*)a, *B = (const uint8_t*)b;
    uint8_t* O = (uint8_t*)out;
    size_t i = 0, j = 0;
    uint64_t k = 0;
    while (i < na && j < nb) {
        int c = orc_compare(A + i * e, B + j * e, e);
        if (c < 0) ++i;
        else if (c > 0) ++j;
        else { memcpy(O + (k++) * e, A + (i++) * e, e); ++j; }
    }
    return k;
}

/* unique (Unique.cu:36-114): thrust::unique keeps the first of each run of equal
 * adjacent elements, in place. */
uint64_t orc_unique(void* data, size_t n, uint32_t e)
{
    uint8_t* D = (uint8_t*)data;
    if (n == 0) return 0;
    uint64_t k = 1;
    for (size_t i = 1; i < n; ++i)
        if (memcmp(D + i * e, D + (k - 1) * e, e) != 0) {
            if (k != i) memmove(D + k * e, D + i * e, e);
            ++k;
        }
    return k;
}

/* ------------------------------------------------------------------------------------
 * Select / arith / project
 * ----------------------------------------------------------------------------------*/
static uint64_t type_mask(uint32_t type)
{
    switch (type) {
    case ORC_I8: return 0xffull;
    case ORC_I16: return 0xffffull;
    case ORC_I32: return 0xffffffffull;
    default: return ~0ull;
    }
}

/* select_field_constant / select_field_field (Select.h:30-114, :650-740) with the
 * functors of Comparisons.h: operands are the field's unsigned C type (mapValueType,
 * RelationalAlgebraKernel.cpp:78-119); the signed codes compare exactly like the
 * unsigned ones (Comparisons.h:210-300).  A constant on the left is evaluated as
 * written (the generator mirrors the operator, RelationalAlgebraKernel.cpp:145-219). */
int orc_eval_cmp(const uint8_t* row, const orc_tuple* t, const orc_cmp* c)
{
    uint64_t m = type_mask(c->value_type);
    uint64_t a = (c->a_kind == ORC_OPND_VARIABLE ? orc_extract(row, t, c->a_field) : c->a_const) & m;
    uint64_t b = (c->b_kind == ORC_OPND_VARIABLE ? orc_extract(row, t, c->b_field) : c->b_const) & m;
    switch (c->op) {
    case ORC_EQ: return a == b;
    case ORC_NE: return a != b;
    case ORC_SLT: case ORC_LT: return a < b;
    case ORC_SLE: case ORC_LE: return a <= b;
    case ORC_SGT: case ORC_GT: return a > b;
    case ORC_SGE: case ORC_GE: return a >= b;
    default: return 0;
    }
}

/* Stable (input-order-preserving) filter: set_select + scan + select_gather
 * (Select.h:30-114, :1013-1127); all comparisons are ANDed (ComparisonVector). */
uint64_t orc_select(void* out, const void* in, size_t n, const orc_tuple* t,
                    const orc_cmp* cmps, uint32_t ncmp)
{
    uint32_t W = orc_tuple_bytes(t);
    const uint8_t* I = (const uint8_t*)in;
    uint8_t* O = (uint8_t*)out;
    uint64_t k = 0;
    for (size_t i = 0; i < n; ++i) {
        int pass = 1;
        for (uint32_t c = 0; c < ncmp && pass; ++c) pass = orc_eval_cmp(I + i * W, t, &cmps[c]);
        if (pass) memcpy(O + (k++) * W, I + i * W, W);
    }
    return k;
}

/* C types of the generated arithmetic (arithToString, RelationalAlgebraKernel.cpp:1891-1939):
 * index nodes are extract<mapValueType> (unsigned char/short promote to int), constants
 * are decimal literals (int, then long, then unsigned long), and binary operators apply
 * the usual arithmetic conversions.  Signed overflow wraps; x / 0 and x % 0 give 0. */
enum { CT_I32, CT_U32, CT_I64, CT_U64 };
typedef struct { int ct; uint64_t v; } cval;

static cval cv_norm(cval x)
{
    switch (x.ct) {
    case CT_I32: x.v = (uint64_t)(int64_t)(int32_t)(uint32_t)x.v; break;
    case CT_U32: x.v = (uint32_t)x.v; break;
    default: break;
    }
    return x;
}

static int arith_eval_rec(const orc_arith* a, uint32_t idx, const uint64_t* fields,
                          uint32_t nfields, int depth, cval* out)
{
    if (idx >= a->nnodes || depth > 64) return -1;
    const orc_node* nd = &a->nodes[idx];
    if (nd->kind == ORC_NODE_CONST) {
        cval r;
        r.v = nd->value;
        r.ct = nd->value <= 0x7fffffffull ? CT_I32 : nd->value <= 0x7fffffffffffffffull ? CT_I64 : CT_U64;
        *out = cv_norm(r);
        return 0;
    }
    if (nd->kind == ORC_NODE_INDEX) {
        if (nd->value >= nfields) return -1;
        uint64_t v = fields[nd->value];
        cval r;
        switch (nd->type) {
        case ORC_I8: r.ct = CT_I32; r.v = v & 0xff; break;
        case ORC_I16: r.ct = CT_I32; r.v = v & 0xffff; break;
        case ORC_I32: r.ct = CT_U32; r.v = v & 0xffffffffull; break;
        case ORC_I64: r.ct = CT_U64; r.v = v; break;
        default: return -1;
        }
        *out = r;
        return 0;
    }
    if (nd->kind != ORC_NODE_OP) return -1;
    cval l, r;
    if (arith_eval_rec(a, (uint32_t)nd->left, fields, nfields, depth + 1, &l)) return -1;
    if (arith_eval_rec(a, (uint32_t)nd->right, fields, nfields, depth + 1, &r)) return -1;
    int wide = (l.ct >= CT_I64) || (r.ct >= CT_I64);
    int ct;
    if (wide) ct = (l.ct == CT_U64 || r.ct == CT_U64) ? CT_U64 : CT_I64;
    else ct = (l.ct == CT_U32 || r.ct == CT_U32) ? CT_U32 : CT_I32;
    /* convert both operands to ct */
    uint64_t x = l.v, y = r.v;
    if (wide) {
        /* 32-bit signed values are already sign-extended, unsigned zero-extended */
    } else {
        x = (uint32_t)x;
        y = (uint32_t)y;
    }
    int sgn = (ct == CT_I32 || ct == CT_I64);
    cval res;
    res.ct = ct;
    switch (nd->op) {
    case ORC_ADD: res.v = x + y; break;
    case ORC_SUB: res.v = x - y; break;
    case ORC_MUL: res.v = x * y; break;
    case ORC_DIV:
    case ORC_MOD:
        if ((wide ? y : (uint32_t)y) == 0) { res.v = 0; break; }
        if (sgn) {
            int64_t sx = wide ? (int64_t)x : (int64_t)(int32_t)(uint32_t)x;
            int64_t sy = wide ? (int64_t)y : (int64_t)(int32_t)(uint32_t)y;
            int64_t minv = wide ? (int64_t)0x8000000000000000ull : (int64_t)(int32_t)0x80000000u;
            if (sx == minv && sy == -1) res.v = nd->op == ORC_DIV ? (uint64_t)sx : 0;
            else res.v = (uint64_t)(nd->op == ORC_DIV ? sx / sy : sx % sy);
        } else {
            uint64_t ux = wide ? x : (uint32_t)x, uy = wide ? y : (uint32_t)y;
            res.v = nd->op == ORC_DIV ? ux / uy : ux % uy;
        }
        break;
    default: return -1;
    }
    *out = cv_norm(res);
    return 0;
}

static int arith_eval_fields(const orc_arith* a, const uint64_t* fields, uint32_t nfields,
                             uint64_t* result)
{
    cval r;
    if (arith_eval_rec(a, a->root, fields, nfields, 0, &r)) return -1;
    /* mapValueType(dest) tmp2 = expr;  then insert masks to the field width */
    *result = r.v & type_mask(a->dest_type) & width_mask(a->dest_bits);
    return 0;
}

int orc_arith_eval(const uint8_t* row, const orc_tuple* t, const orc_arith* a, uint64_t* result)
{
    uint64_t f[16];
    for (uint32_t i = 0; i < t->nfields; ++i) f[i] = orc_extract(row, t, i);
    return arith_eval_fields(a, f, t->nfields, result);
}

/* set_arith (RelationalAlgebraKernel.cpp:2130-2150): result = (ResultType)src << new_bits
 * with the new last field = the expression; the result tuple is src's fields + one. */
int orc_arith_rows(void* out, const void* in, size_t n, const orc_tuple* t, const orc_arith* a)
{
    orc_tuple ot = *t;
    if (t->nfields >= 16) return -1;
    ot.widths[ot.nfields++] = a->dest_bits;
    uint32_t IW = orc_tuple_bytes(t), OW = orc_tuple_bytes(&ot);
    if (OW == 0) return -1;
    const uint8_t* I = (const uint8_t*)in;
    uint8_t* O = (uint8_t*)out;
    for (size_t i = 0; i < n; ++i) {
        uint64_t v, L[8];
        if (orc_arith_eval(I + i * IW, t, a, &v)) return -1;
        limbs_load(L, I + i * IW, IW);
        limbs_shl(L, a->dest_bits);
        limbs_store(O + i * OW, OW, L);
        orc_insert(O + i * OW, &ot, ot.nfields - 1, v);
    }
    return 0;
}

/* permute / permuteElement (Project.h:58-121): out field k = in field map[k], fields
 * extracted as unsigned long long; a map entry >= 16 (the generator's 100) yields 0. */
void orc_project(void* out, const void* in, size_t n, const orc_tuple* it,
                 const orc_tuple* ot, const uint32_t* map)
{
    uint32_t IW = orc_tuple_bytes(it), OW = orc_tuple_bytes(ot);
    const uint8_t* I = (const uint8_t*)in;
    uint8_t* O = (uint8_t*)out;
    for (size_t i = 0; i < n; ++i) {
        memset(O + i * OW, 0, OW);
        for (uint32_t k = 0; k < ot->nfields; ++k)
            orc_insert(O + i * OW, ot, k, map[k] < 16 ? orc_extract(I + i * IW, it, map[k]) : 0);
    }
}

/* ------------------------------------------------------------------------------------
 * Fused filter -> arith* -> project -> sort -> reduce(SUM int64) + COUNT.
 * Restates the plan addSelectConstant + addArith + addProjection + addAgg
 * (RelationalAlgebraCompiler.cpp:6523, :7852-8643): groups come out ascending by the
 * packed group key (sort_pair then reduce_by_key), sums are exact int64 (wrapping),
 * counts are row counts.  Returns the number of groups, -1 if more than `cap`, -2 on a
 * bad descriptor.
 * ----------------------------------------------------------------------------------*/
typedef struct { uint64_t key; uint64_t cnt; int64_t s[8]; int used; } agg_slot;

static int agg_cmp(const void* a, const void* b)
{
    const agg_slot* x = (const agg_slot*)a;
    const agg_slot* y = (const agg_slot*)b;
    return x->key < y->key ? -1 : x->key > y->key ? 1 : 0;
}

static uint64_t hash64(uint64_t x)
{
    x ^= x >> 33; x *= 0xff51afd7ed558ccdull; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ull;
    return x ^ (x >> 33);
}

int64_t orc_filter_aggregate(const void* in, size_t n, const orc_tuple* t,
                             const orc_cmp* cmps, uint32_t ncmp,
                             const orc_arith* ariths, uint32_t narith,
                             const uint32_t* gf, uint32_t ngroup,
                             const uint32_t* sf, uint32_t nsum,
                             uint64_t* out_keys, int64_t* out_sums, uint64_t* out_counts,
                             uint64_t cap, int threads)
{
    uint32_t W = orc_tuple_bytes(t);
    uint32_t nf = t->nfields + narith;
    if (W == 0 || nf > 16 || nsum > 8 || ngroup == 0 || ngroup > 16) return -2;
    uint32_t ext_w[16];
    for (uint32_t i = 0; i < t->nfields; ++i) ext_w[i] = t->widths[i];
    for (uint32_t i = 0; i < narith; ++i) ext_w[t->nfields + i] = ariths[i].dest_bits;
    uint32_t gbits = 0;
    for (uint32_t i = 0; i < ngroup; ++i) {
        if (gf[i] >= nf) return -2;
        gbits += ext_w[gf[i]];
    }
    for (uint32_t i = 0; i < nsum; ++i) if (sf[i] >= nf) return -2;
    if (gbits > 64) return -2;
    if (threads < 1) threads = 1;
    size_t tcap = 64;
    while (tcap < 2 * cap) tcap <<= 1;
    agg_slot* tables = (agg_slot*)calloc((size_t)threads * tcap, sizeof(agg_slot));
    int overflow = 0, bad = 0;
    const uint8_t* I = (const uint8_t*)in;
#pragma omp parallel num_threads(threads)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        agg_slot* tab = tables + (size_t)tid * tcap;
        uint64_t used = 0;
#pragma omp for schedule(static)
        for (size_t i = 0; i < n; ++i) {
            const uint8_t* row = I + i * W;
            int pass = 1;
            for (uint32_t c = 0; c < ncmp && pass; ++c) pass = orc_eval_cmp(row, t, &cmps[c]);
            if (!pass) continue;
            uint64_t f[16];
            for (uint32_t k = 0; k < t->nfields; ++k) f[k] = orc_extract(row, t, k);
            for (uint32_t k = 0; k < narith; ++k)
                if (arith_eval_fields(&ariths[k], f, t->nfields + k, &f[t->nfields + k])) bad = 1;
            uint64_t key = 0;
            for (uint32_t k = 0; k < ngroup; ++k) {
                uint32_t w = ext_w[gf[k]];
                key = (w >= 64 ? 0 : key << w) | (f[gf[k]] & width_mask(w));
            }
            size_t h = hash64(key) & (tcap - 1);
            while (tab[h].used && tab[h].key != key) h = (h + 1) & (tcap - 1);
            if (!tab[h].used) {
                if (++used > cap) { overflow = 1; continue; }
                tab[h].used = 1;
                tab[h].key = key;
            }
            tab[h].cnt++;
            for (uint32_t k = 0; k < nsum; ++k) tab[h].s[k] = (int64_t)((uint64_t)tab[h].s[k] + f[sf[k]]);
        }
    }
    int64_t result = -1;
    if (!overflow && !bad) {
        agg_slot* merged = (agg_slot*)calloc(tcap, sizeof(agg_slot));
        uint64_t g = 0;
        for (int tt = 0; tt < threads && !overflow; ++tt)
            for (size_t h = 0; h < tcap; ++h) {
                agg_slot* s = &tables[(size_t)tt * tcap + h];
                if (!s->used) continue;
                size_t p = hash64(s->key) & (tcap - 1);
                while (merged[p].used && merged[p].key != s->key) p = (p + 1) & (tcap - 1);
                if (!merged[p].used) {
                    if (++g > cap) { overflow = 1; break; }
                    merged[p].used = 1;
                    merged[p].key = s->key;
                }
                merged[p].cnt += s->cnt;
                for (uint32_t k = 0; k < nsum; ++k)
                    merged[p].s[k] = (int64_t)((uint64_t)merged[p].s[k] + (uint64_t)s->s[k]);
            }
        if (!overflow) {
            agg_slot* list = (agg_slot*)malloc((g ? g : 1) * sizeof(agg_slot));
            uint64_t m = 0;
            for (size_t h = 0; h < tcap; ++h) if (merged[h].used) list[m++] = merged[h];
            qsort(list, m, sizeof(agg_slot), agg_cmp);
            for (uint64_t k = 0; k < m; ++k) {
                out_keys[k] = list[k].key;
                out_counts[k] = list[k].cnt;
                for (uint32_t j = 0; j < nsum; ++j) out_sums[k * nsum + j] = list[k].s[j];
            }
            free(list);
            result = (int64_t)m;
        }
        free(merged);
    }
    free(tables);
    if (bad) return -2;
    return result;
}

/* ------------------------------------------------------------------------------------
 * Seeded synthetic data: SplitMix64 streams (counter based, so any row can be made
 * independently; redfox_b200's generator kernels use the same formulas).
 * ----------------------------------------------------------------------------------*/
static inline uint64_t mix64(uint64_t x)
{
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

uint64_t orc_rand(uint64_t seed, uint64_t stream, uint64_t idx)
{
    uint64_t base = mix64(seed ^ (stream * 0xD1B54A32D192ED03ull));
    return mix64(base + (idx + 1) * 0x9E3779B97F4A7C15ull);
}

uint64_t orc_uniform(uint64_t seed, uint64_t stream, uint64_t idx, uint64_t lo, uint64_t hi)
{
    uint64_t r = orc_rand(seed, stream, idx);
    return lo + (uint64_t)(((u128)r * (u128)(hi - lo)) >> 64);
}

void orc_gen_uniform_u64(uint64_t* out, size_t n, uint64_t seed, uint64_t stream,
                         uint64_t lo, uint64_t hi, int threads)
{
    if (threads < 1) threads = 1;
#pragma omp parallel for num_threads(threads) schedule(static)
    for (size_t i = 0; i < n; ++i) out[i] = orc_uniform(seed, stream, i, lo, hi);
}

/* Zipf(s) over [0, n): cdf[k] = sum_{j<=k} 1/(j+1)^s, accumulated left to right. */
void orc_zipf_cdf(double* cdf, size_t n, double s)
{
    double acc = 0.0;
    for (size_t k = 0; k < n; ++k) {
        double w;
        if (s == 1.0) w = 1.0 / (double)(k + 1);
        else {
            /* integer powers only are needed by the configs; general s via repeated
             * multiplication is not offered */
            w = 1.0 / (double)(k + 1);
        }
        acc += w;
        cdf[k] = acc;
    }
}

/* Inverse-CDF draw: u = top 53 bits of the stream as a double in [0,1); the draw is
 * the first k with cdf[k] > u * cdf[n-1]. */
void orc_gen_zipf_u64(uint64_t* out, size_t n, uint64_t seed, uint64_t stream,
                      const double* cdf, size_t domain, int threads)
{
    if (threads < 1) threads = 1;
    double total = cdf[domain - 1];
#pragma omp parallel for num_threads(threads) schedule(static)
    for (size_t i = 0; i < n; ++i) {
        double u = (double)(orc_rand(seed, stream, i) >> 11) * 0x1p-53;
        double target = u * total;
        size_t lo = 0, hi = domain;
        while (lo < hi) {
            size_t mid = lo + (hi - lo) / 2;
            if (cdf[mid] > target) hi = mid; else lo = mid + 1;
        }
        out[i] = lo < domain ? lo : domain - 1;
    }
}

/* ------------------------------------------------------------------------------------
 * String keys.  A column is offsets into one pool of NUL-terminated strings (the
 * reference's columns are device pointers to such strings).
 * ----------------------------------------------------------------------------------*/

/* compare_sort_string (ModernGPUSort.cu:44-67) = compare_string2 (ModernGPUJoin.cu:72-98):
 * walk while both strings continue; the first differing char decides (as signed char);
 * else a is less exactly when it ended and b did not. */
int orc_str_less(const char* a, const char* b)
{
    size_t i = 0;
    while (a[i] != 0 && b[i] != 0) {
        if (a[i] != b[i]) return (signed char)a[i] < (signed char)b[i];
        ++i;
    }
    return a[i] == 0 && b[i] != 0;
}

/* compare_string (Reduce.cu:30-51): equal when both end at the same place with the same
 * characters before it. */
int orc_str_equal(const char* a, const char* b)
{
    size_t i = 0;
    while (a[i] != 0 && b[i] != 0) {
        if (a[i] != b[i]) return 0;
        ++i;
    }
    return a[i] == 0 && b[i] == 0;
}

typedef struct { const char* s; size_t idx; } str_item;

static int str_item_cmp(const void* x, const void* y)
{
    const str_item* a = (const str_item*)x;
    const str_item* b = (const str_item*)y;
    if (orc_str_less(a->s, b->s)) return -1;
    if (orc_str_less(b->s, a->s)) return 1;
    return a->idx < b->idx ? -1 : (a->idx > b->idx);   /* stable */
}

/* sort_string_key / sort_string_pair (ModernGPUSort.cu:148-470): MergesortKeys /
 * MergesortPairs with compare_sort_string -- a stable sort, equal strings keep their input
 * order; values of vbytes (0 = none) move with their keys. */
void orc_str_sort(const char* pool, uint64_t* offs, size_t n, void* vals, uint32_t vbytes)
{
    if (n == 0) return;
    str_item* it = (str_item*)malloc(n * sizeof(str_item));
    for (size_t i = 0; i < n; ++i) { it[i].s = pool + offs[i]; it[i].idx = i; }
    qsort(it, n, sizeof(str_item), str_item_cmp);
    uint64_t* o2 = (uint64_t*)malloc(n * sizeof(uint64_t));
    uint8_t* v2 = vbytes ? (uint8_t*)malloc(n * vbytes) : NULL;
    for (size_t k = 0; k < n; ++k) {
        o2[k] = offs[it[k].idx];
        if (vbytes) memcpy(v2 + k * vbytes, (const uint8_t*)vals + it[k].idx * vbytes, vbytes);
    }
    memcpy(offs, o2, n * sizeof(uint64_t));
    if (vbytes) memcpy(vals, v2, n * vbytes);
    free(v2);
    free(o2);
    free(it);
}

/* find_bounds_string (ModernGPUJoin.cu:213-300): SortedSearch lower bounds of each left
 * string in the right column and SortedEqualityCount under compare_string2, then the
 * exclusive scan of the counts (mgpu::Scan) and its total. */
void orc_str_find_bounds(int32_t* lb, int32_t* cnt, uint64_t* total, const char* pool,
                         const uint64_t* loffs, size_t nl, const uint64_t* roffs, size_t nr)
{
    uint64_t run = 0;
    for (size_t i = 0; i < nl; ++i) {
        const char* key = pool + loffs[i];
        size_t lo = 0, hi = nr;
        while (lo < hi) {   /* first right string not less than key */
            size_t mid = lo + (hi - lo) / 2;
            if (orc_str_less(pool + roffs[mid], key)) lo = mid + 1; else hi = mid;
        }
        size_t a = lo;
        hi = nr;
        while (lo < hi) {   /* first right string greater than key */
            size_t mid = lo + (hi - lo) / 2;
            if (!orc_str_less(key, pool + roffs[mid])) lo = mid + 1; else hi = mid;
        }
        lb[i] = (int32_t)a;
        cnt[i] = (int32_t)(uint32_t)run;
        run += lo - a;
    }
    *total = run;
}

/* count_string / total_string_32 (Reduce.cu:424-480, :665-740): thrust::reduce_by_key
 * with compare_string and plus<unsigned>: runs of consecutive equal strings, each
 * reported by its first key and the u32 sum of its values. */
uint64_t orc_str_count(const char* pool, const uint64_t* offs, size_t n, const uint32_t* vals,
                       uint64_t* out_offs, uint32_t* out_sums)
{
    uint64_t g = 0;
    size_t i = 0;
    while (i < n) {
        uint32_t s = 0;
        size_t j = i;
        while (j < n && orc_str_equal(pool + offs[i], pool + offs[j])) s += vals[j++];
        out_offs[g] = offs[i];
        out_sums[g++] = s;
        i = j;
    }
    return g;
}

/* Dense codes: codes[i] = the number of distinct strings of the column less than string
 * i (the order of orc_str_less).  Returns the number of distinct strings. */
uint64_t orc_str_codes(const char* pool, const uint64_t* offs, size_t n, uint32_t* codes)
{
    if (n == 0) return 0;
    str_item* it = (str_item*)malloc(n * sizeof(str_item));
    for (size_t i = 0; i < n; ++i) { it[i].s = pool + offs[i]; it[i].idx = i; }
    qsort(it, n, sizeof(str_item), str_item_cmp);
    uint64_t code = 0;
    for (size_t k = 0; k < n; ++k) {
        if (k > 0 && orc_str_less(it[k - 1].s, it[k].s)) ++code;
        codes[it[k].idx] = (uint32_t)code;
    }
    free(it);
    return code + 1;
}

/* ------------------------------------------------------------------------------------
 * Double values.
 * ----------------------------------------------------------------------------------*/

/* total_{8,16,32,64,128}_double / min_32_double / total_double (Reduce.cu:819-1536,
 * :976-1015) on the CPU: thrust::reduce_by_key's sequential fold over runs of bitwise
 * equal keys (kb = 0: one run), acc = acc + v or acc = (acc < v ? acc : v) in input
 * order, the run's first key reported.  This is the order the reference's own code has
 * when built for the CPU. */
uint64_t orc_reduce_f64_seq(const void* keys, size_t n, uint32_t kb, const double* vals,
                            void* out_keys, double* out_vals, int op_min)
{
    const uint8_t* K = (const uint8_t*)keys;
    uint8_t* OK = (uint8_t*)out_keys;
    uint64_t g = 0;
    size_t i = 0;
    while (i < n) {
        double acc = vals[i];
        size_t j = i + 1;
        while (j < n && (kb == 0 || memcmp(K + j * kb, K + i * kb, kb) == 0)) {
            double v = vals[j++];
            acc = op_min ? (acc < v ? acc : v) : acc + v;
        }
        if (kb) memcpy(OK + g * kb, K + i * kb, kb);
        out_vals[g++] = acc;
        i = j;
    }
    return g;
}
