/*
 * ref_driver.cpp -- C entry points into the reference's own code, compiled for the CPU.
 *
 * Built by oracle/Makefile (target `ref`) into oracle/_ref/libredfox_ref.so together
 * with the reference's Union.cu, Difference.cu, Unique.cu, Reduce.cu and Sort.cu (thrust
 * 1.7, CPP device system) and its Tuple.h / Comparisons.h / Project.h headers, read in
 * place from the reference tree.  Test infrastructure: it cross-checks the oracle and
 * is the `reference` CPU arm of bench.py; the product never links it.
 */
#include "cuda_stub.h"

#include <redfox/ra/interface/Tuple.h>
#include <redfox/ra/interface/Comparisons.h>
#include <redfox/ra/interface/Project.h>
#include <redfox/ra/interface/Union.h>
#include <redfox/ra/interface/Unique.h>
#include <redfox/ra/interface/Reduce.h>
#include <redfox/ra/interface/Sort.h>

#include <thrust/sort.h>
#include <thrust/reduce.h>
#include <thrust/set_operations.h>
#include <thrust/host_vector.h>

#include <cstdint>
#include <vector>

/* Difference.h and Union.h share one include guard, so declare the entry here
 * (Difference.h:13-14). */
namespace redfox {
extern void difference(void* result, unsigned long long int* size, void* lbegin, void* lend,
                       void* rbegin, void* rend, unsigned int type);
}

using namespace ra::tuple;

/* ---- packing through the reference's insert/extract ---- */
template <typename T, unsigned I>
static void pack_field(typename T::BasicType& e, const uint64_t* const* cols, size_t i)
{
    if (I < 16 && BitsAt<(I < 16 ? I : 15), T>::value > 0)
        e = insert<unsigned long long, (I < 16 ? I : 15), T>(e, (unsigned long long)cols[I][i]);
}
template <typename T, unsigned I>
static void unpack_field(const typename T::BasicType& e, uint64_t* const* cols, size_t i)
{
    if (I < 16 && BitsAt<(I < 16 ? I : 15), T>::value > 0)
        cols[I][i] = (uint64_t)extract<unsigned long long, (I < 16 ? I : 15), T>(e);
}
template <typename T, unsigned N>
static void pack_rows(uint8_t* out, size_t n, const uint64_t* const* cols)
{
    typedef typename T::BasicType B;
    for (size_t i = 0; i < n; ++i) {
        B e = 0;
        pack_field<T, 0>(e, cols, i);
        if (N > 1) pack_field<T, 1>(e, cols, i);
        if (N > 2) pack_field<T, 2>(e, cols, i);
        if (N > 3) pack_field<T, 3>(e, cols, i);
        if (N > 4) pack_field<T, 4>(e, cols, i);
        if (N > 5) pack_field<T, 5>(e, cols, i);
        if (N > 6) pack_field<T, 6>(e, cols, i);
        if (N > 7) pack_field<T, 7>(e, cols, i);
        if (N > 8) pack_field<T, 8>(e, cols, i);
        std::memcpy(out + i * sizeof(B), &e, sizeof(B));
    }
}
template <typename T, unsigned N>
static void unpack_rows(const uint8_t* in, size_t n, uint64_t* const* cols)
{
    typedef typename T::BasicType B;
    for (size_t i = 0; i < n; ++i) {
        B e;
        std::memcpy(&e, in + i * sizeof(B), sizeof(B));
        unpack_field<T, 0>(e, cols, i);
        if (N > 1) unpack_field<T, 1>(e, cols, i);
        if (N > 2) unpack_field<T, 2>(e, cols, i);
        if (N > 3) unpack_field<T, 3>(e, cols, i);
        if (N > 4) unpack_field<T, 4>(e, cols, i);
        if (N > 5) unpack_field<T, 5>(e, cols, i);
        if (N > 6) unpack_field<T, 6>(e, cols, i);
        if (N > 7) unpack_field<T, 7>(e, cols, i);
        if (N > 8) unpack_field<T, 8>(e, cols, i);
    }
}

typedef Tuple<32, 32> T_32_32;
typedef Tuple<16, 16> T_16_16;
typedef Tuple<32, 64> T_32_64;
typedef Tuple<32, 8> T_32_8;
typedef Tuple<32, 32, 32> T_32_32_32;
typedef Tuple<32, 64, 64, 64, 64, 8, 8> T_fact;
typedef Tuple<32, 64, 64, 64, 64, 8, 8, 64> T_fact_a1;
typedef Tuple<32, 64, 64, 64, 64, 8, 8, 64, 64> T_fact_a2;
typedef Tuple<8, 8, 64, 64> T_proj;
typedef Tuple<3, 14, 23, 5, 19> T_odd;
typedef Tuple<7, 33, 64, 40, 21> T_wide;

#define REF_CODEC(name, T, N)                                                            \
    extern "C" void ref_pack_##name(uint8_t* out, size_t n, const uint64_t* const* cols) \
    { pack_rows<T, N>(out, n, cols); }                                                   \
    extern "C" void ref_unpack_##name(const uint8_t* in, size_t n, uint64_t* const* cols) \
    { unpack_rows<T, N>(in, n, cols); }                                                  \
    extern "C" unsigned ref_bytes_##name(void) { return (unsigned)sizeof(T::BasicType); }

REF_CODEC(32_32, T_32_32, 2)
REF_CODEC(16_16, T_16_16, 2)
REF_CODEC(32_64, T_32_64, 2)
REF_CODEC(32_8, T_32_8, 2)
REF_CODEC(32_32_32, T_32_32_32, 3)
REF_CODEC(fact, T_fact, 7)
REF_CODEC(fact_a2, T_fact_a2, 9)
REF_CODEC(proj, T_proj, 4)
REF_CODEC(odd, T_odd, 5)
REF_CODEC(wide, T_wide, 5)

/* ---- the reference's thrust entry points (Union.cu, Difference.cu, Unique.cu, Sort.cu) ---- */
extern "C" uint64_t ref_set_union(void* out, void* a, size_t na, void* b, size_t nb, unsigned esize, unsigned type)
{
    unsigned long long size = 0;
    redfox::set_union(out, &size, a, (char*)a + na * esize, b, (char*)b + nb * esize, type);
    return size / esize;
}
extern "C" uint64_t ref_difference(void* out, void* a, size_t na, void* b, size_t nb, unsigned esize, unsigned type)
{
    unsigned long long size = 0;
    redfox::difference(out, &size, a, (char*)a + na * esize, b, (char*)b + nb * esize, type);
    return size / esize;
}
/* Set intersection has no reference entry (RelationalAlgebraKernel.cpp:919-922); this is
 * the vendored thrust algorithm the other set entries use, on the same element types. */
extern "C" uint64_t ref_intersection_u32(uint32_t* out, const uint32_t* a, size_t na, const uint32_t* b, size_t nb)
{
    return (uint64_t)(thrust::set_intersection(a, a + na, b, b + nb, out) - out);
}
extern "C" uint64_t ref_unique(void* data, size_t n, unsigned esize, unsigned type)
{
    unsigned long long size = n * esize;
    redfox::unique(data, &size, type);
    return size / esize;
}
extern "C" void ref_sort(void* data, size_t n, unsigned esize, unsigned type)
{
    redfox::sort(data, (char*)data + n * esize, type);
}

/* ---- Reduce.cu entry points (byte sizes in and out, as the reference passes them) ---- */
#define REF_REDUCE(fn, kbytes, vbytes)                                                     \
    extern "C" uint64_t ref_##fn(const void* k, const void* v, void* ok, void* ov, size_t n) \
    {                                                                                      \
        unsigned long long ks = n * kbytes, vs = n * vbytes;                              \
        redfox::fn(k, v, ok, ov, &ks, &vs);                                               \
        return ks / kbytes;                                                               \
    }
REF_REDUCE(count_8, 1, 4)
REF_REDUCE(count_16, 2, 4)
REF_REDUCE(count_32, 4, 4)
REF_REDUCE(count_128, 16, 4)
REF_REDUCE(total_64_32, 8, 4)

/* ---- double values (thrust::reduce_by_key / reduce with plus / minimum<double>) ---- */
REF_REDUCE(total_8_double, 1, 8)
REF_REDUCE(total_16_double, 2, 8)
REF_REDUCE(total_32_double, 4, 8)
REF_REDUCE(total_64_double, 8, 8)
REF_REDUCE(total_128_double, 16, 8)
REF_REDUCE(total_string_double, 8, 8)
REF_REDUCE(min_32_double, 4, 8)
extern "C" double ref_total_double(const double* v, size_t n)
{
    double r = 0;
    redfox::total_double(&r, v, v + n);
    return r;
}
extern "C" uint64_t ref_max_double(const double* v, size_t n)
{
    unsigned long long r = 0;
    redfox::max_double(&r, v, v + n);
    return r;
}
extern "C" uint32_t ref_count(const uint32_t* v, size_t n)
{
    unsigned int r = 0;
    redfox::count(&r, v, v + n);
    return r;
}

/* ---- string keys: columns of pointers to NUL-terminated strings (host pointers here) ---- */
REF_REDUCE(count_string, 8, 4)
REF_REDUCE(total_string_32, 8, 4)
extern "C" void ref_sort_string(uint64_t* keys, size_t n)
{
    redfox::sort_string(keys, keys + n);
}

/* thrust::reduce_by_key with plus<long long>: the algorithm of every Reduce.cu entry,
 * at the int64 value type the build adds (the reference has only double / u32 sums). */
extern "C" uint64_t ref_reduce_sum_i64_u32(const uint32_t* k, const int64_t* v, uint32_t* ok, int64_t* ov, size_t n)
{
    return (uint64_t)(thrust::reduce_by_key(k, k + n, v, ok, ov).first - ok);
}
extern "C" uint64_t ref_reduce_sum_i64_u64(const uint64_t* k, const int64_t* v, uint64_t* ok, int64_t* ov, size_t n)
{
    return (uint64_t)(thrust::reduce_by_key(k, k + n, v, ok, ov).first - ok);
}

/* ---- the filter-project-aggregate plan over Tuple<32,64,64,64,64,8,8> written with the
 * reference's own device code paths on the host: select_field_constant's comparison
 * functor (Select.h:30-114, Comparisons.h le), the set_arith bodies the generator emits
 * (RelationalAlgebraKernel.cpp:2130-2150), permuteElement (Project.h:58-100), then a
 * stable sort_pair by the (f1, f2) key and reduce_by_key / count (Reduce.cu) with exact
 * int64 sums.  Returns the number of groups. */
extern "C" int64_t ref_fact_plan(const uint8_t* in, size_t n, unsigned cutoff,
                                 uint64_t* out_keys, int64_t* out_s1, int64_t* out_s2,
                                 uint64_t* out_cnt)
{
    typedef T_fact::BasicType Row;
    typedef T_fact_a1::BasicType Row1;
    typedef T_fact_a2::BasicType Row2;
    typedef T_proj::BasicType Proj;
    std::vector<uint16_t> keys;
    std::vector<int64_t> s1, s2;
    keys.reserve(n);
    s1.reserve(n);
    s2.reserve(n);
    const Row* rows = (const Row*)in;
    ra::comparisons::le<unsigned int> le;
    for (size_t i = 0; i < n; ++i) {
        Row r = rows[i];
        unsigned int date = extract<unsigned int, 0, T_fact>(r);
        if (!le(date, (unsigned int)cutoff)) continue;
        /* arith 1: price * (100 - disc) appended as field 7 */
        Row1 a1 = (Row1)r << (unsigned int)64;
        unsigned long long p1 = (extract<unsigned long long, 2, T_fact>(r)
                                 * (100 - extract<unsigned long long, 3, T_fact>(r)));
        a1 = insert<unsigned long long, 7, T_fact_a1>(a1, p1);
        /* arith 2: price * (100 - disc) * (100 + tax) appended as field 8 */
        Row2 a2 = (Row2)a1 << (unsigned int)64;
        unsigned long long p2 = ((extract<unsigned long long, 2, T_fact_a1>(a1)
                                  * (100 - extract<unsigned long long, 3, T_fact_a1>(a1)))
                                 * (100 + extract<unsigned long long, 4, T_fact_a1>(a1)));
        a2 = insert<unsigned long long, 8, T_fact_a2>(a2, p2);
        /* project (f1, f2, p1, p2) */
        Proj p;
        ra::cuda::permuteElement<T_fact_a2, T_proj,
            ra::cuda::PermuteMap<5, 6, 7, 8, 100, 100, 100, 100, 100, 100, 100, 100, 100, 100, 100, 100> >(p, a2);
        keys.push_back((uint16_t)(extract<unsigned long long, 0, T_proj>(p) << 8
                                  | extract<unsigned long long, 1, T_proj>(p)));
        s1.push_back((int64_t)extract<unsigned long long, 2, T_proj>(p));
        s2.push_back((int64_t)extract<unsigned long long, 3, T_proj>(p));
    }
    size_t m = keys.size();
    std::vector<uint32_t> perm(m);
    for (size_t i = 0; i < m; ++i) perm[i] = (uint32_t)i;
    std::vector<uint16_t> skeys(keys);
    thrust::stable_sort_by_key(skeys.begin(), skeys.end(), perm.begin());
    std::vector<int64_t> v1(m), v2(m);
    std::vector<uint32_t> ones(m, 1u);
    for (size_t i = 0; i < m; ++i) {
        v1[i] = s1[perm[i]];
        v2[i] = s2[perm[i]];
    }
    std::vector<uint16_t> ok(m + 1);
    std::vector<int64_t> o1(m + 1), o2(m + 1);
    std::vector<uint32_t> oc(m + 1);
    size_t g = thrust::reduce_by_key(skeys.begin(), skeys.end(), v1.begin(), ok.begin(), o1.begin()).first - ok.begin();
    thrust::reduce_by_key(skeys.begin(), skeys.end(), v2.begin(), ok.begin(), o2.begin());
    thrust::reduce_by_key(skeys.begin(), skeys.end(), ones.begin(), ok.begin(), oc.begin());
    for (size_t i = 0; i < g; ++i) {
        out_keys[i] = ok[i];
        out_s1[i] = o1[i];
        out_s2[i] = o2[i];
        out_cnt[i] = oc[i];
    }
    return (int64_t)g;
}
