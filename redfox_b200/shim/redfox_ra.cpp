// redfox_ra.cpp -- libredfox_ra.so: the reference's redfox:: entry points for joins,
// reductions and set operations, with its C++ linkage and signatures
// (redfox/ra/interface/ModernGPUJoin.h:15-41, Reduce.h:43-158, Union.h:13,
// Difference.h:13, Unique.h:15, Sort.h:15-17), each forwarding to the rfx_*_compat entry of librfx.so
// that keeps the reference's argument meaning (element counts for find_bounds / join, byte
// counts for reduce / count / set operations, device-resident result sizes, synchronous
// on the default stream).  A generated extern "C" wrapper of the reference links against
// this library unchanged.
#include <cstdint>

#include "shim_common.h"

using redfox_shim::report;

namespace redfox {

#define RFX_SHIM_FIND_BOUNDS(W, BYTES)                                                                    \
  void find_bounds_##W(void* lower_bound, void* left_count, unsigned long long int* result_size,         \
                       void* left_key, unsigned long long int left_size, void* right_key,                \
                       unsigned long long int right_size) {                                               \
    report("find_bounds_" #W,                                                                             \
           rfx_find_bounds_compat(static_cast<int32_t*>(lower_bound), static_cast<int32_t*>(left_count), \
                                  reinterpret_cast<uint64_t*>(result_size), left_key, left_size, right_key,  \
                                  right_size, BYTES));                                                    \
  }

RFX_SHIM_FIND_BOUNDS(8, 1)
RFX_SHIM_FIND_BOUNDS(16, 2)
RFX_SHIM_FIND_BOUNDS(32, 4)
RFX_SHIM_FIND_BOUNDS(64, 8)
RFX_SHIM_FIND_BOUNDS(128, 16)
#undef RFX_SHIM_FIND_BOUNDS

void join(int* left_indices, int* right_indices, unsigned long long int result_size, int* lowerBound,
          int* leftCount, unsigned long long int input_size) {
  report("join", rfx_join_compat(left_indices, right_indices, result_size, lowerBound, leftCount, input_size));
}

#define RFX_SHIM_COUNT(W, BYTES)                                                                          \
  void count_##W(const void* key_begin, const void* value_begin, void* result_key_begin,                 \
                 void* result_value_begin, unsigned long long int* key_size,                             \
                 unsigned long long int* value_size) {                                                   \
    report("count_" #W, rfx_count_compat(key_begin, value_begin, result_key_begin, result_value_begin,   \
                                         reinterpret_cast<uint64_t*>(key_size),                         \
                                         reinterpret_cast<uint64_t*>(value_size), BYTES));               \
  }

RFX_SHIM_COUNT(8, 1)
RFX_SHIM_COUNT(16, 2)
RFX_SHIM_COUNT(32, 4)
RFX_SHIM_COUNT(128, 16)
RFX_SHIM_COUNT(256, 32)
#undef RFX_SHIM_COUNT

void total_64_32(const void* key_begin, const void* value_begin, void* result_key_begin, void* result_value_begin,
                 unsigned long long int* key_size, unsigned long long int* value_size) {
  report("total_64_32", rfx_total_64_32_compat(key_begin, value_begin, result_key_begin, result_value_begin,
                                               reinterpret_cast<uint64_t*>(key_size),
                                               reinterpret_cast<uint64_t*>(value_size)));
}

void set_union(void* result, unsigned long long int* size, void* lbegin, void* lend, void* rbegin, void* rend,
               unsigned int type) {
  report("set_union",
         rfx_set_union_compat(result, reinterpret_cast<uint64_t*>(size), lbegin, lend, rbegin, rend, type));
}

void difference(void* result, unsigned long long int* size, void* lbegin, void* lend, void* rbegin, void* rend,
                unsigned int type) {
  report("difference",
         rfx_difference_compat(result, reinterpret_cast<uint64_t*>(size), lbegin, lend, rbegin, rend, type));
}

void unique(void* begin, unsigned long long int* size, unsigned long long int type) {
  report("unique", rfx_unique_compat(begin, reinterpret_cast<uint64_t*>(size), type));
}

// double values (Reduce.h:85-158): exact sums rounded once, the minimum as the
// reference's fold, max_double / count as the reference reduces them
#define RFX_SHIM_TOTAL_DOUBLE(W, BYTES)                                                                    \
  void total_##W##_double(const void* key_begin, const void* value_begin, void* result_key_begin,         \
                          void* result_value_begin, unsigned long long int* key_size,                     \
                          unsigned long long int* value_size) {                                           \
    report("total_" #W "_double",                                                                          \
           rfx_total_double_compat(key_begin, value_begin, result_key_begin, result_value_begin,          \
                                   reinterpret_cast<uint64_t*>(key_size),                                 \
                                   reinterpret_cast<uint64_t*>(value_size), BYTES));                      \
  }

RFX_SHIM_TOTAL_DOUBLE(8, 1)
RFX_SHIM_TOTAL_DOUBLE(16, 2)
RFX_SHIM_TOTAL_DOUBLE(32, 4)
RFX_SHIM_TOTAL_DOUBLE(64, 8)
RFX_SHIM_TOTAL_DOUBLE(128, 16)
#undef RFX_SHIM_TOTAL_DOUBLE

void total_string_double(const void* key_begin, const void* value_begin, void* result_key_begin,
                         void* result_value_begin, unsigned long long int* key_size,
                         unsigned long long int* value_size) {
  report("total_string_double",
         rfx_total_string_double_compat(key_begin, value_begin, result_key_begin, result_value_begin,
                                        reinterpret_cast<uint64_t*>(key_size),
                                        reinterpret_cast<uint64_t*>(value_size)));
}

void min_32_double(const void* key_begin, const void* value_begin, void* result_key_begin, void* result_value_begin,
                   unsigned long long int* key_size, unsigned long long int* value_size) {
  report("min_32_double", rfx_min_32_double_compat(key_begin, value_begin, result_key_begin, result_value_begin,
                                                   reinterpret_cast<uint64_t*>(key_size),
                                                   reinterpret_cast<uint64_t*>(value_size)));
}

void total_double(void* result, const void* begin, const void* end) {
  report("total_double", rfx_sum_double_compat(result, begin, end));
}

void max_double(void* result, const void* begin, const void* end) {
  report("max_double", rfx_max_double_compat(result, begin, end));
}

void count(void* result, const void* begin, const void* end) {
  report("count", rfx_count_u32_compat(result, begin, end));
}

// string keys: columns of device pointers to NUL-terminated strings
void find_bounds_string(void* lower_bound, void* left_count, unsigned long long int* result_size, void* left_key,
                        unsigned long long int left_size, void* right_key, unsigned long long int right_size) {
  report("find_bounds_string",
         rfx_find_bounds_string_compat(static_cast<int32_t*>(lower_bound), static_cast<int32_t*>(left_count),
                                       reinterpret_cast<uint64_t*>(result_size), left_key, left_size, right_key,
                                       right_size));
}

void count_string(const void* key_begin, const void* value_begin, void* result_key_begin, void* result_value_begin,
                  unsigned long long int* key_size, unsigned long long int* value_size) {
  report("count_string", rfx_count_string_compat(key_begin, value_begin, result_key_begin, result_value_begin,
                                                 reinterpret_cast<uint64_t*>(key_size),
                                                 reinterpret_cast<uint64_t*>(value_size)));
}

// the same computation as count_string in the reference (Reduce.cu:665-740)
void total_string_32(const void* key_begin, const void* value_begin, void* result_key_begin,
                     void* result_value_begin, unsigned long long int* key_size, unsigned long long int* value_size) {
  report("total_string_32", rfx_count_string_compat(key_begin, value_begin, result_key_begin, result_value_begin,
                                                    reinterpret_cast<uint64_t*>(key_size),
                                                    reinterpret_cast<uint64_t*>(value_size)));
}

// Sort.h: whole-key ascending sort of [begin, end) of a DataType (thrust::sort in
// Sort.cu:198-300; keys only, so any correct sort gives the same bytes)
void sort(void* begin, void* end, unsigned long long int type) {
  static const unsigned long long width[] = {0, 1, 2, 4, 8, 16, 32, 64};
  if (type == 0 || type >= sizeof(width) / sizeof(width[0])) {
    report("sort", RFX_ERR_UNSUPPORTED);
    return;
  }
  const unsigned long long bytes = static_cast<char*>(end) - static_cast<char*>(begin);
  report("sort", rfx_mgpu_sort_key(begin, bytes / width[type], type));
}

void sort_string(void* begin, void* end) {
  const unsigned long long bytes = static_cast<char*>(end) - static_cast<char*>(begin);
  report("sort_string", rfx_sort_string_compat(begin, nullptr, bytes / 8, 0));
}

}  // namespace redfox
