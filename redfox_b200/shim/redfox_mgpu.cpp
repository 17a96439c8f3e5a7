// redfox_mgpu.cpp -- libredfox_mgpu.so: redfox::sort_pair / sort_key / sort_string_pair /
// sort_string_key with the signatures of redfox/ra/interface/ModernGPUSort.h:15-18
// (key_type = the key's DataType code, the fifth sort_pair argument = the value's DataType
// code), forwarding to rfx_mgpu_sort_pair / rfx_mgpu_sort_key / rfx_sort_string_compat.
#include "shim_common.h"

using redfox_shim::report;

namespace redfox {

void sort_pair(void* key_begin, void* value_begin, unsigned long long int size, unsigned long long int key_type,
               unsigned long long int value_size) {
  report("sort_pair (moderngpu)", rfx_mgpu_sort_pair(key_begin, value_begin, size, key_type, value_size));
}

void sort_key(void* key_begin, unsigned long long int size, unsigned long long int type) {
  report("sort_key (moderngpu)", rfx_mgpu_sort_key(key_begin, size, type));
}

// string keys (device pointers to NUL-terminated strings); key_type / type are unused
// by the reference too
void sort_string_pair(void* key_begin, void* value_begin, unsigned long long int size, unsigned long long int,
                      unsigned long long int value_type) {
  report("sort_string_pair", rfx_sort_string_compat(key_begin, value_begin, size, value_type));
}

void sort_string_key(void* key_begin, unsigned long long int size, unsigned long long int) {
  report("sort_string_key", rfx_sort_string_compat(key_begin, nullptr, size, 0));
}

}  // namespace redfox
