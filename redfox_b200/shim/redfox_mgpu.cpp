// redfox_mgpu.cpp -- libredfox_mgpu.so: redfox::sort_pair / sort_key with the signatures
// of redfox/ra/interface/ModernGPUSort.h:15,17 (key_type = the key's DataType code, the
// fifth sort_pair argument = the value's DataType code), forwarding to
// rfx_mgpu_sort_pair / rfx_mgpu_sort_key.
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

}  // namespace redfox
