// redfox_b40c.cpp -- libredfox_b40c.so: redfox::sort_pair / sort_key with the signatures
// of redfox/ra/interface/b40cSort.h:15,17 (key_bits = bits of the key to sort on, the
// fifth sort_pair argument = the value's DataType code as the generated wrapper passes
// it), forwarding to rfx_b40c_sort_pair / rfx_b40c_sort_key.  The moderngpu sort has the
// same C++ signatures with another meaning, so it lives in libredfox_mgpu.so, as the two
// lived in separate kernel libraries in the reference.
#include "shim_common.h"

using redfox_shim::report;

namespace redfox {

void sort_pair(void* key_begin, void* value_begin, unsigned long long int size, unsigned long long int key_bits,
               unsigned long long int value_size) {
  report("sort_pair (b40c)", rfx_b40c_sort_pair(key_begin, value_begin, size, key_bits, value_size));
}

void sort_key(void* key_begin, unsigned long long int size, unsigned long long int bits) {
  report("sort_key (b40c)", rfx_b40c_sort_key(key_begin, size, bits));
}

}  // namespace redfox
