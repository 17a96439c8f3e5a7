// sort_k32.cu -- radix sort instantiations for 32-byte keys.
#include "sort_launch.cuh"
namespace rfx {
RFX_INSTANTIATE_SORT(32)
}  // namespace rfx
