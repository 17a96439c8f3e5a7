// sort_k64.cu -- radix sort instantiations for 64-byte keys.
#include "sort_launch.cuh"
namespace rfx {
RFX_INSTANTIATE_SORT(64)
}  // namespace rfx
