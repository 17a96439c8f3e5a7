// sort_k16.cu -- radix sort instantiations for 16-byte keys.
#include "sort_launch.cuh"
namespace rfx {
RFX_INSTANTIATE_SORT(16)
}  // namespace rfx
